"""FP64 CPU oracle for the hotspin solver hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, in plain NumPy float64, the arithmetic of hotspin's CUDA kernel
library (``src/libhotspin/*.cu``) and of the Go host code that sequences it
(``src/hotspin-core/modules``, ``src/hotspin-core/engine``).  Every function cites the
reference file:line it follows.

It exists to CHECK the CUDA path in ``hotspin_b200``: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` may import it.
The product path never routes through it and has no CPU fallback.

Pinning: the exchange and demag restatements are checked against the reference's own
golden dumps (``tests/test-exchange/hex_ref*.dump``, ``tests/test-demag/B_ref*.dump``);
subsampled copies of those goldens live in ``tests/golden/`` together with the script
that extracted them.  Other terms (long field, thermal scaling, heat stencils, solvers)
have no reference golden and are pinned by the reference's kernels rebuilt from source
(``oracle/_ref``), run on a B200 by the GPU tests.

Conventions (reference ``engine/api.go:41-62``, ``common/index.go:68-113``): arrays are in
the reference's *program order* -- shape ``(N0, N1, N2)`` with N2 the fastest index, which
is the user's x -- and vector fields are ``(3, N0, N1, N2)`` with component 0 the program X
axis (user z).
"""
import os

# The reference checkout (read by the fixture script, the dump-file test and the build of
# oracle/_ref); HOTSPIN_REF overrides the default location.
REF_ROOT = os.environ.get("HOTSPIN_REF", "/root/reference")
