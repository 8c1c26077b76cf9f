"""Extract subsampled golden fixtures from the reference's test dumps and pin the oracle.

Run in a container that has the reference checkout (``$HOTSPIN_REF``, default ``/root/reference``):

    python tests/golden/make_golden.py

It regenerates the inputs of the reference's script tests exactly as they do
(``tests/test-exchange/cmp-ref*.py``, ``tests/test-demag/cmp-ref*.py``: Python's Mersenne
Twister seeded with 0, loops ``for k: for j: for i:`` over user indices, the exchange test
drawing one extra number per cell in its lex loop), evaluates the oracle on them, compares
against the FULL golden dumps, and writes

* ``golden_subsample.npz`` -- the golden values at 4096 fixed random cells of each dump
  (all three components, float32 as stored), so tests can compare without the reference;
* ``golden_report.json`` -- the oracle-vs-golden errors measured on the full dumps.

Machines without a reference checkout run the tests on these two files alone.
"""
import json
import math
import os
import random
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import REF_ROOT, demag, fields, native  # noqa: E402
from oracle.dump import read_dump  # noqa: E402

REF = os.path.join(REF_ROOT, "tests")
N = 64
MU0_PY = 1.25663706e-6        # the Python client's mu0 (src/python/hotspin.py.tail:4)
CELL_PROGRAM = (64e-9 / N, 160e-9 / N, 320e-9 / N)   # (z, y, x) user -> program order
N_SAMPLE = 4096


def to_program(a):
    """user [x][y][z] -> program [z][y][x]"""
    return np.ascontiguousarray(np.transpose(a, (2, 1, 0)))


def vec_to_program(v):
    """user components (x, y, z) -> program components (z, y, x), each transposed."""
    return np.stack([to_program(v[2]), to_program(v[1]), to_program(v[0])])


def exchange_inputs():
    random.seed(0)
    msk = np.zeros((N, N, N))
    for k in range(N):
        for j in range(N):
            for i in range(N):
                msk[i, j, k] = random.random()
    lex = np.zeros((N, N, N))
    for k in range(N):
        for j in range(N):
            for i in range(N):
                random.random()
                lex[i, j, k] = math.sqrt(1.0 / (msk[i, j, k] ** 2.0))
    m = np.zeros((3, N, N, N))
    for k in range(N):
        for j in range(N):
            for i in range(N):
                a, b, c = random.random(), random.random(), random.random()
                ln = math.sqrt(a ** 2.0 + b ** 2.0 + c ** 2.0)
                m[:, i, j, k] = (a / ln, b / ln, c / ln)
    return to_program(msk), to_program(lex), vec_to_program(m)


def demag_inputs():
    random.seed(0)
    msk = np.zeros((N, N, N))
    for k in range(N):
        for j in range(N):
            for i in range(N):
                msk[i, j, k] = random.random()
    m = np.zeros((3, N, N, N))
    for k in range(N):
        for j in range(N):
            for i in range(N):
                a, b, c = random.random(), random.random(), random.random()
                ln = math.sqrt(a ** 2 + b ** 2 + c ** 2)
                m[:, i, j, k] = (a / ln, b / ln, c / ln)
    return to_program(msk), vec_to_program(m)


def errors(new, ref):
    d = np.abs(new - ref)
    return dict(max_abs=float(d.max()), max_ref=float(np.abs(ref).max()),
                rel_to_max=float(d.max() / np.abs(ref).max()),
                mean_abs_per_cell=float(d.sum(0).mean()))


def main():
    report = {}
    rng = np.random.default_rng(20240601)
    sample = rng.choice(N ** 3, size=N_SAMPLE, replace=False).astype(np.int64)
    out = {"sample_flat_index": sample}

    msk, lex, m = exchange_inputs()
    lex0 = math.sqrt(2 * 1.3e-11 / (MU0_PY * 800e3 * 800e3))
    for tag, pbc in (("", (0, 0, 0)), ("_pbc", (1, 1, 1))):
        ref, _ = read_dump(os.path.join(REF, "test-exchange", "hex_ref%s.dump" % tag))
        for power in (1, 2):
            H = fields.exchange6(m, lex, 800e3, lex0, CELL_PROGRAM, pbc, weight_power=power)
            report["exchange%s_weightpow%d" % (tag, power)] = errors(H, ref)
        out["hex_ref%s" % tag] = ref.reshape(3, -1)[:, sample].astype(np.float32)

    dmsk, dm = demag_inputs()
    for tag, pbc in (("", (0, 0, 0)), ("_pbc", (2, 4, 8))):
        t0 = time.time()
        logic = demag.pad_size([N, N, N], pbc)
        K = native.kernel_arne(logic, CELL_PROGRAM, pbc, 6)
        Kf = demag.kernel_spectrum(K)
        B = demag.demag_field(dm, dmsk, 800e3, Kf, logic)
        ref, _ = read_dump(os.path.join(REF, "test-demag", "B_ref%s.dump" % tag))
        e = errors(B, ref)
        e["seconds"] = time.time() - t0
        report["demag%s" % tag] = e
        out["B_ref%s" % tag] = ref.reshape(3, -1)[:, sample].astype(np.float32)

    np.savez_compressed(os.path.join(HERE, "golden_subsample.npz"), **out)
    with open(os.path.join(HERE, "golden_report.json"), "w") as f:
        json.dump(report, f, indent=1, sort_keys=True)
    print(json.dumps(report, indent=1, sort_keys=True))


if __name__ == "__main__":
    main()
