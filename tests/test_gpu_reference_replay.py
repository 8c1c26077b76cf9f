"""The reference's own CUDA kernels (oracle/_ref/libhotspin.so, built from the reference
sources) driven through the replay of the Go call sequence, against the FP64 oracle.

This pins the oracle's restatement of every term without a reference golden (long field,
anisotropy, heat stencil, coupling, laser, Drude heat capacity, the LLBar torque with the
reference's cross-product convention) to the reference implementation itself.
"""
import numpy as np
import pytest

from oracle import fields as F
from oracle import replay
from oracle.model import Model, Spec
from tests.gpu_util import rel_err

pytestmark = pytest.mark.gpu

KW = dict(size=(2, 16, 32), cellsize=(4e-9, 4e-9, 4e-9), msat0T0=8e5,
          lex=float(np.sqrt(2 * 1.3e-11 / (F.MU0 * 8e5 ** 2))), gamma_ll=2.2e5, alpha=(0.02, 0.03, 0.04),
          ku=3e4, anis_u=(0.2, 0.3, 1.0), b_ext=(0.01, -0.02, 0.015), demag=True, llb=True, tc=630.0, spin_j=0.5,
          n_spins=8e5 / (2 * F.MUB * 0.5), temperature=300.0, ttm=True, gamma_e=700.0, c_l=3e6, g_ep=6e17,
          k_e=90.0, k_l=0.0, laser_p0=5e20, laser_t0=1e-13, laser_fwhm=1e-13, laser_sigma=30e-9)


@pytest.fixture(scope="module")
def ref(cuda):
    if not replay.available():
        pytest.skip("oracle/_ref/libhotspin.so not built (needs the reference sources)")
    return replay


def test_reference_rhs_matches_oracle(ref, cuda):
    rng = np.random.default_rng(8)
    size = KW["size"]
    m = rng.normal(size=(3,) + size)
    m = m / np.sqrt((m * m).sum(0)) * rng.uniform(0.5, 0.95, size=size)
    Te = rng.uniform(300, 900, size=size)
    Tl = rng.uniform(300, 400, size=size)
    y = {"m": m, "Te": Te, "Tl": Tl}
    want = Model(Spec(**KW)).rhs(0.7e-13, y)
    sim = ref.RefSim(KW, dt=1e-15)
    for k, v in y.items():
        sim.set(k, v)
    out = cuda.zeros_like(sim.y)
    sim.rhs(0.7e-13, sim.y, out)
    got = out.cpu().numpy().reshape((5,) + size)
    assert rel_err(got[:3], want["m"]) < 1e-11
    assert rel_err(got[3], want["Te"]) < 1e-11
    assert rel_err(got[4], want["Tl"]) < 1e-11


def test_reference_dp45_steps_match_oracle(ref, cuda):
    from oracle.solvers import Integrator
    kw = dict(KW, ttm=False, laser_p0=0.0, llb=False, temperature=0.0)
    rng = np.random.default_rng(9)
    m = rng.normal(size=(3,) + kw["size"])
    m /= np.sqrt((m * m).sum(0))
    sim = ref.RefSim(kw, dt=1e-15, rtol=1e-4)
    sim.set("m", m)
    it = Integrator(Model(Spec(**kw)), {"m": m}, "dp45", 1e-15, rtol=1e-4, mindt=1e-20, maxdt=1e-13)
    for _ in range(5):
        sim.step()
        it.step()
    assert sim.t == pytest.approx(it.t, rel=1e-6)
    assert np.abs(sim.get("m") - it.y["m"]).max() < 1e-9
