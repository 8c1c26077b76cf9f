"""Batched simulations (hsb_batch_*) and the continuous-batching loop on the GPU.

A slot's trajectory must not depend on the other slots (bit-identical alone and in a mix),
and must match the plain single-simulation handle within 1e-5 max |dm|.
"""
import numpy as np
import pytest

from hotspin_b200 import serve
from hotspin_b200.sim import Batch, Simulation

pytestmark = pytest.mark.gpu

MU0 = 4e-7 * np.pi
MUB = 9.27400968202020202e-24


def _desc(size, cs, ms, alpha, T, b, seed, llb):
    lex = float(np.sqrt(2 * 1.3e-11 / (MU0 * ms * ms)))
    return dict(size=size, cellsize=(cs, cs, cs), pbc=(0, 0, 0), msat0T0=ms, lex=lex, alpha=(alpha,) * 3,
                b_ext=b, demag=True, normalize=not llb, llb=llb, tc=630.0, spin_j=0.5,
                n_spins=ms / (2 * MUB * 0.5), temperature=T, thermal=True, seed=seed, solver="dp45", dt=1e-15,
                rtol=1e-5, mindt=1e-22, maxdt=1e-12)


def _m0(seed, size, length=1.0):
    m = np.random.default_rng(seed).normal(size=(3,) + size)
    return length * m / np.sqrt((m * m).sum(0))


SIZE = (1, 32, 64)
REQS = [
    (_desc(SIZE, 2e-9, 8e5, 0.02, 0.0, (0.0, 0.01, 0.02), 11, False), _m0(1, SIZE), 3e-12),
    (_desc(SIZE, 3.5e-9, 1.1e6, 0.1, 150.0, (0.03, 0.0, 0.0), 12, False), _m0(2, SIZE), 2e-12),
    (_desc(SIZE, 5e-9, 5e5, 0.05, 450.0, (0.0, 0.0, -0.04), 13, True),
     _m0(3, SIZE, serve.equilibrium_m_half(450.0, 630.0)), 2.5e-12),
]
CLASS = serve.class_desc(REQS[0][0])


def _run_batch(nslot, placement):
    """placement: {slot: request index}; returns {request index: (m, status)}."""
    out = {}
    with Batch(nslot, **CLASS) as b:
        for slot, q in placement.items():
            d, m0, t_end = REQS[q]
            b.admit(slot, m0, t_end, **d)
        for _ in range(100000):
            b.launch(1)
            while not b.poll():
                pass
            if not any(b.slot_status(s)["active"] for s in placement):
                break
        for slot, q in placement.items():
            out[q] = (b.slot_get(slot, "m"), b.slot_status(slot))
    return out


def test_batch_slot_alone_equals_mix_bitwise():
    alone = _run_batch(4, {2: 0})
    mix = _run_batch(4, {0: 0, 1: 1, 3: 2})
    m_a, st_a = alone[0]
    m_m, st_m = mix[0]
    assert st_a["steps"] == st_m["steps"] and st_a["attempts"] == st_m["attempts"]
    assert abs(st_a["t"] - REQS[0][2]) < 1e-18
    np.testing.assert_array_equal(m_a, m_m)
    for q in (1, 2):
        assert abs(mix[q][1]["t"] - REQS[q][2]) < 1e-6 * REQS[q][2]


def test_batch_matches_plain_handle():
    mix = _run_batch(3, {0: 0, 1: 1, 2: 2})
    for q, (d, m0, t_end) in enumerate(REQS):
        with Simulation(**d) as sim:
            sim.set("m", m0)
            sim.run_until(t_end)
            m = sim.get("m")
            st = sim.status()
        dm = float(np.abs(mix[q][0] - m).max())
        assert dm <= 1e-5, (q, dm, st, mix[q][1])
        assert st["steps"] == mix[q][1]["steps"]
        assert np.isfinite(mix[q][0]).all()


def test_batch_rejects_other_class():
    with Batch(2, **CLASS) as b:
        d = dict(REQS[0][0], size=(1, 32, 32))
        with pytest.raises(Exception):
            b.admit(0, np.zeros((3, 1, 32, 32)), 1e-12, **d)
        d = dict(REQS[0][0], solver="rk4")
        with pytest.raises(Exception):
            b.admit(0, REQS[0][1], 1e-12, **d)


def test_footprint_grows_per_slot():
    f1 = Batch.footprint(1, **CLASS)
    f8 = Batch.footprint(8, **CLASS)
    assert 4 * f1 < f8 < 8 * f1 + 1
    ncell = int(np.prod(SIZE))
    # DP45 with a thermal field: 2 states + 2 stage points + 7 stages (3 ch) + 3 + 6 demag-field channels
    assert (f8 - f1) / 7 >= 4 * ncell * (6 + 6 + 21 + 3 + 6)


def test_serving_loop_mixed_sizes_same_as_alone():
    reqs = serve.make_requests(n=10, seed=5, t_end=1e-12, sides=(32, 64), layers=(1, 2))
    srv = serve.Server(hbm_budget=8 << 30, cells_per_class=3 * 64 * 64, max_slots=8)
    try:
        mix = srv.run(reqs, realtime=False)
    finally:
        srv.close()
    assert sorted(mix) == list(range(10))
    # alone through the same loop: bit-identical
    for r in reqs[:3]:
        srv1 = serve.Server(hbm_budget=8 << 30, cells_per_class=3 * 64 * 64, max_slots=8)
        try:
            one = srv1.run([r], realtime=False)
        finally:
            srv1.close()
        np.testing.assert_array_equal(one[r.rid].m, mix[r.rid].m)
    # alone on the plain handle: within 1e-5
    plain, _, _ = serve.run_sequential(reqs[:4])
    for rid, res in plain.items():
        assert float(np.abs(res.m - mix[rid].m).max()) <= 1e-5
        assert mix[rid].status == 0
