"""Host logic of the continuous-batching loop, on CPU with a stand-in for the GPU batch."""
import numpy as np
import pytest

from hotspin_b200 import serve


class FakeBatch:
    """Slots advance 1e-12 s of simulated time per launch; results are m0 scaled by the seed."""
    created = []

    def __init__(self, nslot, **cls):
        self.nslot = nslot
        self.cls = cls
        self.slots = {}
        self.closed = False
        self.launches = 0
        FakeBatch.created.append(self)

    @staticmethod
    def footprint(nslot, **cls):
        s = cls["size"]
        return nslot * s[0] * s[1] * s[2] * 100

    def admit(self, slot, m, t_stop, **kw):
        assert slot not in self.slots and 0 <= slot < self.nslot
        self.slots[slot] = dict(m=np.array(m) * kw["seed"], t=0.0, t_stop=t_stop, steps=0)

    def launch(self, graphs=1):
        self.launches += 1
        for s in self.slots.values():
            if s["t"] < s["t_stop"] - 1e-18:
                s["t"] += 1e-12
                s["steps"] += 1

    def poll(self):
        return True

    def slot_status(self, slot):
        s = self.slots[slot]
        return dict(t=s["t"], dt=1e-12, steps=s["steps"], attempts=s["steps"], rejects=0, status=0,
                    active=s["t"] < s["t_stop"] - 1e-18)

    def slot_get(self, slot, name="m"):
        return self.slots.pop(slot)["m"]

    def close(self):
        self.closed = True


@pytest.fixture
def fake(monkeypatch):
    FakeBatch.created = []
    monkeypatch.setattr(serve, "Batch", FakeBatch)
    return FakeBatch


def _reqs(n, sizes, t_ends, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        size = sizes[i % len(sizes)]
        desc = dict(size=size, cellsize=(2e-9,) * 3, pbc=(0, 0, 0), solver="dp45", rtol=1e-5, demag=True,
                    thermal=True, msat0T0=8e5, dt=1e-15, seed=i + 1)
        out.append(serve.Request(i, desc, rng.normal(size=(3,) + size), t_ends[i % len(t_ends)], 0.0))
    return out


def test_every_request_completes_with_its_own_result(fake):
    reqs = _reqs(23, [(1, 32, 32), (2, 64, 64), (1, 128, 128)], [3e-12, 5e-12, 1e-12])
    srv = serve.Server(hbm_budget=1 << 40, cells_per_class=4 * 32 * 32, max_slots=4)
    res = srv.run(reqs, realtime=False)
    assert sorted(res) == list(range(23))
    for r in reqs:
        np.testing.assert_array_equal(res[r.rid].m, r.m0 * r.desc["seed"])
        assert res[r.rid].steps == round(r.t_end / 1e-12)
    # one class per grid size, slots as configured
    assert len(fake.created) == 3
    assert sorted(b.nslot for b in fake.created) == [1, 1, 4]


def test_slots_are_refilled_while_others_run(fake):
    # one class with 2 slots: a long request and a stream of short ones; the short ones
    # flow through the second slot while the long one is still running
    reqs = _reqs(6, [(1, 32, 32)], [10e-12, 1e-12, 1e-12, 1e-12, 1e-12, 1e-12])
    srv = serve.Server(hbm_budget=1 << 40, cells_per_class=2 * 32 * 32, max_slots=2)
    res = srv.run(reqs, realtime=False)
    b = fake.created[0]
    assert b.nslot == 2
    assert res[0].steps == 10
    assert b.launches <= 11
    assert max(res[k].done for k in range(1, 6)) <= res[0].done


def test_admission_by_footprint_evicts_idle_classes(fake):
    reqs = _reqs(4, [(1, 64, 64), (1, 128, 128)], [1e-12])
    one = fake.footprint(1, size=(1, 128, 128))
    srv = serve.Server(hbm_budget=one + 10, cells_per_class=1, max_slots=1)
    res = srv.run(reqs, realtime=False)
    assert sorted(res) == [0, 1, 2, 3]
    assert srv.stats["deferred_by_footprint"] >= 1
    assert srv.used <= srv.hbm_budget
    assert any(b.closed for b in fake.created)


def test_request_above_budget_is_refused(fake):
    reqs = _reqs(1, [(1, 128, 128)], [1e-12])
    srv = serve.Server(hbm_budget=1000, cells_per_class=1, max_slots=1)
    with pytest.raises(ValueError):
        srv.run(reqs, realtime=False)


def test_request_stream_is_seeded_and_in_range():
    a = serve.make_requests(n=40, seed=3)
    b = serve.make_requests(n=40, seed=3)
    assert [r.arrival for r in a] == [r.arrival for r in b]
    for r in a:
        d = r.desc
        assert d["size"][1] == d["size"][2] and d["size"][1] in (32, 64, 128, 256, 512) and d["size"][0] in (1, 2)
        assert 2e-9 <= d["cellsize"][0] <= 5e-9 and 4e5 <= d["msat0T0"] <= 1.2e6
        assert 0.005 <= d["alpha"][0] <= 0.1 and 0 <= d["temperature"] <= 600
        assert np.linalg.norm(d["b_ext"]) <= 0.05 + 1e-12
        lm = np.sqrt((r.m0 ** 2).sum(0))
        want = serve.equilibrium_m_half(d["temperature"], d["tc"]) if d["llb"] else 1.0
        np.testing.assert_allclose(lm, want, rtol=1e-12)
    gaps = np.diff([0.0] + [r.arrival for r in a])
    assert 0.005 < gaps.mean() < 0.05   # mean 1/50 s


def test_equilibrium_m_half():
    for T in (100.0, 300.0, 600.0):
        me = serve.equilibrium_m_half(T, 630.0)
        assert abs(me - np.tanh(me * 630.0 / T)) < 1e-12
