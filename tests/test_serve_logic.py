"""The continuous-batching loop of loma_phd_b200/serve.py on the CPU, with
fake cases in place of device handles: requests are admitted first come
first served while the memory cap and the slots allow, each advances in
chunks until its steps are done, a finished case frees its slot and bytes
at once, and every request completes with its own step count."""
import itertools

import pytest

from loma_phd_b200 import serve


class FakeCase:
    live = 0
    peak = 0

    def __init__(self, req):
        self.req = req
        self.polls = 0
        self.steps = 0
        self.closed = False
        FakeCase.live += 1
        FakeCase.peak = max(FakeCase.peak, FakeCase.live)

    def step(self, n):
        self.steps += n
        self.polls = 0

    def done(self):
        self.polls += 1
        return self.polls >= 2  # busy for one poll after each chunk

    def diag(self):
        return {"steps": self.steps}

    def get_state(self):
        return {"steps": self.steps}

    def close(self):
        assert not self.closed
        self.closed = True
        FakeCase.live -= 1


@pytest.fixture
def fake(monkeypatch):
    FakeCase.live = FakeCase.peak = 0
    monkeypatch.setattr(serve, "_prepare", lambda req, device: FakeCase(req))
    monkeypatch.setattr(serve, "footprint", lambda p: 1000 + 10 * p.my)
    return FakeCase


def _reqs(n, steps=(5, 17, 40), ny=(33, 65)):
    cyc = itertools.cycle(itertools.product(steps, ny))
    return [serve.RunRequest(rid=i, nx=24, nz=24, ny=y, steps=s, arrival=0.0) for i, (s, y) in zip(range(n), cyc)]


def test_every_request_completes_with_its_steps(fake):
    reqs = _reqs(12)
    out = serve.Server(hbm_cap=10**6, max_active=4, chunk=8, keep_state=True).run(reqs)
    res = out["results"]
    assert [r.rid for r in res] == list(range(12))
    for r, q in zip(res, reqs):
        assert r.diag["steps"] == q.steps and r.state["steps"] == q.steps
    assert out["stats"]["requests"] == 12 and out["stats"]["max_concurrent"] <= 4
    assert fake.live == 0 and fake.peak <= 4


def test_memory_cap_limits_residency(fake):
    reqs = _reqs(9, ny=(65,))
    fp = 1000 + 10 * 65
    out = serve.Server(hbm_cap=3 * fp, max_active=16, chunk=4).run(reqs)
    assert out["stats"]["peak_device_bytes"] <= 3 * fp
    assert fake.peak <= 3
    assert len(out["results"]) == 9


def test_admission_is_first_come_first_served(fake):
    reqs = _reqs(6, steps=(3,), ny=(33,))
    out = serve.Server(hbm_cap=10**6, max_active=1, chunk=8).run(reqs)
    adm = [r.admitted for r in out["results"]]
    assert adm == sorted(adm)


def test_requests_larger_than_the_cap_are_refused(fake):
    with pytest.raises(ValueError):
        serve.Server(hbm_cap=500, max_active=2).run(_reqs(1))
