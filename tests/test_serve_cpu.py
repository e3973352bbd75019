"""The served form's scheduling on the CPU (efs_b200/serve.py): the Server
loop with stand-ins for the CUDA engine and batch, the request stream and
the latency statistics.  The GPU behaviour (each result equal to the same
request alone) is tests/test_gpu_serve.py; here the contract of the loop:
every request runs exactly its step count, member slots and the HBM budget
are respected (a request larger than the budget still runs, alone), arrival
order is kept, and a chunk never runs past the nearest member's end."""
import numpy as np
import pytest

from efs_b200 import serve


class FakeEngine:
    energy_log = []                             # (grid side, reduction used) per retirement
    made = []                                   # every engine constructed

    def __init__(self, device=0):
        self.steps, self.bytes, self.destroyed = 0, 0, False
        self.numLines = [4, 4, 4]
        FakeEngine.made.append(self)

    def initGPU(self):
        return True

    def deviceBytes(self):
        return self.bytes

    def computeEnergy(self, lagged=True):
        FakeEngine.energy_log.append((self.numLines[0], "alloc"))
        return float(self.steps)

    def energyNoAlloc(self):
        FakeEngine.energy_log.append((self.numLines[0], "noalloc"))
        return float(self.steps)

    def destroy(self):
        self.destroyed = True

    def getState(self):
        return {"steps": self.steps}

    def setState(self, blob):
        self.steps = blob["steps"]


class FakeBatch:
    log = []                                    # (members, steps, member bytes) per iterate

    def __init__(self, engines):
        self.engines = list(engines)
        assert len(set(map(id, self.engines))) == len(self.engines)

    def iterate(self, n):
        FakeBatch.log.append((len(self.engines), n, sum(e.bytes for e in self.engines)))
        for e in self.engines:
            assert not e.destroyed
            e.steps += n

    def sync(self):
        pass

    def destroy(self):
        pass


@pytest.fixture
def fake(monkeypatch):
    FakeBatch.log = []
    monkeypatch.setattr(serve, "CudaEngine", FakeEngine)
    monkeypatch.setattr(serve, "CudaBatch", FakeBatch)

    def configure(engine, job):
        live = [e for e in FakeEngine.made if not e.destroyed and e is not engine]
        fail = job.get("fail")                  # "always", or "beside": only while other solves are resident
        if fail == "always" or (fail == "beside" and live):
            fake.configure_failures += 1
            raise serve.EfsError(4, "cudaMalloc failed (fake)")
        engine.bytes = job["bytes"]
        engine.numLines = list(job.get("grid", (4, 4, 4)))
        return None
    monkeypatch.setattr(serve.workloads, "configure", configure)
    FakeEngine.made = []
    fake = FakeBatch
    fake.configure_failures = 0
    return fake


def job(side, nbytes):
    return {"grid": [side, side, side], "bytes": nbytes}


def drain(server, limit=10000):
    for _ in range(limit):
        if not server.round() and not server.waiting and not server.active:
            return
    raise AssertionError("server did not drain")


def test_every_request_runs_its_steps_within_slots(fake):
    s = serve.Server(hbm_budget=1e15, max_members=3, chunk=100)
    steps = [250, 100, 730, 40, 333, 512, 99]
    ids = [s.submit(job(16 + 8 * i, 1000), n, arrival=float(i)) for i, n in enumerate(steps)]
    drain(s)
    assert len(s.finished) == len(steps)
    by_id = {r.rid: r for r in s.finished}
    for rid, n in zip(ids, steps):
        assert by_id[rid].result["energy"] == float(n)           # FakeEngine counts its timesteps
        assert by_id[rid].engine is None
    assert max(m for m, _, _ in fake.log) <= 3
    assert max(n for _, n, _ in fake.log) <= 100
    assert [r.rid for r in sorted(s.finished, key=lambda r: r.admitted)] == ids   # FIFO admission
    assert s.used == 0


def test_chunk_stops_at_the_nearest_end(fake):
    s = serve.Server(hbm_budget=1e15, max_members=4, chunk=256)
    s.submit(job(16, 10), 300, arrival=0.0)
    s.submit(job(16, 10), 70, arrival=0.0)
    s.round()                                    # admits both (nothing was running)
    s.round()
    assert fake.log[0][1] == 70                  # stops where the shorter one ends
    drain(s)
    assert sorted(r.result["energy"] for r in s.finished) == [70.0, 300.0]


def test_hbm_budget(fake):
    est = serve.estimate_bytes(job(64, 0))       # admission is decided on this estimate
    budget = 2.5 * est                           # two 64^3 solves fit, a third does not
    s = serve.Server(hbm_budget=budget, max_members=64, chunk=50)
    for i in range(5):
        s.submit(job(64, est), 120, arrival=float(i))
    big = job(128, 0)
    big["bytes"] = serve.estimate_bytes(big)     # larger than the whole budget
    assert big["bytes"] > budget
    huge = s.submit(big, 60, arrival=10.0)
    drain(s)
    assert len(s.finished) == 6
    assert max(m for m, _, _ in fake.log) == 2
    assert all(used <= budget for m, _, used in fake.log if m > 1)
    lone = [m for m, _, used in fake.log if used > budget]
    assert lone and all(m == 1 for m in lone)    # the oversize request ran, alone
    assert any(r.rid == huge for r in s.finished)
    assert s.used == 0


def test_retirement_energy_does_not_allocate(fake):
    """Retiring a solve reads its energy through the allocation-free entry
    point, so the retirement stays inside the budget the loop accounts for;
    a grid beyond that entry point's fixed scratch (more than 2^30 interior
    cells) uses the allocating reduction."""
    FakeEngine.energy_log = []
    s = serve.Server(hbm_budget=1e15, max_members=4, chunk=64)
    s.submit(job(40, 1000), 10, arrival=0.0)
    s.submit(job(1100, 1000), 10, arrival=0.0)   # 1099^3 > 2^30 interior cells
    drain(s)
    assert sorted(FakeEngine.energy_log) == [(40, "noalloc"), (1100, "alloc")]


def test_eviction_lets_a_short_request_pass(fake):
    """With one member slot, a long solve is evicted (state to the host) when a
    request of at most 1/4 of its remaining steps waits, resumes afterwards
    from its saved state and still runs exactly its step count; without
    eviction the short request waits for the long one."""
    def run(evict):
        s = serve.Server(hbm_budget=1e15, max_members=1, chunk=100, evict_ratio=4.0 if evict else None)
        long_id = s.submit(job(40, 1000), 2000, arrival=0.0)
        s.round()                                  # the long solve is resident
        s.round()
        short_id = s.submit(job(16, 1000), 150, arrival=0.0)
        drain(s)
        by = {r.rid: r for r in s.finished}
        return s, by[long_id], by[short_id]
    s, lng, sht = run(True)
    assert s.evicted == 1 and lng.evictions == 1
    assert lng.result["energy"] == 2000.0 and sht.result["energy"] == 150.0     # exact step counts
    assert sht.done < lng.done                    # the short request finished first
    s0, lng0, sht0 = run(False)
    assert s0.evicted == 0 and sht0.done > lng0.done
    assert s.used == 0


def test_eviction_respects_the_limit_and_ratio(fake):
    s = serve.Server(hbm_budget=1e15, max_members=1, chunk=100, evict_ratio=4.0, max_evictions=1)
    a = s.submit(job(40, 1000), 1000, arrival=0.0)
    s.round()
    s.round()
    s.submit(job(16, 1000), 500, arrival=0.0)     # not short enough: 500 > remaining / 4
    s.submit(job(16, 1000), 50, arrival=0.0)
    drain(s)
    by = {r.rid: r for r in s.finished}
    assert by[a].evictions == 0                   # the head of the queue decides, and it was too long
    s = serve.Server(hbm_budget=1e15, max_members=1, chunk=100, evict_ratio=2.0, max_evictions=1)
    a = s.submit(job(40, 1000), 3000, arrival=0.0)
    s.round()
    for _ in range(3):
        s.submit(job(16, 1000), 100, arrival=0.0)
    drain(s)
    assert s.evicted == 1                         # at most once per solve
    assert {r.rid: r for r in s.finished}[a].result["energy"] == 3000.0


def test_a_request_that_cannot_allocate_alone_fails_cleanly(fake):
    s = serve.Server(hbm_budget=1e15, max_members=4, chunk=100)
    ok1 = s.submit(job(16, 1000), 300, arrival=0.0)
    bad = s.submit(dict(job(24, 1000), fail="always"), 200, arrival=0.0)
    ok2 = s.submit(job(32, 1000), 150, arrival=0.0)
    drain(s)
    assert sorted(r.rid for r in s.finished) == [ok1, ok2]
    assert [r.rid for r in s.failed] == [bad]
    r = s.failed[0]
    assert "EFS_ERR_OOM" in r.result["error"] and r.engine is None and r.done is not None
    assert all(e.destroyed for e in FakeEngine.made)           # the failed engine was freed too
    assert s.used == 0 and not s.waiting and not s.active
    # it failed beside residents first (waits), then alone (fails): two attempts
    assert fake.configure_failures == 2


def test_a_request_that_fails_beside_residents_waits_for_them(fake):
    s = serve.Server(hbm_budget=1e15, max_members=4, chunk=100)
    a = s.submit(job(16, 1000), 1000, arrival=0.0)
    s.round()
    late = s.submit(dict(job(24, 1000), fail="beside"), 250, arrival=0.0)
    b = s.submit(job(16, 1000), 100, arrival=0.0)      # behind it in arrival order
    drain(s)
    assert not s.failed
    by = {r.rid: r for r in s.finished}
    assert set(by) == {a, late, b}
    assert by[late].result["energy"] == 250.0
    assert by[late].admitted >= by[a].done                      # admitted once the resident solve left
    assert by[b].admitted >= by[late].admitted                  # arrival order kept behind it
    # one failed attempt: no retry while the same solves stay resident
    assert fake.configure_failures == 1
    assert s.used == 0 and all(e.destroyed for e in FakeEngine.made)


def test_request_stream_and_latency_stats():
    a = serve.request_stream(5.0, 20.0, seed=4)
    b = serve.request_stream(5.0, 20.0, seed=4)
    assert a == b and 60 <= len(a) <= 140
    t = [x[0] for x in a]
    assert all(0 < u < v for u, v in zip(t, t[1:])) and t[-1] < 20.0
    assert all(s % 8 == 0 and 40 <= s <= 300 for _, _, s, _ in a)
    assert all(5000 <= n <= 25000 for _, _, _, n in a)
    frac = sum(k == "tfsf" for _, k, _, _ in a) / len(a)
    assert 0.1 < frac < 0.5

    class R:
        def __init__(self, arrival, done):
            self.arrival, self.done = arrival, done
    st = serve.latency_stats([R(0.0, float(k)) for k in range(1, 101)])
    assert st["completed"] == 100
    assert st["p50_s"] == pytest.approx(np.percentile(np.arange(1, 101), 50))
    assert st["p99_s"] == pytest.approx(np.percentile(np.arange(1, 101), 99))
    assert serve.latency_stats([]) == {"completed": 0}
