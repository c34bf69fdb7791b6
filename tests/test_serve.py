"""The tracking-job server: admission against the HBM budget, FIFO order,
errors through the futures (CPU, with a fake context), and -- on the GPU --
identical results for jobs run alone and in a concurrent mix."""
import threading
import time

import numpy as np
import pytest

from specklesource_b200 import abi, serve


class FakeContext:
    """Stands in for runtime.Context: records concurrency, sleeps a little."""
    lock = threading.Lock()
    running = 0
    max_running = 0
    batch_calls = []

    def __init__(self, device):
        self.closed = False

    def _run(self, p):
        with FakeContext.lock:
            FakeContext.running += 1
            FakeContext.max_running = max(FakeContext.max_running, FakeContext.running)
        time.sleep(0.02)
        with FakeContext.lock:
            FakeContext.running -= 1
        if p.nR == 13:
            raise RuntimeError("planted failure")
        g = np.full((p.nA, p.nR), float(p.nR), np.float32)
        return {"offR": g, "offA": g.copy(), "corr": g.copy(), "type": np.ones((p.nA, p.nR), np.uint8)}

    def strack(self, p, a, b):
        return self._run(p)

    def strackw(self, p, a, b):
        return self._run(p)

    def strack_batch(self, ps, a, b):
        FakeContext.batch_calls.append(len(ps))
        return [self._run(p) for p in ps]

    def cull(self, cp, offR, offA, corr, mt):
        return {"offRS": offR + 1}

    def close(self):
        self.closed = True


def _job(nR, nA=4, kind="strack", cull=False):
    img = np.zeros((8, 8), np.complex64)
    return serve.Job(kind=kind, params=abi.TrackParams(nR=nR, nA=nA), img1=img, img2=img,
                     cull=abi.CullParams(nR=nR, nA=nA) if cull else None, tag=nR)


def test_budget_limits_concurrency_and_order():
    FakeContext.running = FakeContext.max_running = 0
    one = serve.job_device_bytes(_job(10))
    # room for two jobs at a time although four slots are free
    with serve.JobServer(slots=4, hbm_budget=2.5 * one, context_factory=FakeContext) as srv:
        futs = [srv.submit(_job(10 + (k % 2) * 0)) for k in range(8)]
        res = [f.result(timeout=10) for f in futs]
        assert srv.peak_bytes <= 2.5 * one
    assert FakeContext.max_running == 2
    assert all(r["track"]["offR"][0, 0] == 10 for r in res)
    assert all(r["end"] >= r["start"] >= r["arrival"] for r in res)


def test_fifo_admission_and_cull_and_errors():
    FakeContext.running = FakeContext.max_running = 0
    with serve.JobServer(slots=1, hbm_budget=1e12, context_factory=FakeContext) as srv:
        jobs = [_job(nR, cull=True) for nR in (5, 6, 13, 7)]
        futs = [srv.submit(j) for j in jobs]
        assert futs[0].result(timeout=10)["cull"]["offRS"][0, 0] == 6
        with pytest.raises(RuntimeError, match="planted"):
            futs[2].result(timeout=10)
        assert futs[3].result(timeout=10)["track"]["offR"][0, 0] == 7
        assert [t for t, _ in srv.started] == [5, 6, 13, 7]


def test_job_above_budget_is_refused():
    with serve.JobServer(slots=1, hbm_budget=1000, context_factory=FakeContext) as srv:
        f = srv.submit(_job(100, 100))
        with pytest.raises(ValueError, match="HBM budget"):
            f.result(timeout=5)


class HoldingContext(FakeContext):
    """A fake context that keeps device buffers after a job, like the
    library's contexts: it holds `need` bytes once it has run a job, until
    release() is called."""
    log = []

    def __init__(self, device):
        super().__init__(device)
        self.held = 0

    def _run(self, p):
        r = super()._run(p)
        self.held = serve.job_device_bytes(_job(p.nR, p.nA))
        HoldingContext.log.append(self.held)
        return r

    def device_bytes(self):
        return self.held

    def release(self):
        self.held = 0


def test_budget_counts_buffers_held_by_idle_slots():
    """Idle slots still hold their last job's buffers and the budget counts
    them: a job that fits only once they are freed makes the idle slots
    release their buffers first."""
    FakeContext.running = FakeContext.max_running = 0
    one = serve.job_device_bytes(_job(10))
    big = _job(200, 400)  # 80,000 points: about twice a small job's buffers
    need_big = serve.job_device_bytes(big)
    budget = 2.2 * one
    assert 2 * one <= budget < one + need_big and need_big <= budget
    with serve.JobServer(slots=2, hbm_budget=budget, context_factory=HoldingContext) as srv:
        first = [f.result(timeout=10) for f in [srv.submit(_job(10)) for _ in range(2)]]
        assert {r["slot"] for r in first} == {0, 1}  # both ran at once; both slots now hold buffers
        assert srv.reserved_bytes() == 2 * one
        r = srv.submit(big).result(timeout=10)
        assert srv.releases >= 1  # an idle slot gave its buffers back before the big job started
        assert srv.peak_bytes <= budget
        assert srv.reserved_bytes() <= budget
    assert r["track"]["offR"][0, 0] == 200


def test_queued_strack_jobs_share_a_batched_call():
    """Continuous batching: jobs that queue while a slot is busy and can share
    flags go into one strack_batch call; each future gets its own result, in
    submission order; a job with other flags starts a new batch."""
    FakeContext.running = FakeContext.max_running = 0
    FakeContext.batch_calls = []
    with serve.JobServer(slots=1, hbm_budget=1e12, context_factory=FakeContext, max_batch=4) as srv:
        jobs = [_job(nR) for nR in (5, 6, 7, 8, 9, 10)]
        jobs[4].params.hanningFlag = 0  # cannot join the others' batch
        futs = [srv.submit(j) for j in jobs]
        res = [f.result(timeout=10) for f in futs]
    assert [r["track"]["offR"][0, 0] for r in res] == [5, 6, 7, 8, 9, 10]
    assert max(srv.batches) > 1 and sum(srv.batches) == 6
    assert FakeContext.batch_calls  # the batched entry point was used
    assert [t for t, _ in srv.started] == [5, 6, 7, 8, 9, 10]


def test_latency_stats():
    rs = [{"arrival": 0.0, "start": 0.0005 * k, "end": 0.001 * k} for k in range(1, 101)]
    st = serve.latency_stats(rs)
    assert abs(st["p50"] - 50.5) < 1e-6 and st["max"] == 100.0
    assert abs(st["wait_p50"] - 25.25) < 1e-6 and abs(st["service_p50"] - 25.25) < 1e-6


@pytest.mark.gpu
def test_same_result_alone_and_in_the_mix():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from specklesource_b200 import build, runtime, synth
    build.build()
    jobs = []
    for k, (na, nr) in enumerate([(512, 768), (640, 1024), (512, 512), (768, 768), (600, 900), (512, 1024)]):
        s1, s2 = synth.small_pair(device="cuda", na=na, nr=nr, seed=20 + k)
        W = (32, 48, 64)[k % 3]
        nRg, nAg = (nr - 2 * W) // (W // 2), (na - 2 * W) // (W // 2)
        if k % 2 == 0:
            p = abi.TrackParams(rStart=W, aStart=W, deltaR=W // 2, deltaA=W // 2, nR=nRg, nA=nAg, wR=W, wA=W,
                                wRa=W, wAa=W, noComplex=k % 4 == 2)
            kind = "strack"
        else:
            p = abi.TrackParams(rStart=2 * W, aStart=2 * W, deltaR=W // 2, deltaA=W // 2, nR=nRg - 4,
                                nA=nAg - 4, wR=W, wA=W, wRa=2 * W, wAa=2 * W, edgePadR=8, edgePadA=8,
                                navgR=2, navgA=2)
            kind = "strackw"
        jobs.append(serve.Job(kind=kind, params=p, img1=s1, img2=s2,
                              cull=abi.CullParams(nR=p.nR, nA=p.nA, islandThresh=4), tag=k))
    with runtime.Context(0) as ctx:
        alone = [serve.run_job(ctx, j) for j in jobs]
    with serve.JobServer(slots=3, hbm_budget=60e9) as srv:
        mixed = [f.result(timeout=600) for f in [srv.submit(j) for j in jobs]]
    assert len({r["slot"] for r in mixed}) > 1
    for a, m in zip(alone, mixed):
        for k in ("offR", "offA", "corr", "type"):
            assert np.array_equal(a["track"][k], m["track"][k], equal_nan=True), k
        for k in ("offRS", "offAS", "type"):
            assert np.array_equal(a["cull"][k], m["cull"][k], equal_nan=True), k


@pytest.mark.gpu
def test_queued_strack_jobs_share_batched_calls():
    """Continuous batching: strack jobs of one window queued behind a busy
    slot run together in one sb_strack_batch call, each with the result it
    has alone (tracking and culling)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from specklesource_b200 import build, runtime, synth
    build.build()
    jobs = []
    for k, (na, nr) in enumerate([(512, 768), (640, 1024), (512, 512), (768, 768), (600, 900), (512, 1024)]):
        s1, s2 = synth.small_pair(device="cuda", na=na, nr=nr, seed=60 + k)
        W = 32
        p = abi.TrackParams(rStart=W, aStart=W, deltaR=W // 2, deltaA=W // 2, nR=(nr - 2 * W) // (W // 2),
                            nA=(na - 2 * W) // (W // 2), wR=W, wA=W, wRa=W, wAa=W)
        jobs.append(serve.Job(kind="strack", params=p, img1=s1, img2=s2,
                              cull=abi.CullParams(nR=p.nR, nA=p.nA, islandThresh=4), tag=k))
    with runtime.Context(0) as ctx:
        alone = [serve.run_job(ctx, j) for j in jobs]
    with serve.JobServer(slots=1, hbm_budget=60e9, max_batch=4) as srv:
        batched = [f.result(timeout=600) for f in [srv.submit(j) for j in jobs]]
        sizes = list(srv.batches)
    assert max(sizes) > 1 and sum(sizes) == len(jobs), sizes
    for a, m in zip(alone, batched):
        for k in ("offR", "offA", "corr", "type"):
            assert np.array_equal(a["track"][k], m["track"][k], equal_nan=True), k
        for k in ("offRS", "offAS", "type"):
            assert np.array_equal(a["cull"][k], m["cull"][k], equal_nan=True), k


@pytest.mark.gpu
def test_device_memory_stays_within_the_budget():
    """Mixed jobs under a budget that fits about one job at a time: after
    every job the device memory all slots' contexts hold (sb_context_device_bytes)
    is within the budget, and the results are those of the jobs run alone."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from specklesource_b200 import build, runtime, synth
    build.build()
    jobs = []
    for k, (na, nr, W) in enumerate([(768, 1024, 64), (512, 768, 32), (1024, 1024, 48), (640, 896, 64),
                                      (512, 512, 32), (896, 768, 48)]):
        s1, s2 = synth.small_pair(device="cpu", na=na, nr=nr, seed=40 + k)
        a, b = synth.to_numpy(s1), synth.to_numpy(s2)  # host images: their device copies count
        p = abi.TrackParams(rStart=W, aStart=W, deltaR=W // 2, deltaA=W // 2, nR=(nr - 2 * W) // (W // 2),
                            nA=(na - 2 * W) // (W // 2), wR=W, wA=W, wRa=W, wAa=W)
        jobs.append(serve.Job(kind="strack", params=p, img1=a, img2=b,
                              cull=abi.CullParams(nR=p.nR, nA=p.nA), tag=k))
    with runtime.Context(0) as ctx:
        alone = [serve.run_job(ctx, j) for j in jobs]
    budget = 1.3 * max(serve.job_device_bytes(j) for j in jobs)
    with serve.JobServer(slots=3, hbm_budget=budget) as srv:
        futs = [srv.submit(j) for j in jobs]
        mixed = [f.result(timeout=600) for f in futs]
        held = [c.device_bytes() for c in srv._ctx]
        assert sum(held) <= budget, (held, budget)
        assert srv.peak_bytes <= budget
        for r in mixed:  # what the job's own context held when it finished
            assert r["held_bytes"] <= budget
    for a, m in zip(alone, mixed):
        for k in ("offR", "offA", "corr", "type"):
            assert np.array_equal(a["track"][k], m["track"][k], equal_nan=True), k


def test_estimate_counts_the_peak_hand_off_once_per_chunk():
    """The complex stage's 960-byte peak hand-off is held for at most one list
    chunk (524,288 points); -gauss keeps the fit in the complex kernel."""
    small = serve.job_device_bytes(_job(100, 100))
    big = serve.job_device_bytes(_job(2000, 1000))
    gauss = _job(2000, 1000)
    gauss.params.gaussFlag = 1
    per_point = serve._STRACK_POINT_BYTES
    assert small - 100 * 100 * per_point >= 100 * 100 * 960
    assert big - serve.job_device_bytes(gauss) == (1 << 19) * 960
