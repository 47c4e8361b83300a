"""Continuous-batching reconstruction server.

CPU tests drive the admission logic in dry-run mode (workers hold each request
for a fixed time without touching a GPU); GPU tests check that a request's
result does not depend on what runs beside it, and that graph-captured solver
iterations give the eager result."""
import time

import numpy as np
import pytest

from conftest import rel


@pytest.fixture(scope="module")
def LB():
    import lamino_b200
    lamino_b200.lib()
    return lamino_b200


def _req(nproj=4, det=(8, 8), ngam=1, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(ngam):
        th = rng.uniform(0, np.pi, nproj).astype(np.float32)
        out.append((rng.random((nproj,) + det, dtype=np.float32), th, np.float32(0.3 * i)))
    return out


def test_footprint_grows_with_size(LB):
    p = LB.ReconParams()
    small = LB.mbir_footprint(2, [(16, 32, 32)], (32, 8, 32), p)
    big = LB.mbir_footprint(2, [(16, 64, 64)], (64, 16, 64), p)
    two = LB.mbir_footprint(3, [(16, 64, 64)] * 2, (64, 16, 64), p)
    one = LB.mbir_footprint(3, [(16, 64, 64)], (64, 16, 64), p)
    assert 0 < small < big
    assert two > one
    fp16 = LB.mbir_footprint(2, [(16, 64, 64)], (64, 16, 64), LB.ReconParams(op_kind="toeplitz_fp16"))
    assert fp16 < big


def test_dry_run_budget_and_slots(LB):
    """Never more bytes in use than the budget, never more requests than slots."""
    p = LB.ReconParams()
    recon = (8, 8, 8)
    fp = LB.mbir_footprint(2, [(4, 8, 8)], recon, p)
    with LB.ReconServer(budget_bytes=int(2.5 * fp), slots=4, dry_run_ms=40) as srv:
        ids = [srv.submit(2, _req(seed=i), recon, p) for i in range(8)]
        for i in ids:
            vol, t = srv.wait(i)
            assert vol.shape == (3,) + recon
            assert t["latency_s"] >= t["run_s"] >= 0.035
        st = srv.stats()
    assert st["submitted"] == 8 and st["completed"] == 8 and st["failed"] == 0
    assert st["peak_in_use"] <= st["budget"]
    assert st["peak_active"] == 2  # 2 fit in 2.5 footprints; 4 slots do not matter
    assert st["in_use"] == 0 and st["active"] == 0 and st["queued"] == 0


def test_dry_run_slot_limit(LB):
    p = LB.ReconParams()
    recon = (8, 8, 8)
    with LB.ReconServer(budget_bytes=1 << 40, slots=3, dry_run_ms=30) as srv:
        ids = [srv.submit(1, _req(seed=i), recon, p) for i in range(7)]
        for i in ids:
            srv.wait(i)
        st = srv.stats()
    assert st["peak_active"] == 3 and st["completed"] == 7


def test_dry_run_fifo_admission(LB):
    """A large request at the head of the queue blocks later small ones even when
    those would fit (no overtaking), so a large request cannot starve."""
    p = LB.ReconParams()
    small_recon, big_recon = (8, 8, 8), (48, 16, 48)
    fs = LB.mbir_footprint(2, [(4, 8, 8)], small_recon, p)
    fb = LB.mbir_footprint(2, [(4, 48, 48)], big_recon, p)
    budget = fb + fs // 2  # the big one runs alone
    assert fs + fb > budget and 2 * fs <= budget
    with LB.ReconServer(budget_bytes=budget, slots=4, dry_run_ms=60) as srv:
        t0 = time.perf_counter()
        a = srv.submit(2, _req(seed=1), small_recon, p)
        b = srv.submit(2, _req(det=(48, 48), seed=2), big_recon, p)
        c = srv.submit(2, _req(seed=3), small_recon, p)
        subs = {a: t0, b: time.perf_counter(), c: time.perf_counter()}
        res = {i: srv.wait(i)[1] for i in (a, b, c)}
    start = {i: subs[i] + res[i]["queue_s"] for i in res}
    done = {i: subs[i] + res[i]["latency_s"] for i in res}
    slack = 5e-3
    assert start[b] >= done[a] - slack  # b waited for a's memory
    assert start[c] >= start[b] - slack  # c did not overtake b
    assert start[c] >= done[b] - slack  # and c did not fit beside b


def test_dry_run_rejects_oversize_and_times_out(LB):
    p = LB.ReconParams()
    recon = (8, 8, 8)
    fp = LB.mbir_footprint(1, [(4, 8, 8)], recon, p)
    with LB.ReconServer(budget_bytes=fp - 1, slots=1, dry_run_ms=10) as srv:
        with pytest.raises(LB.LaminoError) as e:
            srv.submit(1, _req(), recon, p)
        assert e.value.code == 2
    with LB.ReconServer(budget_bytes=fp, slots=1, dry_run_ms=300) as srv:
        rid = srv.submit(1, _req(), recon, p)
        with pytest.raises(LB.LaminoError) as e:
            srv.wait(rid, timeout=0.01)
        assert e.value.code == 5
        vol, t = srv.wait(rid)  # still there after the timeout
        assert t["run_s"] >= 0.25
        with pytest.raises(LB.LaminoError):
            srv.wait(rid)  # forgotten once collected


def test_dry_run_shutdown_fails_queued_requests(LB):
    """Closing the server while a request is queued and another thread waits for it:
    the waiter gets LAMINO_ERR_STATE, the running request completes, close returns."""
    import threading
    p = LB.ReconParams()
    recon = (8, 8, 8)
    srv = LB.ReconServer(budget_bytes=1 << 40, slots=1, dry_run_ms=300)
    a = srv.submit(1, _req(seed=1), recon, p)
    b = srv.submit(1, _req(seed=2), recon, p)
    got = {}

    def waiter(rid, key):
        try:
            got[key] = srv.wait(rid)[1]["run_s"]
        except LB.LaminoError as e:
            got[key] = e.code

    ts = [threading.Thread(target=waiter, args=(a, "a")), threading.Thread(target=waiter, args=(b, "b"))]
    for t in ts:
        t.start()
    time.sleep(0.05)
    srv.close()
    for t in ts:
        t.join(10)
    assert got["b"] == 7 and got["a"] >= 0.25


def test_server_bad_arguments(LB):
    with pytest.raises(LB.LaminoError):
        LB.ReconServer(budget_bytes=0, slots=1, dry_run_ms=1)
    with pytest.raises(LB.LaminoError):
        LB.ReconServer(budget_bytes=1 << 30, slots=0, dry_run_ms=1)
    with LB.ReconServer(budget_bytes=1 << 30, slots=1, dry_run_ms=1) as srv:
        with pytest.raises(LB.LaminoError):
            srv.submit(4, _req(), (8, 8, 8))
        with pytest.raises(ValueError):
            srv.submit(1, [(np.zeros((4, 8, 8), np.float32), np.zeros(3, np.float32), 0.0)], (8, 8, 8))


def test_batch_checks_before_device_work(LB):
    """lamino_mbir3_batch validates every request (and its footprint against the
    budget) before it touches a device, so these run without a GPU."""
    out, info = LB.mbir3_batch([])
    assert out == [] and info["steps"] == 0
    req = (_req(nproj=4, det=(16, 16)), (16, 8, 16), LB.ReconParams())
    fp = LB.mbir_footprint(3, [(4, 16, 16)], (16, 8, 16), LB.ReconParams())
    with pytest.raises(LB.LaminoError) as e:  # larger than the budget
        LB.mbir3_batch([req, req], budget_bytes=fp - 1)
    assert e.value.args[0].startswith("lamino error 2")
    with pytest.raises(LB.LaminoError):
        LB.mbir3_batch([req], budget_bytes=0)
    with pytest.raises(LB.LaminoError):
        LB.mbir3_batch([req], threads=0)
    with pytest.raises(ValueError):
        LB.mbir3_batch([([], (16, 8, 16), None)])


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------

def _problem(O, recon, nproj, det, gammas, seed):
    rng = np.random.default_rng(seed)
    m = O.synthetic_magnetization(recon, seed=seed, sigma=1.0).astype(np.float64)
    plan = O.NufftPlan(recon, exact=True)
    data = []
    for n, g in zip(nproj, gammas):
        th = rng.uniform(0, 2 * np.pi, n).astype(np.float32)
        pg = O.PolarGrid(th, det[0], det[1], np.float32(g))
        proj = O.forward(m, pg, pg.gamma, plan) + 0.05
        data.append((proj.astype(np.float32), th, np.float32(g)))
    return data


@pytest.mark.gpu
def test_graphs_match_eager(L, O):
    """Graph-replayed solver iterations give the eager result (host inputs run on a
    private stream, so the graphs are in use)."""
    recon = (10, 6, 12)
    data = _problem(O, recon, (7, 6), (11, 13), (0.0, 0.6), seed=5)
    for method in (1, 2, 3):
        fn = {1: L.MBIR1, 2: L.MBIR2, 3: L.MBIR3}[method]
        for kind in ("toeplitz", "mixed") if method != 3 else ("toeplitz",):
            a = fn(data, recon, L.ReconParams(maxIters=5, innerIters=2, op_kind=kind, use_graphs=False))
            b = fn(data, recon, L.ReconParams(maxIters=5, innerIters=2, op_kind=kind, use_graphs=True))
            assert rel(b, a) < 1e-5, (method, kind)


@pytest.mark.gpu
def test_graphs_on_torch_stream(L, O):
    """Device inputs on a non-default torch stream: the graphs are captured on the
    caller's stream; the result matches the host-input call."""
    import torch
    recon = (8, 5, 9)
    data = _problem(O, recon, (6, 5), (9, 11), (0.0, 0.8), seed=3)
    want = L.MBIR2(data, recon, L.ReconParams(maxIters=4, innerIters=2, use_graphs=False))
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        dd = [(torch.from_numpy(p).cuda(), th, g) for p, th, g in data]
        got = L.MBIR2(dd, recon, L.ReconParams(maxIters=4, innerIters=2))
    s.synchronize()
    assert rel(got.cpu().numpy(), want) < 1e-5


@pytest.mark.gpu
def test_server_results_independent_of_batch(L, O):
    """Each of several mixed requests (different sizes, methods, operator forms)
    served concurrently gives what the direct call gives alone."""
    reqs = [
        (1, _problem(O, (8, 5, 9), (6, 5), (9, 11), (0.0, 0.8), 3), (8, 5, 9),
         L.ReconParams(maxIters=4, innerIters=2)),
        (2, _problem(O, (12, 6, 10), (9,), (13, 11), (0.4,), 4), (12, 6, 10),
         L.ReconParams(maxIters=4, innerIters=2, op_kind="mixed")),
        (3, _problem(O, (10, 4, 10), (5, 6), (9, 13), (0.0, 0.5), 6), (10, 4, 10),
         L.ReconParams(maxIters=5, innerIters=3)),
        (2, _problem(O, (6, 6, 6), (4,), (7, 7), (0.2,), 7), (6, 6, 6),
         L.ReconParams(maxIters=3, innerIters=2, op_kind="toeplitz_fp16")),
        (1, _problem(O, (9, 5, 8), (6,), (9, 9), (0.3,), 8), (9, 5, 8),
         L.ReconParams(maxIters=3, op_kind="nufft")),
    ]
    direct = [{1: L.MBIR1, 2: L.MBIR2, 3: L.MBIR3}[m](d, r, p) for m, d, r, p in reqs]
    with L.ReconServer(budget_bytes=4 << 30, slots=3) as srv:
        ids = [srv.submit(m, d, r, p) for m, d, r, p in reqs]
        got = [srv.wait(i, timeout=120)[0] for i in ids]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0 and st["peak_active"] >= 2
    for k, (g, w) in enumerate(zip(got, direct)):
        assert rel(g, w) < 1e-5, k


@pytest.mark.gpu
def test_server_reports_failed_requests(L, O):
    """A request that fails inside its worker (an invalid NUFFT tolerance) comes
    back as an error from wait(), is counted as failed, and does not disturb the
    requests around it."""
    good = _problem(O, (8, 5, 9), (6,), (9, 11), (0.0,), 3)
    with L.ReconServer(budget_bytes=4 << 30, slots=2) as srv:
        a = srv.submit(1, good, (8, 5, 9), L.ReconParams(maxIters=3))
        b = srv.submit(1, good, (8, 5, 9), L.ReconParams(maxIters=3, op_kind="nufft", eps=1e-12))
        c = srv.submit(1, good, (8, 5, 9), L.ReconParams(maxIters=3))
        va, _ = srv.wait(a, timeout=120)
        with pytest.raises(L.LaminoError) as e:
            srv.wait(b, timeout=120)
        assert e.value.code == 1 and "tolerance" in str(e.value)
        vc, _ = srv.wait(c, timeout=120)
        st = srv.stats()
    assert st["failed"] == 1 and st["completed"] == 2 and st["in_use"] == 0
    assert rel(vc, va) < 1e-6
