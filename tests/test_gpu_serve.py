"""The serving loop (vsmc_cuda_cv_server): requests of different sizes,
admitted by device memory, observations streamed one at a time from a
client thread in random interleaving.  Each request's per-observation
results must equal the same filter run alone (vsmc_cuda_cv_filter), bit for
bit, whatever it shared its ticks with."""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SPECS = [(1000, 30, 101, 0), (2048, 12, 7, 1), (2049, 25, 8, 2), (5000, 40, 9, 3),
         (300, 7, 10, 4), (16387, 20, 11, 5), (65536, 9, 12, 6), (4096, 15, 13, 7)]


@pytest.fixture(scope="module")
def capi():
    from vsmc_b200 import capi as C

    C.lib()
    return C


def alone(capi, N, T, seed, sid, ox, oy, scheme, form):
    with capi.CVFilter(N, T, scheme=scheme, form=form, seed=seed, stream_id=sid) as f:
        f.set_observations_host(ox, oy)
        f.initialize()
        if T > 1:
            f.iterate(T - 1)
        return f.history()


def stream_requests(capi, srv, specs, obs, rng, delay=True):
    """Client thread: open requests in random order over time and feed each
    its observations one at a time; returns request ids in spec order."""
    ids = [None] * len(specs)
    order = list(range(len(specs)))
    rng.shuffle(order)
    err = []

    def client():
        try:
            pos = {}
            opened = []
            while order or any(pos[k] < specs[k][1] for k in opened):
                if order and (not opened or rng.random() < 0.3):
                    k = order.pop()
                    N, T, seed, sid = specs[k]
                    ids[k] = srv.open(N, T, seed, sid)
                    pos[k] = 0
                    opened.append(k)
                live = [k for k in opened if pos[k] < specs[k][1]]
                pick = [k for k in live if rng.random() < 0.5] or live[:1]
                srv.observe([ids[k] for k in pick], [obs[k][0][pos[k]] for k in pick],
                            [obs[k][1][pos[k]] for k in pick])
                for k in pick:
                    pos[k] += 1
                    if pos[k] == specs[k][1]:
                        srv.close(ids[k])
                if delay and rng.random() < 0.2:
                    time.sleep(0.0005)
        except Exception as e:  # reported by the caller
            err.append(e)

    th = threading.Thread(target=client)
    th.start()
    th.join(120)
    assert not th.is_alive()
    assert not err, err
    return ids


def collect(srv, n_expected):
    got = []
    total = 0
    deadline = time.time() + 120
    while total < n_expected and time.time() < deadline:
        r = srv.poll(wait_ms=100)
        got.append(r)
        total += r.size
    assert total == n_expected
    return np.concatenate(got)


@pytest.mark.parametrize("form", [0, 1])
def test_server_results_equal_alone(capi, form):
    scheme = 0
    obs = [capi.cv_simulate(T, obs_seed=200 + k, stream_id=sid)
           for k, (N, T, seed, sid) in enumerate(SPECS)]
    rng = np.random.default_rng(7 + form)
    with capi.CVServer(16, scheme=scheme, form=form) as srv:
        ids = stream_requests(capi, srv, SPECS, obs, rng)
        res = collect(srv, sum(T for _, T, _, _ in SPECS))
        srv.drain(10000)
        st = srv.stats()
    assert st["opened"] == len(SPECS) and st["admitted"] == len(SPECS)
    assert st["steps"] == res.size
    assert np.all(res["status"] == 0)
    assert np.all(res["done_ns"] >= res["submit_ns"])
    for k, (N, T, seed, sid) in enumerate(SPECS):
        r = np.sort(res[res["request"] == ids[k]], order="t")
        assert np.array_equal(r["t"], np.arange(T))
        h = alone(capi, N, T, seed, sid, *obs[k], scheme, form)
        assert np.array_equal(r["ess"], h["ess"]), k
        assert np.array_equal(r["logz_inc"], h["logz_inc"]), k
        assert np.array_equal(r["resampled"], h["resampled"]), k
        assert np.array_equal(r["log_evidence"], np.cumsum(h["logz_inc"])), k


def test_server_admission_by_budget(capi):
    """A budget for about two filters: requests wait for memory, all finish,
    at most two are on the device at once, results unchanged."""
    specs = [(8192, 10, 30 + k, k) for k in range(6)]
    obs = [capi.cv_simulate(T, obs_seed=300 + k, stream_id=sid)
           for k, (N, T, seed, sid) in enumerate(specs)]
    with capi.CVBatch(1) as b:
        one = b.slot_bytes(8192, 10)
    with capi.CVServer(8, scheme=3, hbm_budget=2 * one + one // 3) as srv:
        ids = stream_requests(capi, srv, specs, obs, np.random.default_rng(3), delay=False)
        res = collect(srv, sum(T for _, T, _, _ in specs))
        st = srv.stats()
    assert st["max_active"] <= 2
    assert st["admitted"] == len(specs) and st["completed"] >= len(specs) - 2
    for k, (N, T, seed, sid) in enumerate(specs):
        r = np.sort(res[res["request"] == ids[k]], order="t")
        h = alone(capi, N, T, seed, sid, *obs[k], 3, 0)
        assert np.array_equal(r["logz_inc"], h["logz_inc"]), k


def test_server_bad_calls(capi):
    with capi.CVBatch(1) as b:
        one = b.slot_bytes(4096, 5)
    with capi.CVServer(2, hbm_budget=one) as srv:
        with pytest.raises(capi.VsmcCudaError) as e:
            srv.open(8192, 5)  # alone exceeds the budget
        assert e.value.status == capi.ENOMEM
        r = srv.open(4096, 2)
        with pytest.raises(capi.VsmcCudaError):
            srv.observe([r + 100], [0.0], [0.0])  # unknown request
        srv.observe([r, r], [0.1, 0.2], [0.0, 0.1])
        with pytest.raises(capi.VsmcCudaError):
            srv.observe([r], [0.3], [0.0])  # beyond T_max
        srv.close(r)
        with pytest.raises(capi.VsmcCudaError):
            srv.close(r)  # closed twice
        srv.drain(10000)
        res = srv.poll()
        assert res.size == 2 and np.all(res["status"] == 0)


@pytest.mark.parametrize("form", [0, 1])
def test_server_catch_up(capi, form):
    """Every observation of every request is submitted at once: the loop
    catches up several steps per request per tick (fewer ticks than steps),
    and every per-observation result still equals the filter run alone."""
    specs = SPECS[:6]
    obs = [capi.cv_simulate(T, obs_seed=400 + k, stream_id=sid)
           for k, (N, T, seed, sid) in enumerate(specs)]
    with capi.CVServer(16, scheme=3, form=form) as srv:
        ids = [srv.open(N, T, seed, sid) for (N, T, seed, sid) in specs]
        Tmax = max(T for _, T, _, _ in specs)
        for t in range(Tmax):
            live = [k for k in range(len(specs)) if t < specs[k][1]]
            srv.observe([ids[k] for k in live], [obs[k][0][t] for k in live],
                        [obs[k][1][t] for k in live])
        for k in range(len(specs)):
            srv.close(ids[k])
        res = collect(srv, sum(T for _, T, _, _ in specs))
        srv.drain(10000)
        st = srv.stats()
    assert st["steps"] == res.size
    assert st["ticks"] < res.size
    assert np.all(res["status"] == 0)
    for k, (N, T, seed, sid) in enumerate(specs):
        r = np.sort(res[res["request"] == ids[k]], order="t")
        assert np.array_equal(r["t"], np.arange(T))
        h = alone(capi, N, T, seed, sid, *obs[k], 3, form)
        assert np.array_equal(r["ess"], h["ess"]), k
        assert np.array_equal(r["logz_inc"], h["logz_inc"]), k
        assert np.array_equal(r["resampled"], h["resampled"]), k
        assert np.array_equal(r["log_evidence"], np.cumsum(h["logz_inc"])), k


def test_server_degenerate_request_in_a_burst(capi):
    """A NaN observation in the middle of a burst: that request's steps
    before it succeed, it and every later step report EDEGENERATE, and the
    request sharing its ticks is unaffected (equal to its filter alone)."""
    T = 10
    ox, oy = capi.cv_simulate(T, obs_seed=500, stream_id=0)
    bx, by = capi.cv_simulate(T, obs_seed=501, stream_id=1)
    bad_x = ox.copy()
    bad_x[3] = np.nan
    with capi.CVServer(4, scheme=0) as srv:
        a = srv.open(4096, T, 21, 0)
        b = srv.open(3000, T, 22, 1)
        for t in range(T):
            srv.observe([a, b], [bad_x[t], bx[t]], [oy[t], by[t]])
        srv.close(a)
        srv.close(b)
        res = collect(srv, 2 * T)
    ra = np.sort(res[res["request"] == a], order="t")
    rb = np.sort(res[res["request"] == b], order="t")
    assert np.all(ra["status"][:3] == 0)
    assert np.all(ra["status"][3:] == capi.EDEGENERATE)
    assert np.all(np.isnan(ra["ess"][3:]))
    assert np.all(rb["status"] == 0)
    h = alone(capi, 3000, T, 22, 1, bx, by, 0, 0)
    assert np.array_equal(rb["ess"], h["ess"])
    assert np.array_equal(rb["logz_inc"], h["logz_inc"])
