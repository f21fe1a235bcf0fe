"""Many filters in one batch (vsmc_cuda_cv_batch).

A filter's results must not depend on what else shares its launches: every
slot of a batch equals a single vsmc_cuda_cv_filter with the same
configuration bit for bit (histories, log-evidence), whether the batch runs
all series to the end at once or advances filters one observation at a time
in arbitrary groups, and the FP64 form of a slot matches the oracle's golden
run within the single filter's tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL_FP64 = 1e-9
KEYS = ("ess", "resampled", "logz_inc", "mean_x", "mean_y")

# (N, T, seed, stream_id): ragged sizes around the 2048-particle tile
SPECS = [(1000, 100, 101, 0), (2048, 12, 7, 1), (2049, 25, 8, 2), (5000, 40, 9, 3),
         (300, 7, 10, 4), (16387, 20, 11, 5), (65536, 9, 12, 6), (2, 5, 13, 7)]


@pytest.fixture(scope="module")
def capi():
    from vsmc_b200 import capi as C

    C.lib()
    return C


def series(capi, golden, k, T, sid):
    if k == 0:
        return golden["cv_obs_x"][:T].copy(), golden["cv_obs_y"][:T].copy()
    return capi.cv_simulate(T, obs_seed=100 + k, stream_id=sid)


def single(capi, N, T, scheme, form, seed, sid, ox, oy):
    with capi.CVFilter(N, T, scheme=scheme, form=form, seed=seed, stream_id=sid) as f:
        f.set_observations_host(ox, oy)
        f.initialize()
        if T > 1:
            f.iterate(T - 1)
        h = f.history()
        h["logz"] = f.log_evidence()
    return h


def assert_same(h, s, what):
    for k in KEYS:
        assert np.array_equal(h[k], s[k]), (what, k)


@pytest.mark.parametrize("tiling", [0, 4, 64])
@pytest.mark.parametrize("form", [0, 1])
@pytest.mark.parametrize("scheme", range(6))
def test_batch_run_equals_single(golden, capi, scheme, form, tiling):
    """Every slot equals the lone filter bit for bit whether it runs
    grid-per-filter (tiling 0), block-per-filter (tiling 64: all of SPECS)
    or either, by size (tiling 4: filters of at most 4 tiles block)."""
    obs = [series(capi, golden, k, T, sid) for k, (N, T, seed, sid) in enumerate(SPECS)]
    with capi.CVBatch(len(SPECS), scheme=scheme, form=form) as b:
        slots = [b.admit(N, T, seed, sid) for (N, T, seed, sid) in SPECS]
        b.set_observations(slots, obs)
        b.set_tiling(tiling)
        b.run(slots)
        last = b.read_last(slots)
        hist = [b.history(s) for s in slots]
    for k, (N, T, seed, sid) in enumerate(SPECS):
        s = single(capi, N, T, scheme, form, seed, sid, *obs[k])
        assert_same(hist[k], s, (scheme, form, N))
        assert last["log_evidence"][k] == s["logz"]
        assert last["ess"][k] == s["ess"][-1]
        assert last["resampled"][k] == s["resampled"][-1]
    if form == 0:
        h = hist[0]
        assert np.array_equal(h["resampled"], golden[f"cv_s{scheme}_resampled"])
        ref = golden[f"cv_s{scheme}_logz"]
        assert abs(last["log_evidence"][0] - ref) <= RTOL_FP64 * abs(ref)


@pytest.mark.parametrize("form", [0, 1])
def test_batch_streamed_equals_run(golden, capi, form):
    """Serving order: filters admitted at different times, one observation
    appended per step, ticks over random subsets; the results equal a run of
    the same filters in one batch."""
    scheme = 3
    obs = [series(capi, golden, k, T, sid) for k, (N, T, seed, sid) in enumerate(SPECS)]
    with capi.CVBatch(len(SPECS), scheme=scheme, form=form) as b:
        slots = [b.admit(N, T, seed, sid) for (N, T, seed, sid) in SPECS]
        b.set_observations(slots, obs)
        b.run(slots)
        ref = [b.history(s) for s in slots]
        ref_logz = b.read_last(slots)["log_evidence"]
    rng = np.random.default_rng(42)
    with capi.CVBatch(len(SPECS) + 2, scheme=scheme, form=form) as b:
        # two filler filters take the first slots, then leave
        fill = [b.admit(4096, 50, 1, 90), b.admit(3000, 50, 2, 91)]
        fobs = [capi.cv_simulate(50, obs_seed=7, stream_id=90 + i) for i in range(2)]
        b.set_observations(fill, fobs)
        b.step(fill)
        pos = {}
        slot_of = {}
        pending = list(range(len(SPECS)))
        rng.shuffle(pending)
        admitted = []
        released = False
        while pending or any(pos[k] < SPECS[k][1] for k in admitted):
            # admit up to two new filters per tick
            for _ in range(min(2, len(pending))):
                k = pending.pop()
                N, T, seed, sid = SPECS[k]
                slot_of[k] = b.admit(N, T, seed, sid)
                pos[k] = 0
                admitted.append(k)
            live = [k for k in admitted if pos[k] < SPECS[k][1]]
            tick = [k for k in live if rng.random() < 0.7] or live[:1]
            sl = [slot_of[k] for k in tick]
            b.append_observations(sl, [obs[k][0][pos[k]] for k in tick],
                                  [obs[k][1][pos[k]] for k in tick])
            b.step(sl + ([] if released else fill[:1]))
            for k in tick:
                pos[k] += 1
            if not released and len(admitted) >= 4:
                for f in fill:
                    b.release(f)
                released = True
        got = [b.history(slot_of[k]) for k in range(len(SPECS))]
        logz = b.read_last([slot_of[k] for k in range(len(SPECS))])["log_evidence"]
    for k in range(len(SPECS)):
        assert_same(got[k], ref[k], k)
        assert logz[k] == ref_logz[k]


def test_batch_admission_budget(capi):
    with capi.CVBatch(3) as b0:
        one = b0.slot_bytes(4096, 10)
    assert one > 4096 * 80
    with capi.CVBatch(3, hbm_budget=2 * one + one // 2) as b:
        s0 = b.admit(4096, 10)
        s1 = b.admit(4096, 10)
        assert b.bytes_in_use() == 2 * one
        with pytest.raises(capi.VsmcCudaError) as e:
            b.admit(4096, 10)
        assert e.value.status == capi.ENOMEM
        small = b.admit(1024, 10)  # fits in the remaining half
        with pytest.raises(capi.VsmcCudaError) as e:
            b.admit(2, 1)  # every slot in use
        assert e.value.status == capi.ENOMEM
        b.release(s1)
        s3 = b.admit(4096, 10)
        assert s3 == s1
        assert b.bytes_in_use() == 2 * one + b.slot_bytes(1024, 10)
        del s0, small


def test_batch_bad_calls(capi):
    with capi.CVBatch(4) as b:
        s = b.admit(1024, 3)
        with pytest.raises(capi.VsmcCudaError) as e:
            b.step([s])  # no observation yet
        assert e.value.status == capi.EINVAL
        b.set_observations([s], [capi.cv_simulate(3, obs_seed=1)])
        with pytest.raises(capi.VsmcCudaError):
            b.step([s, s])  # listed twice
        with pytest.raises(capi.VsmcCudaError):
            b.step([3])  # not admitted
        with pytest.raises(capi.VsmcCudaError):
            b.set_observations([s], [capi.cv_simulate(4, obs_seed=1)])  # > T_max
        b.run([s])
        assert b.iter_size(s) == 3
        with pytest.raises(capi.VsmcCudaError):
            b.step([s])  # observations used up
        with pytest.raises(capi.VsmcCudaError):
            b.append_observations([s], [0.0], [0.0])  # series full
        b.initialize([s])
        assert b.iter_size(s) == 0
        b.run([s])
        h = b.history(s)
        assert h["ess"].size == 3 and np.all(np.isfinite(h["ess"]))


def test_batch_nan_observation_is_degenerate(capi):
    with capi.CVBatch(2) as b:
        good, bad = b.admit(2048, 4, 1, 0), b.admit(2048, 4, 2, 1)
        ox, oy = capi.cv_simulate(4, obs_seed=3)
        bx = ox.copy()
        bx[2] = np.nan
        b.set_observations([good, bad], [(ox, oy), (bx, oy)])
        b.run([good, bad])
        r = b.read_last([good])
        assert np.isfinite(r["log_evidence"][0])
        with pytest.raises(capi.VsmcCudaError) as e:
            b.read_last([good, bad])
        assert e.value.status == capi.EDEGENERATE


def test_batch_graph_and_direct_runs_agree(golden, capi):
    """A run recorded as a CUDA graph (and relaunched) equals direct launches."""
    obs = [series(capi, golden, k, T, sid) for k, (N, T, seed, sid) in enumerate(SPECS)]
    out = []
    for graphs in (True, False):
        with capi.CVBatch(len(SPECS), scheme=1, form=1) as b:
            b.set_graphs(graphs)
            slots = [b.admit(N, T, seed, sid) for (N, T, seed, sid) in SPECS]
            b.set_observations(slots, obs)
            runs = []
            for _ in range(3):  # the second and third runs relaunch the graph
                b.initialize(slots)
                b.run(slots)
                runs.append([b.history(s) for s in slots])
            out.append(runs)
    for r in range(3):
        for k in range(len(SPECS)):
            assert_same(out[0][r][k], out[1][r][k], (r, k))


@pytest.mark.parametrize("form", [0, 1])
def test_batch_launch_shapes_agree(golden, capi, form):
    """Every launch shape (move CTAs per SM, finalize width) and the
    autotuner's choice give the same results bit for bit; the narrow
    finalize is skipped for a batch holding a filter of more than 256
    tiles."""
    specs = SPECS + [(1 << 20, 6, 14, 8)]
    for big in (False, True):
        sp = specs if big else SPECS
        obs = [series(capi, golden, k, T, sid) for k, (N, T, seed, sid) in enumerate(sp)]
        out = {}
        for shape in ((3, 1024), (2, 1024), (4, 256), (3, 256), "auto"):
            with capi.CVBatch(len(sp), scheme=5 if big else 3, form=form) as b:
                slots = [b.admit(N, T, seed, sid) for (N, T, seed, sid) in sp]
                b.set_observations(slots, obs)
                if shape == "auto":
                    mv, fin = b.autotune(slots)
                    assert mv in (2, 3, 4) and fin in (256, 1024)
                    if big:
                        assert fin == 1024
                else:
                    b.set_launch_shape(*shape)
                b.run(slots)
                out[shape] = [b.history(s) for s in slots]
                out[shape].append(b.read_last(slots)["log_evidence"])
        for shape, h in out.items():
            for k in range(len(sp)):
                assert_same(h[k], out[(3, 1024)][k], (big, shape, k))
            assert np.array_equal(h[-1], out[(3, 1024)][-1])


def test_batch_launch_shape_rejects(capi):
    with capi.CVBatch(2, scheme=0) as b:
        for shape in ((1, 1024), (5, 1024), (3, 512)):
            with pytest.raises(capi.VsmcCudaError):
                b.set_launch_shape(*shape)


def test_batch_read_steps(golden, capi):
    """Several observations appended per slot, one run through them all:
    read_steps gives each slot's last steps exactly as its history has them,
    and the running log-evidence is the sequential sum of the increments."""
    specs = SPECS[:5]
    obs = [series(capi, golden, k, T, sid) for k, (N, T, seed, sid) in enumerate(specs)]
    with capi.CVBatch(len(specs), scheme=0, form=0) as b:
        slots = [b.admit(N, T, seed, sid) for (N, T, seed, sid) in specs]
        pos = [0] * len(specs)
        rng = np.random.default_rng(5)
        while any(pos[k] < specs[k][1] for k in range(len(specs))):
            counts = [min(int(rng.integers(1, 5)), specs[k][1] - pos[k]) for k in range(len(specs))]
            live = [k for k in range(len(specs)) if counts[k] > 0]
            for j in range(max(counts)):
                rnd = [k for k in live if counts[k] > j]
                b.append_observations([slots[k] for k in rnd],
                                      [obs[k][0][pos[k] + j] for k in rnd],
                                      [obs[k][1][pos[k] + j] for k in rnd])
            b.run([slots[k] for k in live])
            got = b.read_steps([slots[k] for k in live], [counts[k] for k in live])
            off = 0
            for k in live:
                h = b.history(slots[k])
                sl = slice(pos[k], pos[k] + counts[k])
                g = slice(off, off + counts[k])
                assert np.array_equal(got["ess"][g], h["ess"][sl]), k
                assert np.array_equal(got["logz_inc"][g], h["logz_inc"][sl]), k
                assert np.array_equal(got["resampled"][g], h["resampled"][sl]), k
                off += counts[k]
                pos[k] += counts[k]
            assert np.all(got["status"] == 0)
        last = b.read_last(slots)
    for k, (N, T, seed, sid) in enumerate(specs):
        s = single(capi, N, T, 0, 0, seed, sid, *obs[k])
        assert last["log_evidence"][k] == np.cumsum(s["logz_inc"])[-1]
    with capi.CVBatch(1) as b:
        s0 = b.admit(1000, 4)
        with pytest.raises(capi.VsmcCudaError):
            b.read_steps([s0], [1])  # no step taken yet


@pytest.mark.parametrize("graphs", [True, False])
def test_block_tiling_graph_and_rerun(golden, capi, graphs):
    """Block-per-filter beside grid-per-filter in one run, recorded as a CUDA
    graph (or launched directly), run twice after a re-initialise (which
    keeps each resample engine's position, as Sampler::initialize does):
    each run equals the same run of the all-grid batch."""
    scheme = 0
    obs = [series(capi, golden, k, T, sid) for k, (N, T, seed, sid) in enumerate(SPECS)]
    res = {}
    for tiling in (0, 2):
        with capi.CVBatch(len(SPECS), scheme=scheme) as b:
            b.set_graphs(graphs)
            slots = [b.admit(N, T, seed, sid) for (N, T, seed, sid) in SPECS]
            b.set_observations(slots, obs)
            b.set_tiling(tiling)
            assert b.tiling() == tiling
            runs = []
            for _ in range(2):
                b.initialize(slots)
                b.run(slots)
                runs.append(([b.history(s) for s in slots],
                             b.read_last(slots)["log_evidence"]))
            res[tiling] = runs
    for run in range(2):
        for k in range(len(SPECS)):
            assert_same(res[2][run][0][k], res[0][run][0][k], (run, k))
        assert np.array_equal(res[2][run][1], res[0][run][1])


def test_autotune_picks_a_tiling(golden, capi):
    obs = [series(capi, golden, k, T, sid) for k, (N, T, seed, sid) in enumerate(SPECS)]
    with capi.CVBatch(len(SPECS), scheme=3) as b:
        slots = [b.admit(N, T, seed, sid) for (N, T, seed, sid) in SPECS]
        b.set_observations(slots, obs)
        b.autotune(slots)
        assert b.tiling() in (0, 1, 2, 4, 8, 16, 32, 64)
        b.run(slots)
        hist = [b.history(s) for s in slots]
    for k, (N, T, seed, sid) in enumerate(SPECS):
        s = single(capi, N, T, 3, 0, seed, sid, *obs[k])
        assert_same(hist[k], s, N)
