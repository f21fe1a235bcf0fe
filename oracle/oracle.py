"""ctypes front-end to the checkers (TEST INFRASTRUCTURE).

Two shared libraries, both built by ``oracle/Makefile``:

* ``build/liboracle.so`` -- the C restatement ``smc_oracle.c`` (always built);
* ``_ref/libvsmc_ref.so`` -- ``ref_harness.cpp`` over the unmodified vSMC
  headers (built where the vSMC include tree exists; the built file travels).

Only tests, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` may
import this module, and only to check or to time the reference.  The product
(``vsmc_b200``) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "build", "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libvsmc_ref.so")

SCHEMES = {
    "Multinomial": 0,
    "Residual": 1,
    "Stratified": 2,
    "Systematic": 3,
    "ResidualStratified": 4,
    "ResidualSystematic": 5,
}

# dt, sd_pos, sd_vel, sd_pos0, sd_vel0, scale, nu
CV_DEFAULT = (0.1, 0.02, 0.5, 2.0, 1.0, 10.0, 10.0)

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build() -> None:
    """Build both checkers (the reference one only where the environment's
    VSMC_ROOT names a vSMC tree; otherwise a prebuilt _ref/ is used)."""
    cmd = ["make", "-s", "-C", HERE]
    if os.environ.get("VSMC_ROOT"):
        cmd.append("VSMC_ROOT=" + os.environ["VSMC_ROOT"])
    subprocess.run(cmd, check=True)


class _CVParam(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("dt", "sd_pos", "sd_vel", "sd_pos0", "sd_vel0", "scale", "nu")]


class _CVOut(C.Structure):
    _fields_ = [
        ("ess", C.POINTER(C.c_double)),
        ("resampled", C.POINTER(C.c_int32)),
        ("logz_inc", C.POINTER(C.c_double)),
        ("mean_x", C.POINTER(C.c_double)),
        ("mean_y", C.POINTER(C.c_double)),
        ("final_state", C.POINTER(C.c_double)),
        ("final_lw", C.POINTER(C.c_double)),
        ("words_used", C.POINTER(C.c_uint64)),
        ("last_copy_from", C.POINTER(C.c_int64)),
    ]


class _OrcThreefry(C.Structure):
    _fields_ = [("key", C.c_uint64 * 4), ("ctr", C.c_uint64 * 4),
                ("buf", C.c_uint64 * 4), ("index", C.c_uint)]


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        L.orc_philox_stream.argtypes = [_u32p, _u32p, C.c_uint64, C.c_uint64, _u32p]
        L.orc_threefry_stream.argtypes = [_u64p, _u64p, C.c_uint64, C.c_uint64, _u64p]
        L.orc_philox4x32_block.argtypes = [_u32p, _u32p, _u32p]
        L.orc_threefry4x64_block.argtypes = [_u64p, _u64p, _u64p]
        L.orc_canonical_u64.argtypes = [C.c_uint64]
        L.orc_canonical_u64.restype = C.c_double
        L.orc_canonical_u32x2.argtypes = [C.c_uint32, C.c_uint32]
        L.orc_canonical_u32x2.restype = C.c_double
        L.orc_add_log_weight.argtypes = [C.c_size_t, _f64p, _f64p, C.c_void_p]
        L.orc_add_log_weight.restype = C.c_double
        L.orc_threefry_seed.argtypes = [C.POINTER(_OrcThreefry), C.c_uint64]
        L.orc_threefry_next.argtypes = [C.POINTER(_OrcThreefry)]
        L.orc_threefry_next.restype = C.c_uint64
        L.orc_threefry_words_used.argtypes = [C.POINTER(_OrcThreefry)]
        L.orc_threefry_words_used.restype = C.c_uint64
        L.orc_resample.argtypes = [C.c_int, C.c_size_t, C.c_size_t,
                                   C.POINTER(_OrcThreefry), _f64p, _i64p,
                                   C.c_void_p, C.POINTER(C.c_size_t)]
        L.orc_inversion.argtypes = [C.c_size_t, C.c_size_t, _f64p, _f64p, _i64p]
        L.orc_cfrp_trans.argtypes = [C.c_size_t, C.c_size_t, _i64p, _i64p]
        L.orc_cv_loglik.argtypes = [C.POINTER(_CVParam)] + [C.c_double] * 4
        L.orc_cv_loglik.restype = C.c_double
        L.orc_cv_init_particle.argtypes = [C.POINTER(_CVParam), _u32p, C.c_uint32,
                                           C.c_uint32, _f64p]
        L.orc_cv_move_particle.argtypes = [C.POINTER(_CVParam), _u32p, C.c_uint32,
                                           C.c_uint32, C.c_uint32, _f64p]
        L.orc_cv_simulate.argtypes = [C.POINTER(_CVParam), C.c_uint32, C.c_uint32,
                                      C.c_size_t, _f64p, _f64p, C.c_void_p]
        L.orc_cv_filter.argtypes = [C.POINTER(_CVParam), C.c_size_t, C.c_size_t,
                                    C.c_int, C.c_double, C.c_uint32, C.c_uint32,
                                    _f64p, _f64p, C.POINTER(_CVOut)]
        L.orc_cv_filter.restype = C.c_double
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            build()
        if not os.path.exists(REF_SO):
            raise RuntimeError("reference harness not built (vSMC headers absent)")
        L = C.CDLL(REF_SO)
        L.ref_philox_stream.argtypes = [_u32p, _u32p, C.c_uint64, C.c_uint64, _u32p]
        L.ref_threefry_stream.argtypes = [_u64p, _u64p, C.c_uint64, C.c_uint64, _u64p]
        L.ref_resample.argtypes = [C.c_int, C.c_uint64, C.c_uint64, C.c_uint64,
                                   C.c_uint64, _f64p, _i64p, C.c_void_p]
        L.ref_resample.restype = C.c_uint64
        L.ref_weight_set.argtypes = [C.c_uint64, _f64p, C.c_void_p, _f64p, _f64p]
        L.ref_weight_set.restype = C.c_double
        L.ref_cv_filter.argtypes = [C.c_int, C.c_int, _f64p, C.c_uint64, C.c_uint64,
                                    C.c_int, C.c_double, C.c_uint, C.c_uint,
                                    _f64p, _f64p] + [C.c_void_p] * 10
        L.ref_cv_filter.restype = C.c_double
        L.ref_max_threads.restype = C.c_int
        _ref = L
    return _ref


# ------------------------------------------------------------ RNG streams --

def philox_stream(key, ctr, n, skip=0, use_ref=False):
    out = np.zeros(n, np.uint32)
    k = np.asarray(key, np.uint32)
    c = np.asarray(ctr, np.uint32)
    (ref().ref_philox_stream if use_ref else lib().orc_philox_stream)(k, c, skip, n, out)
    return out


def threefry_stream(key, ctr, n, skip=0, use_ref=False):
    out = np.zeros(n, np.uint64)
    k = np.asarray(key, np.uint64)
    c = np.asarray(ctr, np.uint64)
    (ref().ref_threefry_stream if use_ref else lib().orc_threefry_stream)(k, c, skip, n, out)
    return out


def canonical_u64(x):
    return lib().orc_canonical_u64(int(x))


def canonical_u32x2(a, b):
    return lib().orc_canonical_u32x2(int(a), int(b))


# --------------------------------------------------------------- weights --

def add_log_weight(lw, inc=None):
    """WeightSet::set_log_weight(lw) [then add_log_weight(inc)] -> (ess, w, lw)."""
    lw = np.array(lw, np.float64)
    w = np.zeros_like(lw)
    L = lib()
    ess = L.orc_add_log_weight(lw.size, lw, w, None)
    if inc is not None:
        inc = np.ascontiguousarray(inc, np.float64)
        ess = L.orc_add_log_weight(lw.size, lw, w, inc.ctypes.data)
    return ess, w, lw


def ref_weight_set(lw, inc=None):
    lw = np.ascontiguousarray(lw, np.float64)
    w = np.zeros_like(lw)
    lwo = np.zeros_like(lw)
    incp = None if inc is None else np.ascontiguousarray(inc, np.float64)
    ess = ref().ref_weight_set(lw.size, lw, None if incp is None else incp.ctypes.data, w, lwo)
    return ess, w, lwo


def ref_weight_prospective(lw, inc, use_log, cess):
    """WeightSet::set_log_weight(lw) then ess(inc, use_log) or cess(inc,
    use_log), through vSMC."""
    L = ref()
    L.ref_weight_prospective.restype = C.c_double
    L.ref_weight_prospective.argtypes = [C.c_uint64, _f64p, _f64p, C.c_int, C.c_int]
    lw = np.ascontiguousarray(lw, np.float64)
    inc = np.ascontiguousarray(inc, np.float64)
    return L.ref_weight_prospective(lw.size, lw, inc, 1 if use_log else 0,
                                    1 if cess else 0)


# -------------------------------------------------------------- resample --

def resample(scheme, weights, seed, skip=0, M=None, N=None, want_uniforms=False):
    """Resample<scheme>(M, N, Threefry4x64(seed) after `skip` words, w) then
    cfrp_trans.  Returns (replication, copy_from, words_drawn, uniforms)."""
    w = np.ascontiguousarray(weights, np.float64)
    M = w.size if M is None else M
    N = M if N is None else N
    L = lib()
    eng = _OrcThreefry()
    L.orc_threefry_seed(C.byref(eng), seed)
    for _ in range(skip):
        L.orc_threefry_next(C.byref(eng))
    rep = np.zeros(max(M, 1), np.int64)
    uni = np.zeros(max(N, 1), np.float64)
    nu = C.c_size_t(0)
    L.orc_resample(scheme, M, N, C.byref(eng), w, rep, uni.ctypes.data, C.byref(nu))
    words = L.orc_threefry_words_used(C.byref(eng)) - skip
    cf = np.zeros(max(N, 1), np.int64)
    if N > 0 and M > 0:
        L.orc_cfrp_trans(M, N, rep, cf)
    out = (rep[:M], cf[:N], int(words))
    if want_uniforms:
        out = out + (uni[: nu.value].copy(),)
    return out


def ref_resample(scheme, weights, seed, skip=0, M=None, N=None):
    w = np.ascontiguousarray(weights, np.float64)
    M = w.size if M is None else M
    N = M if N is None else N
    rep = np.zeros(max(M, 1), np.int64)
    cf = np.zeros(max(N, 1), np.int64)
    words = ref().ref_resample(scheme, M, N, seed, skip, w, rep, cf.ctypes.data)
    return rep[:M], cf[:N], int(words)


def inversion(weights, uniforms, N=None):
    w = np.ascontiguousarray(weights, np.float64)
    u = np.ascontiguousarray(uniforms, np.float64)
    N = u.size if N is None else N
    rep = np.zeros(max(w.size, 1), np.int64)
    lib().orc_inversion(w.size, N, w, u, rep)
    return rep[: w.size]


def cfrp_trans(rep, N=None):
    r = np.ascontiguousarray(rep, np.int64)
    N = int(r.sum()) if N is None else N
    cf = np.zeros(max(N, 1), np.int64)
    lib().orc_cfrp_trans(r.size, N, r, cf)
    return cf[:N]


# -------------------------------------------------------------- CV model --

def _param(p=CV_DEFAULT):
    return _CVParam(*p)


def cv_simulate(T, obs_seed, stream=0, param=CV_DEFAULT, want_truth=False):
    ox = np.zeros(T, np.float64)
    oy = np.zeros(T, np.float64)
    truth = np.zeros((T, 4), np.float64)
    lib().orc_cv_simulate(C.byref(_param(param)), obs_seed, stream, T, ox, oy,
                          truth.ctypes.data)
    return (ox, oy, truth) if want_truth else (ox, oy)


def cv_loglik(x, y, ox, oy, param=CV_DEFAULT):
    return lib().orc_cv_loglik(C.byref(_param(param)), x, y, ox, oy)


def cv_init_particle(key, pid, stream=0, param=CV_DEFAULT):
    s = np.zeros(4, np.float64)
    lib().orc_cv_init_particle(C.byref(_param(param)), np.asarray(key, np.uint32),
                               pid, stream, s)
    return s


def cv_move_particle(s, key, it, pid, stream=0, param=CV_DEFAULT):
    s = np.array(s, np.float64)
    lib().orc_cv_move_particle(C.byref(_param(param)), np.asarray(key, np.uint32),
                               it, pid, stream, s)
    return s


class CVResult(dict):
    pass


def cv_filter(N, T, scheme, obs_x, obs_y, seed=101, stream=0, threshold=0.5,
              param=CV_DEFAULT, want_state=False):
    """The oracle's FP64 filter.  Returns a dict with logz, ess, resampled,
    logz_inc, mean_x, mean_y (and state, lw, words_used)."""
    ox = np.ascontiguousarray(obs_x, np.float64)
    oy = np.ascontiguousarray(obs_y, np.float64)
    r = CVResult(
        ess=np.zeros(T), resampled=np.zeros(T, np.int32), logz_inc=np.zeros(T),
        mean_x=np.zeros(T), mean_y=np.zeros(T))
    st = np.zeros(4 * N) if want_state else None
    lw = np.zeros(N) if want_state else None
    wu = np.zeros(1, np.uint64)
    out = _CVOut(_ptr(r["ess"], C.c_double), _ptr(r["resampled"], C.c_int32),
                 _ptr(r["logz_inc"], C.c_double), _ptr(r["mean_x"], C.c_double),
                 _ptr(r["mean_y"], C.c_double), _ptr(st, C.c_double),
                 _ptr(lw, C.c_double), _ptr(wu, C.c_uint64), None)
    r["logz"] = lib().orc_cv_filter(C.byref(_param(param)), N, T, scheme, threshold,
                                    seed, stream, ox, oy, C.byref(out))
    r["words_used"] = int(wu[0])
    if want_state:
        r["state"] = st.reshape(4, N)
        r["lw"] = lw
    return r


def ref_cv_filter(N, T, scheme, obs_x, obs_y, seed=101, stream=0, threshold=0.5,
                  param=CV_DEFAULT, backend=0, nthreads=0, want_state=False):
    """The same filter through vSMC's Sampler (backend 0 OMP, 1 STD, 2 SEQ)."""
    ox = np.ascontiguousarray(obs_x, np.float64)
    oy = np.ascontiguousarray(obs_y, np.float64)
    r = CVResult(
        ess=np.zeros(T), resampled=np.zeros(T, np.int32), logz_inc=np.zeros(T),
        mean_x=np.zeros(T), mean_y=np.zeros(T))
    st = np.zeros(4 * N) if want_state else None
    lw = np.zeros(N) if want_state else None
    wu = np.zeros(1, np.uint64)
    sec = np.zeros(1)
    r["step_seconds"] = np.zeros(T)
    p = np.asarray(param, np.float64)
    args = [r["ess"], r["resampled"], r["logz_inc"], r["mean_x"], r["mean_y"], st, lw,
            wu, sec, r["step_seconds"]]
    r["logz"] = ref().ref_cv_filter(backend, nthreads, p, N, T, scheme, threshold, seed,
                                    stream, ox, oy,
                                    *[a.ctypes.data if a is not None else None
                                      for a in args])
    r["words_used"] = int(wu[0])
    r["seconds"] = float(sec[0])
    if want_state:
        r["state"] = st.reshape(4, N)
        r["lw"] = lw
    return r


def ref_cv_filter_trace(N, T, scheme, obs_x, obs_y, seed=101, stream=0, threshold=0.5,
                        param=CV_DEFAULT, nthreads=0, weights_step=None):
    """vSMC's Sampler (StateOMP) on the filter, with a trace of the run:
    ``copy_from`` (T x N int32; rows of steps that resampled are
    Particle::resample's copy_from), ``words_before`` (the resample engine's
    words drawn before each step's resampling) and, for ``weights_step``, the
    normalised weights that step resampled with."""
    ox = np.ascontiguousarray(obs_x, np.float64)
    oy = np.ascontiguousarray(obs_y, np.float64)
    L = ref()
    L.ref_cv_filter_trace.restype = C.c_double
    L.ref_cv_filter_trace.argtypes = [C.c_int, C.c_void_p, C.c_uint64, C.c_uint64,
                                      C.c_int, C.c_double, C.c_uint, C.c_uint,
                                      C.c_void_p, C.c_void_p] + [C.c_void_p] * 8 + [
                                      C.c_uint64, C.c_void_p, C.c_void_p]
    r = CVResult(
        ess=np.zeros(T), resampled=np.zeros(T, np.int32), logz_inc=np.zeros(T),
        mean_x=np.zeros(T), mean_y=np.zeros(T))
    r["copy_from"] = np.full((T, N), -1, np.int32)
    r["words_before"] = np.zeros(T, np.uint64)
    wu = np.zeros(1, np.uint64)
    sec = np.zeros(1)
    w = np.zeros(N) if weights_step is not None else None
    p = np.asarray(param, np.float64)
    r["logz"] = L.ref_cv_filter_trace(
        nthreads, p.ctypes.data, N, T, scheme, threshold, seed, stream,
        ox.ctypes.data, oy.ctypes.data, r["ess"].ctypes.data, r["resampled"].ctypes.data,
        r["logz_inc"].ctypes.data, r["mean_x"].ctypes.data, r["mean_y"].ctypes.data,
        wu.ctypes.data, r["copy_from"].ctypes.data,
        None if w is None else w.ctypes.data, 0 if weights_step is None else weights_step,
        r["words_before"].ctypes.data, sec.ctypes.data)
    r["words_used"] = int(wu[0])
    r["seconds"] = float(sec[0])
    if w is not None:
        r["weights"] = w
    return r


def ref_cv_summary(N, T, scheme, obs_x, obs_y, seed=101, stream=0, threshold=0.5,
                   param=CV_DEFAULT) -> str:
    """The summary table vSMC's `os << sampler` writes for the same filter
    (Sampler::print, core/sampler.hpp:684-721; monitor "pos" named pos.x and
    pos.y as in example/pf/include/pf_smp_do.hpp)."""
    ox = np.ascontiguousarray(obs_x, np.float64)
    oy = np.ascontiguousarray(obs_y, np.float64)
    p = np.asarray(param, np.float64)
    L = ref()
    L.ref_cv_summary.restype = C.c_uint64
    L.ref_cv_summary.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_int, C.c_double,
                                 C.c_uint, C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p,
                                 C.c_uint64]
    args = (p.ctypes.data, N, T, scheme, threshold, seed, stream,
            ox.ctypes.data, oy.ctypes.data)
    n = L.ref_cv_summary(*args, None, 0)
    buf = C.create_string_buffer(int(n) + 1)
    L.ref_cv_summary(*args, buf, int(n) + 1)
    return buf.value.decode()


PAPER_REF_SO = os.path.join(HERE, "_ref", "libvsmc_paper_ref.so")


def paper_ref_available() -> bool:
    return os.path.exists(PAPER_REF_SO)


def ref_paper_pf_summary(N, T, obs_x, obs_y, seed=101) -> str:
    """`os << sampler` of the reference's example/paper particle filter
    (paper_pf.cpp's own cv, cv_init, cv_move and monitor, Stratified at
    ESS < N/2, through vSMC's Sampler) on the given observations, which are
    written to the 100-row data file the example reads."""
    import tempfile

    L = C.CDLL(PAPER_REF_SO)
    L.ref_paper_pf_summary.restype = C.c_uint64
    L.ref_paper_pf_summary.argtypes = [C.c_uint64, C.c_uint64, C.c_uint, C.c_char_p,
                                       C.c_char_p, C.c_uint64]
    ox = np.zeros(100)
    oy = np.zeros(100)
    ox[:len(obs_x)] = obs_x
    oy[:len(obs_y)] = obs_y
    fd, path = tempfile.mkstemp(suffix=".data")
    try:
        with os.fdopen(fd, "w") as f:
            for a, b in zip(ox, oy):
                f.write(f"{float(a)!r} {float(b)!r}\n")
        n = L.ref_paper_pf_summary(N, T, seed, path.encode(), None, 0)
        buf = C.create_string_buffer(int(n) + 1)
        L.ref_paper_pf_summary(N, T, seed, path.encode(), buf, int(n) + 1)
    finally:
        os.unlink(path)
    return buf.value.decode()


def ref_max_threads() -> int:
    return ref().ref_max_threads()


# ----------------------------------------------------------------- GMM ----

GMM_REF_SO = os.path.join(HERE, "_ref", "libvsmc_gmm_ref.so")
_gmm_ref = None


def gmm_ref_available() -> bool:
    return os.path.exists(GMM_REF_SO)


def gmm_simulate(n=1000, seed=1):
    """The mixture data (orc_gmm_simulate)."""
    out = np.zeros(n)
    L = lib()
    L.orc_gmm_simulate.argtypes = [C.c_uint32, C.c_size_t, C.c_void_p]
    L.orc_gmm_simulate.restype = None
    L.orc_gmm_simulate(seed, n, out.ctypes.data)
    return out


def _gmm_outputs(N, iters, sweeps):
    T = iters + 1
    r = CVResult(ess=np.zeros(T), resampled=np.zeros(T, np.int32), zinc=np.zeros(T),
                 integrand=np.zeros(T), grid=np.zeros(T),
                 accept=np.zeros((T, 1 + 3 * sweeps), np.int64),
                 params=np.zeros((N, 14)), lw=np.zeros(N), words=np.zeros(N, np.uint64))
    order = ("ess", "resampled", "zinc", "integrand", "grid", "accept", "params", "lw", "words")
    return r, [r[k].ctypes.data for k in order]


def gmm_smc(data, N, iters=100, power=4, sweeps=5, sd=0.1, scheme=3, threshold=0.5,
            seed=101):
    """The tempered SMC sampler, C restatement (orc_gmm_smc)."""
    data = np.ascontiguousarray(data, np.float64)
    L = lib()
    L.orc_gmm_smc.argtypes = ([C.c_void_p, C.c_size_t, C.c_size_t, C.c_size_t, C.c_int,
                               C.c_int, C.c_double, C.c_int, C.c_double, C.c_uint32]
                              + [C.c_void_p] * 10)
    L.orc_gmm_smc.restype = C.c_double
    r, ptrs = _gmm_outputs(N, iters, sweeps)
    pl = np.zeros(1)
    r["logz"] = L.orc_gmm_smc(data.ctypes.data, data.size, N, iters, power, sweeps, sd,
                              scheme, threshold, seed, *ptrs, pl.ctypes.data)
    r["path_logz"] = float(pl[0])
    return r


def gmm_loglik(data, mu, lam, weight):
    L = lib()
    L.orc_gmm_loglik.argtypes = [C.c_void_p, C.c_size_t] + [C.c_void_p] * 3
    L.orc_gmm_loglik.restype = C.c_double
    data = np.ascontiguousarray(data, np.float64)
    a = [np.ascontiguousarray(v, np.float64) for v in (mu, lam, weight)]
    return L.orc_gmm_loglik(data.ctypes.data, data.size, *[v.ctypes.data for v in a])


def gmm_ref():
    global _gmm_ref
    if _gmm_ref is None:
        if not os.path.exists(GMM_REF_SO):
            build()
        if not os.path.exists(GMM_REF_SO):
            raise RuntimeError("GMM reference harness not built (vSMC tree absent)")
        L = C.CDLL(GMM_REF_SO)
        L.ref_gmm_smc.argtypes = ([C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_int,
                                   C.c_int, C.c_double, C.c_int, C.c_double, C.c_uint,
                                   C.c_int] + [C.c_void_p] * 11)
        L.ref_gmm_smc.restype = C.c_double
        L.ref_gmm_summary.argtypes = ([C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_int,
                                       C.c_double, C.c_int, C.c_double, C.c_uint, C.c_void_p,
                                       C.c_uint64])
        L.ref_gmm_summary.restype = C.c_uint64
        _gmm_ref = L
    return _gmm_ref


def ref_gmm_smc(data, N, iters=100, power=4, sweeps=5, sd=0.1, scheme=3, threshold=0.5,
                seed=101, nthreads=0):
    """The same sampler through vSMC with the reference's example/gmm classes."""
    data = np.ascontiguousarray(data, np.float64)
    r, ptrs = _gmm_outputs(N, iters, sweeps)
    pl, sec = np.zeros(1), np.zeros(1)
    r["logz"] = gmm_ref().ref_gmm_smc(data.ctypes.data, data.size, N, iters, power, sweeps,
                                      sd, scheme, threshold, seed, nthreads, *ptrs,
                                      pl.ctypes.data, sec.ctypes.data)
    r["path_logz"] = float(pl[0])
    r["seconds"] = float(sec[0])
    return r


def ref_gmm_summary(data, N, iters=100, sweeps=5, sd=0.1, scheme=3, threshold=0.5,
                    seed=101) -> str:
    data = np.ascontiguousarray(data, np.float64)
    L = gmm_ref()
    args = (data.ctypes.data, data.size, N, iters, sweeps, sd, scheme, threshold, seed)
    n = L.ref_gmm_summary(*args, None, 0)
    buf = C.create_string_buffer(int(n) + 1)
    L.ref_gmm_summary(*args, buf, int(n) + 1)
    return buf.value.decode()
