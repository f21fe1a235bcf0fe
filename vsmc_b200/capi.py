"""ctypes binding of libvsmc_cuda (the C ABI declared in include/vsmc_cuda.h).

This is the Python host mirror used by the tests and bench.py: it calls the
sm_100a kernels through the C ABI with raw device pointers and raises
``VsmcCudaError`` on any non-zero status.  There is no CPU path: loading
fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libvsmc_cuda.so")

OK, EINVAL, ENOMEM, EDEGENERATE, ETIMEOUT, ECUDA = range(6)

# vsmc::ResampleScheme values (include/vsmc/resample/common.hpp:124-131)
Multinomial, Residual, Stratified, Systematic, ResidualStratified, ResidualSystematic = range(6)
SCHEME_NAMES = ("Multinomial", "Residual", "Stratified", "Systematic",
                "ResidualStratified", "ResidualSystematic")
FP64, MIXED = 0, 1


class VsmcCudaError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        super().__init__(f"{where}: status {status} ({message})")
        self.status = status


class CVConfig(C.Structure):
    _fields_ = [
        ("N", C.c_uint64), ("T_max", C.c_uint64), ("scheme", C.c_int),
        ("form", C.c_int), ("threshold", C.c_double), ("seed", C.c_uint32),
        ("stream_id", C.c_uint32), ("dt", C.c_double), ("sd_pos", C.c_double),
        ("sd_vel", C.c_double), ("sd_pos0", C.c_double), ("sd_vel0", C.c_double),
        ("scale", C.c_double), ("nu", C.c_double)]


class ThreefryState(C.Structure):
    _fields_ = [("key", C.c_uint64 * 4), ("ctr", C.c_uint64 * 4),
                ("offset", C.c_uint64)]


class CVResult(C.Structure):
    _fields_ = [("request", C.c_uint64), ("t", C.c_uint64), ("ess", C.c_double),
                ("logz_inc", C.c_double), ("log_evidence", C.c_double),
                ("resampled", C.c_int32), ("status", C.c_int32),
                ("submit_ns", C.c_int64), ("done_ns", C.c_int64)]


class ServerCounters(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("opened", "admitted", "completed", "ticks", "steps",
                                          "particle_steps", "max_active", "waiting",
                                          "active")] + [("busy_seconds", C.c_double)]


class GmmConfig(C.Structure):
    _fields_ = [("N", C.c_uint64), ("iters", C.c_uint64), ("power", C.c_int),
                ("sweeps", C.c_int), ("sd", C.c_double), ("scheme", C.c_int),
                ("threshold", C.c_double), ("seed", C.c_uint32), ("form", C.c_int),
                ("group", C.c_int)]


_lib = None


def lib():
    """Load libvsmc_cuda.so (built by vsmc_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m vsmc_b200.build` "
            "(nvcc, sm_100a); there is no CPU fallback")
    L = C.CDLL(LIB_PATH)
    vp, u64, i32, f64 = C.c_void_p, C.c_uint64, C.c_int, C.c_double
    L.vsmc_cuda_last_error.restype = C.c_char_p
    L.vsmc_cuda_status_string.restype = C.c_char_p
    L.vsmc_cuda_status_string.argtypes = [i32]
    L.vsmc_cuda_abi_version.restype = i32
    L.vsmc_cuda_philox4x32_words.argtypes = [vp, vp, u64, u64, vp, vp]
    L.vsmc_cuda_threefry4x64_words.argtypes = [vp, vp, u64, u64, vp, vp]
    L.vsmc_cuda_weight_add_log.argtypes = [u64, vp, vp, vp, C.POINTER(f64), vp]
    L.vsmc_cuda_resample_workspace_size.restype = C.c_size_t
    L.vsmc_cuda_resample_workspace_size.argtypes = [u64]
    L.vsmc_cuda_resample.argtypes = [i32, u64, vp, vp, u64, C.POINTER(ThreefryState),
                                     vp, vp, vp, C.c_size_t, vp]
    L.vsmc_cuda_copy_f64.argtypes = [u64, C.c_uint32, vp, vp, vp, vp]
    L.vsmc_cuda_math_eval.argtypes = [C.c_int, u64, vp, vp, vp]
    L.vsmc_cuda_resample_mn_workspace_size.restype = C.c_size_t
    L.vsmc_cuda_resample_mn_workspace_size.argtypes = [u64, u64]
    L.vsmc_cuda_resample_mn.argtypes = [i32, u64, u64, vp, vp, u64,
                                        C.POINTER(ThreefryState), vp, vp, vp,
                                        C.c_size_t, vp]
    L.vsmc_cuda_weight_ess.argtypes = [u64, vp, vp, vp, i32, C.POINTER(f64), vp]
    L.vsmc_cuda_weight_cess.argtypes = [u64, vp, vp, i32, C.POINTER(f64), vp]
    L.vsmc_cuda_resample_noalloc.argtypes = [i32, u64, vp, vp, u64,
                                             C.POINTER(ThreefryState), vp, vp, vp]
    L.vsmc_cuda_cv_config_default.argtypes = [C.POINTER(CVConfig)]
    L.vsmc_cuda_cv_config_default.restype = None
    L.vsmc_cuda_cv_device_bytes.argtypes = [C.POINTER(CVConfig)]
    L.vsmc_cuda_cv_device_bytes.restype = C.c_size_t
    L.vsmc_cuda_cv_create.argtypes = [C.POINTER(CVConfig), vp, C.POINTER(vp)]
    L.vsmc_cuda_cv_destroy.argtypes = [vp]
    L.vsmc_cuda_cv_set_observations.argtypes = [vp, vp, vp, u64, i32]
    L.vsmc_cuda_cv_initialize.argtypes = [vp]
    L.vsmc_cuda_cv_iterate.argtypes = [vp, u64]
    L.vsmc_cuda_cv_synchronize.argtypes = [vp]
    L.vsmc_cuda_cv_iter_size.argtypes = [vp, C.POINTER(u64)]
    L.vsmc_cuda_cv_history.argtypes = [vp, vp, vp, vp, vp, vp]
    L.vsmc_cuda_cv_log_evidence.argtypes = [vp, C.POINTER(f64)]
    L.vsmc_cuda_cv_read_state.argtypes = [vp, vp, vp, vp, vp, vp]
    L.vsmc_cuda_cv_resample_words.argtypes = [vp, C.POINTER(u64)]
    L.vsmc_cuda_cv_copy_from.argtypes = [vp, vp, vp]
    L.vsmc_cuda_cv_append_observations.argtypes = [vp, vp, vp, u64, i32]
    L.vsmc_cuda_cv_read_step.argtypes = [vp, u64, vp, vp, vp, i32]
    L.vsmc_cuda_cv_set_timing.argtypes = [vp, i32]
    L.vsmc_cuda_cv_set_ancestry.argtypes = [vp, vp, vp, vp]
    L.vsmc_cuda_cv_complete_monitor.argtypes = [vp]
    L.vsmc_cuda_cv_timing.argtypes = [vp, C.POINTER(f64), C.POINTER(f64), C.POINTER(u64),
                                      C.POINTER(u64)]
    L.vsmc_cuda_cv_simulate.argtypes = [C.POINTER(CVConfig), C.c_uint32, u64, vp, vp, vp]
    u32 = C.c_uint32
    L.vsmc_cuda_cv_batch_slot_bytes.restype = u64
    L.vsmc_cuda_cv_batch_slot_bytes.argtypes = [C.POINTER(CVConfig), u64, u64]
    L.vsmc_cuda_cv_batch_create.argtypes = [C.POINTER(CVConfig), u32, u64, vp, C.POINTER(vp)]
    L.vsmc_cuda_cv_batch_destroy.argtypes = [vp]
    L.vsmc_cuda_cv_batch_admit.argtypes = [vp, u64, u64, u32, u32, C.POINTER(u32)]
    L.vsmc_cuda_cv_batch_release.argtypes = [vp, u32]
    L.vsmc_cuda_cv_batch_bytes_in_use.argtypes = [vp, C.POINTER(u64)]
    L.vsmc_cuda_cv_batch_set_observations.argtypes = [vp, u32, vp, vp, vp, vp, i32]
    L.vsmc_cuda_cv_batch_append_observations.argtypes = [vp, u32, vp, vp, vp]
    L.vsmc_cuda_cv_batch_initialize.argtypes = [vp, u32, vp]
    L.vsmc_cuda_cv_batch_step.argtypes = [vp, u32, vp]
    L.vsmc_cuda_cv_batch_run.argtypes = [vp, u32, vp]
    L.vsmc_cuda_cv_batch_read_last.argtypes = [vp, u32, vp, vp, vp, vp, vp, vp]
    L.vsmc_cuda_cv_batch_iter_size.argtypes = [vp, u32, C.POINTER(u64)]
    L.vsmc_cuda_cv_batch_history.argtypes = [vp, u32, vp, vp, vp, vp, vp]
    L.vsmc_cuda_cv_batch_synchronize.argtypes = [vp]
    L.vsmc_cuda_cv_batch_launches.argtypes = [vp, C.POINTER(u64)]
    L.vsmc_cuda_cv_batch_set_graphs.argtypes = [vp, i32]
    L.vsmc_cuda_cv_batch_set_launch_shape.argtypes = [vp, C.c_int, C.c_int]
    L.vsmc_cuda_cv_batch_read_steps.argtypes = [vp, u32, vp, vp, vp, vp, vp, vp]
    L.vsmc_cuda_cv_batch_set_tiling.argtypes = [vp, C.c_int]
    L.vsmc_cuda_cv_batch_tiling.argtypes = [vp, C.POINTER(C.c_int)]
    L.vsmc_cuda_cv_batch_autotune.argtypes = [vp, u32, vp, C.POINTER(C.c_int),
                                              C.POINTER(C.c_int)]
    L.vsmc_cuda_cv_server_create.argtypes = [C.POINTER(CVConfig), u32, u64, C.POINTER(vp)]
    L.vsmc_cuda_cv_server_destroy.argtypes = [vp]
    L.vsmc_cuda_cv_server_now_ns.argtypes = [vp]
    L.vsmc_cuda_cv_server_now_ns.restype = C.c_int64
    L.vsmc_cuda_cv_server_open.argtypes = [vp, u64, u64, u32, u32, C.POINTER(u64)]
    L.vsmc_cuda_cv_server_observe.argtypes = [vp, u32, vp, vp, vp, vp]
    L.vsmc_cuda_cv_server_close.argtypes = [vp, u64]
    L.vsmc_cuda_cv_server_poll.argtypes = [vp, vp, u32, C.POINTER(u32), i32]
    L.vsmc_cuda_cv_server_drain.argtypes = [vp, i32]
    L.vsmc_cuda_cv_server_stats.argtypes = [vp, C.POINTER(ServerCounters)]
    L.vsmc_cuda_gmm_config_default.argtypes = [C.POINTER(GmmConfig)]
    L.vsmc_cuda_gmm_config_default.restype = None
    L.vsmc_cuda_gmm_create.argtypes = [C.POINTER(GmmConfig), vp, u64, vp, C.POINTER(vp)]
    L.vsmc_cuda_gmm_destroy.argtypes = [vp]
    L.vsmc_cuda_gmm_initialize.argtypes = [vp]
    L.vsmc_cuda_gmm_iterate.argtypes = [vp, u64]
    L.vsmc_cuda_gmm_iter_size.argtypes = [vp, C.POINTER(u64)]
    L.vsmc_cuda_gmm_history.argtypes = [vp] + [vp] * 6
    L.vsmc_cuda_gmm_log_evidence.argtypes = [vp, C.POINTER(f64), C.POINTER(f64)]
    L.vsmc_cuda_gmm_read_params.argtypes = [vp, vp, vp, vp]
    L.vsmc_cuda_gmm_loglik.argtypes = [vp, i32, vp]
    L.vsmc_cuda_gmm_group.argtypes = [vp, C.POINTER(C.c_int)]
    L.vsmc_cuda_gmm_set_timing.argtypes = [vp, i32]
    L.vsmc_cuda_gmm_timing.argtypes = [vp, C.POINTER(f64), C.POINTER(u64), C.POINTER(u64)]
    L.vsmc_cuda_gmm_simulate.argtypes = [u32, u64, vp]
    _lib = L
    return L


def check(status: int, where: str) -> None:
    if status != OK:
        msg = lib().vsmc_cuda_last_error().decode(errors="replace")
        raise VsmcCudaError(status, where, msg)


def _np_ptr(a):
    return None if a is None else a.ctypes.data


# --------------------------------------------------------------- RNG -------

def philox4x32_words(key, ctr, skip, n, out_ptr, stream=None):
    k = (C.c_uint32 * 2)(*key)
    c = (C.c_uint32 * 4)(*ctr)
    check(lib().vsmc_cuda_philox4x32_words(k, c, skip, n, out_ptr, stream),
          "vsmc_cuda_philox4x32_words")


def threefry4x64_words(key, ctr, skip, n, out_ptr, stream=None):
    k = (C.c_uint64 * 4)(*key)
    c = (C.c_uint64 * 4)(*ctr)
    check(lib().vsmc_cuda_threefry4x64_words(k, c, skip, n, out_ptr, stream),
          "vsmc_cuda_threefry4x64_words")


# ----------------------------------------------------------- weights -------

def weight_add_log(N, lw_ptr, w_ptr=None, inc_ptr=None, stream=None) -> float:
    ess = C.c_double(0.0)
    check(lib().vsmc_cuda_weight_add_log(N, lw_ptr, w_ptr, inc_ptr, C.byref(ess), stream),
          "vsmc_cuda_weight_add_log")
    return ess.value


# ---------------------------------------------------------- resample -------

def resample_workspace_size(N) -> int:
    return int(lib().vsmc_cuda_resample_workspace_size(N))


def threefry_state(seed=0, key=None, ctr=(0, 0, 0, 0), offset=0) -> ThreefryState:
    st = ThreefryState()
    k = key if key is not None else (seed, 0, 0, 0)
    for i in range(4):
        st.key[i] = k[i]
        st.ctr[i] = ctr[i]
    st.offset = offset
    return st


def resample(scheme, N, weight_ptr, rng: ThreefryState, rep_ptr, cf_ptr, ws_ptr, ws_bytes,
             uniforms_ptr=None, n_uniforms=0, stream=None) -> int:
    """Returns the number of engine words drawn; rng.offset advances."""
    before = rng.offset
    check(lib().vsmc_cuda_resample(scheme, N, weight_ptr, uniforms_ptr, n_uniforms,
                                   C.byref(rng), rep_ptr, cf_ptr, ws_ptr, ws_bytes, stream),
          "vsmc_cuda_resample")
    return int(rng.offset - before)


def resample_mn_workspace_size(M, N) -> int:
    return int(lib().vsmc_cuda_resample_mn_workspace_size(M, N))


def resample_mn(scheme, M, N, weight_ptr, rng: ThreefryState, rep_ptr, cf_ptr, ws_ptr,
                ws_bytes, uniforms_ptr=None, n_uniforms=0, stream=None) -> int:
    """Resample(M, N) + cfrp_trans(M, N); returns the engine words drawn."""
    before = rng.offset
    check(lib().vsmc_cuda_resample_mn(scheme, M, N, weight_ptr, uniforms_ptr, n_uniforms,
                                      C.byref(rng), rep_ptr, cf_ptr, ws_ptr, ws_bytes,
                                      stream),
          "vsmc_cuda_resample_mn")
    return int(rng.offset - before)


def weight_ess(N, lw_ptr, w_ptr, inc_ptr, use_log, stream=None) -> float:
    """WeightSet::ess(inc, use_log) of device weights (see the C ABI)."""
    v = C.c_double()
    check(lib().vsmc_cuda_weight_ess(N, lw_ptr, w_ptr, inc_ptr, 1 if use_log else 0,
                                     C.byref(v), stream), "vsmc_cuda_weight_ess")
    return v.value


def weight_cess(N, w_ptr, inc_ptr, use_log, stream=None) -> float:
    """WeightSet::cess(inc, use_log) of device weights (see the C ABI)."""
    v = C.c_double()
    check(lib().vsmc_cuda_weight_cess(N, w_ptr, inc_ptr, 1 if use_log else 0,
                                      C.byref(v), stream), "vsmc_cuda_weight_cess")
    return v.value


NOALLOC_MAX_N = 262144


def resample_noalloc(scheme, N, weight_ptr, rng: ThreefryState, rep_ptr, cf_ptr,
                     uniforms_ptr=None, n_uniforms=0, stream=None) -> int:
    """vsmc_cuda_resample on the library's static scratch (no allocation);
    N <= NOALLOC_MAX_N.  Returns the engine words drawn."""
    before = rng.offset
    check(lib().vsmc_cuda_resample_noalloc(scheme, N, weight_ptr, uniforms_ptr, n_uniforms,
                                           C.byref(rng), rep_ptr, cf_ptr, stream),
          "vsmc_cuda_resample_noalloc")
    return int(rng.offset - before)


def copy_f64(N, dim, src_ptr, dst_ptr, cf_ptr, stream=None):
    check(lib().vsmc_cuda_copy_f64(N, dim, src_ptr, dst_ptr, cf_ptr, stream),
          "vsmc_cuda_copy_f64")


def math_eval(fn, n, in_ptr, out_ptr, stream=None) -> None:
    """The library's FP64 log (fn 0) or exp (fn 1) of n device doubles."""
    check(lib().vsmc_cuda_math_eval(fn, n, in_ptr, out_ptr, stream),
          "vsmc_cuda_math_eval")


# -------------------------------------------------------- CV filter -------

def cv_config(**kw) -> CVConfig:
    c = CVConfig()
    lib().vsmc_cuda_cv_config_default(C.byref(c))
    for k, v in kw.items():
        if not hasattr(c, k):
            raise KeyError(k)
        setattr(c, k, v)
    return c


def cv_simulate(T, obs_seed, stream_id=0, want_truth=False, **params):
    """The workload's observation series (host computation, no device)."""
    import numpy as np
    c = cv_config(stream_id=stream_id, **params)
    ox, oy = np.zeros(T), np.zeros(T)
    truth = np.zeros((T, 4))
    check(lib().vsmc_cuda_cv_simulate(C.byref(c), obs_seed, T, ox.ctypes.data,
                                      oy.ctypes.data, truth.ctypes.data),
          "vsmc_cuda_cv_simulate")
    return (ox, oy, truth) if want_truth else (ox, oy)


class CVFilter:
    """The constant-velocity Student-t filter as a device-resident Sampler:
    ``initialize()`` and ``iterate(n)`` mirror vsmc::Sampler (core/sampler.hpp:
    450-483); histories mirror ess_history / resampled_history / Monitor."""

    def __init__(self, N, T_max, scheme=Multinomial, form=FP64, threshold=0.5, seed=101,
                 stream_id=0, stream=None, **params):
        self.cfg = cv_config(N=N, T_max=T_max, scheme=scheme, form=form,
                             threshold=threshold, seed=seed, stream_id=stream_id, **params)
        self.N = N
        self.stream = stream
        h = C.c_void_p()
        check(lib().vsmc_cuda_cv_create(C.byref(self.cfg), stream, C.byref(h)),
              "vsmc_cuda_cv_create")
        self.h = h

    @staticmethod
    def device_bytes(**kw) -> int:
        c = cv_config(**kw)
        return int(lib().vsmc_cuda_cv_device_bytes(C.byref(c)))

    def close(self):
        if getattr(self, "h", None):
            check(lib().vsmc_cuda_cv_destroy(self.h), "vsmc_cuda_cv_destroy")
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_observations(self, ox_ptr, oy_ptr, T, on_device):
        check(lib().vsmc_cuda_cv_set_observations(self.h, ox_ptr, oy_ptr, T,
                                                  1 if on_device else 0),
              "vsmc_cuda_cv_set_observations")

    def set_observations_host(self, ox, oy):
        """numpy float64 arrays; copied before returning."""
        import numpy as np
        self._ox = np.ascontiguousarray(ox, np.float64)
        self._oy = np.ascontiguousarray(oy, np.float64)
        self.set_observations(self._ox.ctypes.data, self._oy.ctypes.data, self._ox.size, False)
        self.synchronize()

    def initialize(self):
        check(lib().vsmc_cuda_cv_initialize(self.h), "vsmc_cuda_cv_initialize")

    def iterate(self, num=1):
        check(lib().vsmc_cuda_cv_iterate(self.h, num), "vsmc_cuda_cv_iterate")

    def synchronize(self):
        check(lib().vsmc_cuda_cv_synchronize(self.h), "vsmc_cuda_cv_synchronize")

    def iter_size(self) -> int:
        n = C.c_uint64()
        check(lib().vsmc_cuda_cv_iter_size(self.h, C.byref(n)), "vsmc_cuda_cv_iter_size")
        return int(n.value)

    def history(self):
        import numpy as np
        T = self.iter_size()
        r = dict(ess=np.zeros(T), resampled=np.zeros(T, np.int32), logz_inc=np.zeros(T),
                 mean_x=np.zeros(T), mean_y=np.zeros(T))
        check(lib().vsmc_cuda_cv_history(self.h, *[_np_ptr(r[k]) for k in
                                                   ("ess", "resampled", "logz_inc",
                                                    "mean_x", "mean_y")]),
              "vsmc_cuda_cv_history")
        return r

    def log_evidence(self) -> float:
        v = C.c_double()
        check(lib().vsmc_cuda_cv_log_evidence(self.h, C.byref(v)), "vsmc_cuda_cv_log_evidence")
        return v.value

    def read_state(self):
        import numpy as np
        s = np.zeros((4, self.N))
        lw = np.zeros(self.N)
        check(lib().vsmc_cuda_cv_read_state(self.h, _np_ptr(s[0]), _np_ptr(s[1]),
                                            _np_ptr(s[2]), _np_ptr(s[3]), _np_ptr(lw)),
              "vsmc_cuda_cv_read_state")
        return s, lw

    def append_observations(self, ox_ptr, oy_ptr, n, on_device=False):
        check(lib().vsmc_cuda_cv_append_observations(self.h, ox_ptr, oy_ptr, n,
                                                     1 if on_device else 0),
              "vsmc_cuda_cv_append_observations")

    def read_step(self, t, ess_ptr=None, logz_ptr=None, res_ptr=None, synchronize=True):
        check(lib().vsmc_cuda_cv_read_step(self.h, t, ess_ptr, logz_ptr, res_ptr,
                                           1 if synchronize else 0),
              "vsmc_cuda_cv_read_step")

    def complete_monitor(self):
        """Asynchronously completes the last step's monitor (see the C ABI)."""
        check(lib().vsmc_cuda_cv_complete_monitor(self.h), "vsmc_cuda_cv_complete_monitor")

    def set_ancestry(self, record_ptr=None, replay_ptr=None, replay_flags_ptr=None):
        check(lib().vsmc_cuda_cv_set_ancestry(self.h, record_ptr, replay_ptr,
                                              replay_flags_ptr),
              "vsmc_cuda_cv_set_ancestry")

    def set_timing(self, enable=True):
        check(lib().vsmc_cuda_cv_set_timing(self.h, 1 if enable else 0),
              "vsmc_cuda_cv_set_timing")

    def timing(self):
        """(move_ms, step_ms, steps, launches) summed since set_timing(True)."""
        mv, st, n, la = C.c_double(), C.c_double(), C.c_uint64(), C.c_uint64()
        check(lib().vsmc_cuda_cv_timing(self.h, C.byref(mv), C.byref(st), C.byref(n),
                                         C.byref(la)), "vsmc_cuda_cv_timing")
        return mv.value, st.value, int(n.value), int(la.value)

    def resample_words(self) -> int:
        v = C.c_uint64()
        check(lib().vsmc_cuda_cv_resample_words(self.h, C.byref(v)),
              "vsmc_cuda_cv_resample_words")
        return int(v.value)

    def copy_from(self):
        import numpy as np
        cf = np.zeros(self.N, np.int32)
        r = C.c_int32()
        check(lib().vsmc_cuda_cv_copy_from(self.h, _np_ptr(cf), C.byref(r)),
              "vsmc_cuda_cv_copy_from")
        return cf, bool(r.value)


class CVBatch:
    """Many constant-velocity filters resident on one device (slots).  The
    scheme, form, threshold and model parameters are shared; N, T_max, seed
    and stream_id are per slot.  ``step(slots)`` advances each listed filter
    by one step in one launch per kernel; ``run(slots)`` steps each until its
    observations are used up."""

    def __init__(self, capacity, scheme=Multinomial, form=FP64, threshold=0.5,
                 hbm_budget=0, stream=None, **params):
        self.model = cv_config(N=2, T_max=1, scheme=scheme, form=form,
                               threshold=threshold, **params)
        self.capacity = capacity
        self.stream = stream
        h = C.c_void_p()
        check(lib().vsmc_cuda_cv_batch_create(C.byref(self.model), capacity, hbm_budget,
                                              stream, C.byref(h)),
              "vsmc_cuda_cv_batch_create")
        self.h = h
        self.N = {}

    def slot_bytes(self, N, T_max) -> int:
        return int(lib().vsmc_cuda_cv_batch_slot_bytes(C.byref(self.model), N, T_max))

    def close(self):
        if getattr(self, "h", None):
            check(lib().vsmc_cuda_cv_batch_destroy(self.h), "vsmc_cuda_cv_batch_destroy")
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @staticmethod
    def _slots(slots):
        import numpy as np
        a = np.ascontiguousarray(np.atleast_1d(np.asarray(slots, dtype=np.uint32)))
        return a, a.size

    def admit(self, N, T_max, seed=101, stream_id=0) -> int:
        s = C.c_uint32()
        check(lib().vsmc_cuda_cv_batch_admit(self.h, N, T_max, seed, stream_id, C.byref(s)),
              "vsmc_cuda_cv_batch_admit")
        self.N[int(s.value)] = N
        return int(s.value)

    def release(self, slot):
        check(lib().vsmc_cuda_cv_batch_release(self.h, slot), "vsmc_cuda_cv_batch_release")
        self.N.pop(slot, None)

    def bytes_in_use(self) -> int:
        v = C.c_uint64()
        check(lib().vsmc_cuda_cv_batch_bytes_in_use(self.h, C.byref(v)),
              "vsmc_cuda_cv_batch_bytes_in_use")
        return int(v.value)

    def set_observations(self, slots, series):
        """series: one (obs_x, obs_y) pair of float64 arrays per slot."""
        import numpy as np
        a, n = self._slots(slots)
        T = np.array([len(x) for x, _ in series], np.uint64)
        ox = np.ascontiguousarray(np.concatenate([x for x, _ in series]), np.float64)
        oy = np.ascontiguousarray(np.concatenate([y for _, y in series]), np.float64)
        check(lib().vsmc_cuda_cv_batch_set_observations(self.h, n, a.ctypes.data, T.ctypes.data,
                                                        ox.ctypes.data, oy.ctypes.data, 0),
              "vsmc_cuda_cv_batch_set_observations")

    def set_observations_packed(self, slots, T, ox_ptr, oy_ptr, on_device):
        import numpy as np
        a, n = self._slots(slots)
        Ta = np.ascontiguousarray(T, np.uint64)
        check(lib().vsmc_cuda_cv_batch_set_observations(self.h, n, a.ctypes.data, Ta.ctypes.data,
                                                        ox_ptr, oy_ptr, 1 if on_device else 0),
              "vsmc_cuda_cv_batch_set_observations")

    def append_observations(self, slots, x, y):
        import numpy as np
        a, n = self._slots(slots)
        xa = np.ascontiguousarray(np.atleast_1d(x), np.float64)
        ya = np.ascontiguousarray(np.atleast_1d(y), np.float64)
        check(lib().vsmc_cuda_cv_batch_append_observations(self.h, n, a.ctypes.data,
                                                           xa.ctypes.data, ya.ctypes.data),
              "vsmc_cuda_cv_batch_append_observations")

    def initialize(self, slots):
        a, n = self._slots(slots)
        check(lib().vsmc_cuda_cv_batch_initialize(self.h, n, a.ctypes.data),
              "vsmc_cuda_cv_batch_initialize")

    def step(self, slots):
        a, n = self._slots(slots)
        check(lib().vsmc_cuda_cv_batch_step(self.h, n, a.ctypes.data), "vsmc_cuda_cv_batch_step")

    def run(self, slots):
        a, n = self._slots(slots)
        check(lib().vsmc_cuda_cv_batch_run(self.h, n, a.ctypes.data), "vsmc_cuda_cv_batch_run")

    def read_last(self, slots):
        """dict of ess, logz_inc, resampled, log_evidence (one entry per slot)."""
        import numpy as np
        a, n = self._slots(slots)
        r = dict(ess=np.zeros(n), logz_inc=np.zeros(n), resampled=np.zeros(n, np.int32),
                 log_evidence=np.zeros(n), status=np.zeros(n, np.int32))
        check(lib().vsmc_cuda_cv_batch_read_last(self.h, n, a.ctypes.data,
                                                 *[_np_ptr(r[k]) for k in
                                                   ("ess", "logz_inc", "resampled",
                                                    "log_evidence", "status")]),
              "vsmc_cuda_cv_batch_read_last")
        return r

    def iter_size(self, slot) -> int:
        v = C.c_uint64()
        check(lib().vsmc_cuda_cv_batch_iter_size(self.h, slot, C.byref(v)),
              "vsmc_cuda_cv_batch_iter_size")
        return int(v.value)

    def history(self, slot):
        import numpy as np
        T = self.iter_size(slot)
        r = dict(ess=np.zeros(T), resampled=np.zeros(T, np.int32), logz_inc=np.zeros(T),
                 mean_x=np.zeros(T), mean_y=np.zeros(T))
        check(lib().vsmc_cuda_cv_batch_history(self.h, slot,
                                               *[_np_ptr(r[k]) for k in
                                                 ("ess", "resampled", "logz_inc",
                                                  "mean_x", "mean_y")]),
              "vsmc_cuda_cv_batch_history")
        return r

    def synchronize(self):
        check(lib().vsmc_cuda_cv_batch_synchronize(self.h), "vsmc_cuda_cv_batch_synchronize")

    def read_steps(self, slots, counts):
        """The last counts[k] steps of each slot, packed in list order:
        dict of ess, logz_inc, resampled (sum(counts)) and status (n)."""
        import numpy as np

        a, n = self._slots(slots)
        c = np.ascontiguousarray(counts, dtype=np.uint32)
        tot = int(c.sum())
        out = {"ess": np.empty(tot), "logz_inc": np.empty(tot),
               "resampled": np.empty(tot, np.int32), "status": np.empty(n, np.int32)}
        rc = lib().vsmc_cuda_cv_batch_read_steps(
            self.h, n, a.ctypes.data, c.ctypes.data, out["ess"].ctypes.data,
            out["logz_inc"].ctypes.data, out["resampled"].ctypes.data,
            out["status"].ctypes.data)
        if rc not in (OK, EDEGENERATE):
            check(rc, "vsmc_cuda_cv_batch_read_steps")
        return out

    def set_launch_shape(self, move_blocks, final_threads):
        check(lib().vsmc_cuda_cv_batch_set_launch_shape(self.h, move_blocks, final_threads),
              "vsmc_cuda_cv_batch_set_launch_shape")

    def set_tiling(self, block_tiles):
        """Filters of at most block_tiles tiles run block-per-filter."""
        check(lib().vsmc_cuda_cv_batch_set_tiling(self.h, block_tiles),
              "vsmc_cuda_cv_batch_set_tiling")

    def tiling(self) -> int:
        v = C.c_int()
        check(lib().vsmc_cuda_cv_batch_tiling(self.h, C.byref(v)), "vsmc_cuda_cv_batch_tiling")
        return v.value

    def autotune(self, slots):
        """Pick the launch shapes by timing a trial copy; returns
        (move CTAs per SM, finalize threads)."""
        a, n = self._slots(slots)
        mv, fin = C.c_int(), C.c_int()
        check(lib().vsmc_cuda_cv_batch_autotune(self.h, n, a.ctypes.data, C.byref(mv),
                                                C.byref(fin)), "vsmc_cuda_cv_batch_autotune")
        return mv.value, fin.value

    def set_graphs(self, enable=True):
        check(lib().vsmc_cuda_cv_batch_set_graphs(self.h, 1 if enable else 0),
              "vsmc_cuda_cv_batch_set_graphs")

    def launches(self) -> int:
        v = C.c_uint64()
        check(lib().vsmc_cuda_cv_batch_launches(self.h, C.byref(v)),
              "vsmc_cuda_cv_batch_launches")
        return int(v.value)


RESULT_DTYPE = [("request", "<u8"), ("t", "<u8"), ("ess", "<f8"), ("logz_inc", "<f8"),
                ("log_evidence", "<f8"), ("resampled", "<i4"), ("status", "<i4"),
                ("submit_ns", "<i8"), ("done_ns", "<i8")]


class CVServer:
    """Persistent request loop (vsmc_cuda_cv_server): open filter requests,
    stream observations, poll one result per observation."""

    def __init__(self, max_filters, scheme=Multinomial, form=FP64, threshold=0.5,
                 hbm_budget=0, **params):
        import numpy as np
        self.model = cv_config(N=2, T_max=1, scheme=scheme, form=form,
                               threshold=threshold, **params)
        h = C.c_void_p()
        check(lib().vsmc_cuda_cv_server_create(C.byref(self.model), max_filters, hbm_budget,
                                               C.byref(h)), "vsmc_cuda_cv_server_create")
        self.h = h
        self._buf = np.zeros(65536, dtype=RESULT_DTYPE)
        assert self._buf.itemsize == C.sizeof(CVResult)

    def close_server(self):
        if getattr(self, "h", None):
            check(lib().vsmc_cuda_cv_server_destroy(self.h), "vsmc_cuda_cv_server_destroy")
            self.h = None

    def __del__(self):
        try:
            self.close_server()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close_server()

    def now_ns(self) -> int:
        return int(lib().vsmc_cuda_cv_server_now_ns(self.h))

    def open(self, N, T_max, seed=101, stream_id=0) -> int:
        r = C.c_uint64()
        check(lib().vsmc_cuda_cv_server_open(self.h, N, T_max, seed, stream_id, C.byref(r)),
              "vsmc_cuda_cv_server_open")
        return int(r.value)

    def observe(self, requests, x, y, submit_ns=None):
        import numpy as np
        r = np.ascontiguousarray(np.atleast_1d(requests), np.uint64)
        xa = np.ascontiguousarray(np.atleast_1d(x), np.float64)
        ya = np.ascontiguousarray(np.atleast_1d(y), np.float64)
        sn = None if submit_ns is None else np.ascontiguousarray(np.atleast_1d(submit_ns),
                                                                  np.int64)
        check(lib().vsmc_cuda_cv_server_observe(self.h, r.size, r.ctypes.data, xa.ctypes.data,
                                                ya.ctypes.data, _np_ptr(sn)),
              "vsmc_cuda_cv_server_observe")

    def close(self, request):
        check(lib().vsmc_cuda_cv_server_close(self.h, request), "vsmc_cuda_cv_server_close")

    def poll(self, wait_ms=0):
        """Results available now (a numpy structured array)."""
        import numpy as np
        n = C.c_uint32()
        check(lib().vsmc_cuda_cv_server_poll(self.h, self._buf.ctypes.data, self._buf.size,
                                             C.byref(n), wait_ms), "vsmc_cuda_cv_server_poll")
        return self._buf[:n.value].copy()

    def drain(self, timeout_ms=60000):
        check(lib().vsmc_cuda_cv_server_drain(self.h, timeout_ms), "vsmc_cuda_cv_server_drain")

    def stats(self) -> dict:
        c = ServerCounters()
        check(lib().vsmc_cuda_cv_server_stats(self.h, C.byref(c)), "vsmc_cuda_cv_server_stats")
        return {k: getattr(c, k) for k, _ in ServerCounters._fields_}


# ------------------------------------------------------------- GMM -------

def gmm_simulate(n=1000, seed=1):
    """The mixture data (host computation, no device)."""
    import numpy as np
    out = np.zeros(n)
    check(lib().vsmc_cuda_gmm_simulate(seed, n, out.ctypes.data), "vsmc_cuda_gmm_simulate")
    return out


class GmmSampler:
    """Tempered SMC sampler for the 1-D Gaussian mixture (vsmc_cuda_gmm):
    ``initialize()`` and ``iterate(n)`` as vsmc::Sampler."""

    def __init__(self, data, N=1 << 16, iters=100, power=4, sweeps=5, sd=0.1,
                 scheme=Systematic, threshold=0.5, seed=101, form=FP64, group=0, stream=None):
        import numpy as np
        c = GmmConfig()
        lib().vsmc_cuda_gmm_config_default(C.byref(c))
        for k, v in dict(N=N, iters=iters, power=power, sweeps=sweeps, sd=sd, scheme=scheme,
                         threshold=threshold, seed=seed, form=form, group=group).items():
            setattr(c, k, v)
        self.cfg = c
        self.N, self.sweeps = N, sweeps
        d = np.ascontiguousarray(data, np.float64)
        h = C.c_void_p()
        check(lib().vsmc_cuda_gmm_create(C.byref(c), d.ctypes.data, d.size, stream, C.byref(h)),
              "vsmc_cuda_gmm_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            check(lib().vsmc_cuda_gmm_destroy(self.h), "vsmc_cuda_gmm_destroy")
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def initialize(self):
        check(lib().vsmc_cuda_gmm_initialize(self.h), "vsmc_cuda_gmm_initialize")

    def iterate(self, num=1):
        check(lib().vsmc_cuda_gmm_iterate(self.h, num), "vsmc_cuda_gmm_iterate")

    def iter_size(self) -> int:
        v = C.c_uint64()
        check(lib().vsmc_cuda_gmm_iter_size(self.h, C.byref(v)), "vsmc_cuda_gmm_iter_size")
        return int(v.value)

    def history(self):
        import numpy as np
        T = self.iter_size()
        r = dict(ess=np.zeros(T), resampled=np.zeros(T, np.int32), zinc=np.zeros(T),
                 integrand=np.zeros(T), grid=np.zeros(T),
                 accept=np.zeros((T, 1 + 3 * self.sweeps), np.int64))
        check(lib().vsmc_cuda_gmm_history(self.h, *[_np_ptr(r[k]) for k in
                                                    ("ess", "resampled", "zinc", "integrand",
                                                     "grid", "accept")]),
              "vsmc_cuda_gmm_history")
        return r

    def log_evidence(self):
        """(SMC estimate, path-sampling estimate)."""
        a, b = C.c_double(), C.c_double()
        check(lib().vsmc_cuda_gmm_log_evidence(self.h, C.byref(a), C.byref(b)),
              "vsmc_cuda_gmm_log_evidence")
        return a.value, b.value

    def read_params(self):
        import numpy as np
        p = np.zeros((self.N, 14))
        lw = np.zeros(self.N)
        w = np.zeros(self.N, np.uint64)
        check(lib().vsmc_cuda_gmm_read_params(self.h, p.ctypes.data, lw.ctypes.data,
                                              w.ctypes.data), "vsmc_cuda_gmm_read_params")
        return p, lw, w

    def loglik(self, form):
        import numpy as np
        out = np.zeros(self.N)
        check(lib().vsmc_cuda_gmm_loglik(self.h, form, out.ctypes.data), "vsmc_cuda_gmm_loglik")
        return out

    def group(self) -> int:
        v = C.c_int()
        check(lib().vsmc_cuda_gmm_group(self.h, C.byref(v)), "vsmc_cuda_gmm_group")
        return v.value

    def set_timing(self, enable=True):
        check(lib().vsmc_cuda_gmm_set_timing(self.h, 1 if enable else 0),
              "vsmc_cuda_gmm_set_timing")

    def timing(self):
        """(mcmc_ms, steps, launches)."""
        a, b, c = C.c_double(), C.c_uint64(), C.c_uint64()
        check(lib().vsmc_cuda_gmm_timing(self.h, C.byref(a), C.byref(b), C.byref(c)),
              "vsmc_cuda_gmm_timing")
        return a.value, int(b.value), int(c.value)
