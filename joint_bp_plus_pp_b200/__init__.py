"""joint_bp_plus_pp_b200 -- B200-native joint X/Z BP + post-processing Monte-Carlo decoder.

Python mirror of the C ABI in include/jbp_b200.h (ctypes).  The decoding runs in the
in-tree CUDA library lib/libjbp_b200.so; importing this package never falls back to a
CPU implementation: if the library is missing, Decoder() raises.

    from joint_bp_plus_pp_b200 import Decoder, Options
    dec = Decoder.from_params()                       # the shipped [[9216,4612]] code
    stats, per_trial = dec.simulate(seed=106, ntrials=10000, p=0.04,
                                    opts=Options(precision="fp32", max_iter=1000, enable_pp=False))
"""
import ctypes
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "lib" / "libjbp_b200.so"
DATA_DIR = PKG / "data"
DEFAULT_PARAMS = DATA_DIR / "H_P768_J3_L12_dmax3_nc0-3_1-2_seed11579811919164041.txt"

PREC = {"fp64": 0, "fp32": 1, "fp16": 2}
SAMPLER = {"philox": 0, "mt19937": 1}
ENGINE = {"auto": 0, "resident": 1, "slots": 2, "table": 3}
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "I/O error", 4: "unsupported", 5: "timeout", 6: "aborted"}


class JbpError(RuntimeError):
    """A failed call: `code` is the JBP_ERR_* status; for JBP_ERR_TIMEOUT (5) and JBP_ERR_ABORTED
    (6), `stats` holds the counters of the trials that finished before the run stopped (None
    otherwise)."""

    def __init__(self, code, msg, stats=None):
        super().__init__(f"jbp error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code
        self.stats = stats


class COptions(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("max_iter", ctypes.c_int), ("damping", ctypes.c_double),
                ("flip_hist", ctypes.c_int), ("enable_pp", ctypes.c_int), ("freeze_syn", ctypes.c_int),
                ("check_warmup", ctypes.c_int), ("check_interval", ctypes.c_int), ("slots", ctypes.c_int),
                ("iters_per_launch", ctypes.c_int), ("watchdog_ms", ctypes.c_int), ("profile", ctypes.c_int),
                ("use_prior", ctypes.c_int), ("prior", ctypes.c_double * 4), ("engine", ctypes.c_int),
                ("p_max", ctypes.c_double), ("learned_from", ctypes.c_int), ("learned_order", ctypes.c_int),
                ("learned_cols", ctypes.c_int), ("collect_every", ctypes.c_int)]


TRIAL_DTYPE = np.dtype([("iterations", np.int32), ("syndrome_ok", np.uint8), ("bp_ok", np.uint8),
                        ("success", np.uint8), ("exact", np.uint8), ("stab_equiv", np.uint8),
                        ("pp_success", np.uint8), ("pp_ets", np.uint8), ("pp_flip", np.uint8),
                        ("pp_osd", np.uint8), ("ets_used_flags", np.uint8), ("pp_in_decode", np.uint8),
                        ("reserved", np.uint8)])
assert TRIAL_DTYPE.itemsize == 16

STAT_FIELDS = ["trials", "failures", "bp_fail", "pp_success", "flip_pp_success", "osd_pp_success", "stab_success",
               "ets_used", "ets_saved", "ets6_used", "ets6_saved", "ets12_used", "ets12_saved", "exact",
               "total_iters"]


class CStats(ctypes.Structure):
    _fields_ = [(f, ctypes.c_longlong) for f in STAT_FIELDS] + [("device_ms", ctypes.c_double),
                                                                ("kernel_launches", ctypes.c_longlong),
                                                                ("bp_trial_iterations", ctypes.c_longlong),
                                                                ("check_ms", ctypes.c_double),
                                                                ("var_ms", ctypes.c_double),
                                                                ("profiled_iterations", ctypes.c_longlong),
                                                                ("slots", ctypes.c_longlong),
                                                                ("learned_attempts", ctypes.c_longlong),
                                                                ("learned_success", ctypes.c_longlong),
                                                                ("test_ms", ctypes.c_double),
                                                                ("syndrome_tests", ctypes.c_longlong)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


@dataclass
class Options:
    """Decoder options with the reference CLI defaults (jointbp_ets.cpp:4841-4866)."""
    precision: str = "fp64"
    max_iter: int = 50
    damping: float = 0.0
    flip_hist: int = 5
    enable_pp: bool = True
    freeze_syn: bool = False
    check_warmup: int = 0
    check_interval: int = 1
    slots: int = 0
    iters_per_launch: int = 0
    watchdog_ms: int = 0
    profile: bool = False
    prior: tuple = None    # (I, X, Z, Y) probabilities used as given instead of those of p
    engine: str = "auto"   # "auto", "resident" (shared-memory trial-resident tier) or "slots"
    learned_from: int = 0  # > 0: stalled trials try the learned flip proposal from this iteration
    p_max: float = 0.0     # > p: per-trial error rate uniform in [p, p_max) (simulate)
    learned_order: str = "model"   # "model": the network's scores; "llr": |LLR| order (the baseline)
    learned_cols: int = 0  # qubits the proposal's elimination may use, in that order (0 = 512)
    collect_every: int = 0  # stall-state collection: 1 in this many quiet, correct qubits (0 = 32)

    def to_c(self):
        pr = (ctypes.c_double * 4)(*(self.prior or (0.0, 0.0, 0.0, 0.0)))
        return COptions(PREC[self.precision], self.max_iter, self.damping, self.flip_hist, int(self.enable_pp),
                        int(self.freeze_syn), self.check_warmup, self.check_interval, self.slots,
                        self.iters_per_launch, self.watchdog_ms, int(self.profile), int(self.prior is not None), pr,
                        ENGINE[self.engine], float(self.p_max), int(self.learned_from),
                        {"model": 0, "llr": 1}[self.learned_order], int(self.learned_cols),
                        int(self.collect_every))


_lib = None


def load_library(path=None):
    """Loads lib/libjbp_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(f"{p} not built: run `python -m joint_bp_plus_pp_b200.build`")
    lib = ctypes.CDLL(str(p))
    vp, i, ll, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double
    lib.jbp_last_error.restype = ctypes.c_char_p
    lib.jbp_version.restype = ctypes.c_char_p
    lib.jbp_create_from_params.argtypes = [ctypes.c_char_p, ctypes.c_char_p, i, ctypes.POINTER(vp)]
    lib.jbp_create_from_checks.argtypes = [i, i, vp, vp, i, vp, vp, i, ctypes.POINTER(vp)]
    lib.jbp_add_ets_group.argtypes = [vp, i, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p]
    lib.jbp_destroy.argtypes = [vp]
    lib.jbp_destroy.restype = None
    lib.jbp_code_info.argtypes = [vp] + [ctypes.POINTER(i)] * 6
    lib.jbp_code_checks.argtypes = [vp, i, vp, vp]
    lib.jbp_simulate.argtypes = [vp, ctypes.POINTER(COptions), ctypes.c_uint64, ll, ll, d, i, ctypes.POINTER(CStats),
                                 vp, vp]
    lib.jbp_decode_errors.argtypes = [vp, ctypes.POINTER(COptions), ll, vp, d, vp, vp, ctypes.POINTER(CStats)]
    lib.jbp_decode_syndromes.argtypes = [vp, ctypes.POINTER(COptions), ll, vp, vp, d, vp, vp, ctypes.POINTER(CStats)]
    lib.jbp_decode_errors_llr.argtypes = [vp, ctypes.POINTER(COptions), ll, vp, d, vp, vp, ctypes.POINTER(CStats)]
    lib.jbp_autotune.argtypes = [vp, ctypes.POINTER(COptions), d, ll, ctypes.POINTER(COptions), ctypes.POINTER(d)]
    lib.jbp_code_graph_checks.argtypes = [vp, ctypes.POINTER(ll), ctypes.POINTER(i), ctypes.POINTER(i)]
    lib.jbp_graph_checks.argtypes = [i, i, vp, vp, i, vp, vp, ctypes.POINTER(ll), ctypes.POINTER(i), ctypes.POINTER(i)]
    lib.jbp_measure_sfu.argtypes = [i, ctypes.POINTER(d), ctypes.POINTER(d), ctypes.POINTER(d)]
    lib.jbp_check_reciprocal.argtypes = [i, ctypes.c_ulonglong, ll, ctypes.POINTER(ll), ctypes.POINTER(ll)]
    lib.jbp_debug_fail_allocation.argtypes = [ll]
    lib.jbp_request_abort.argtypes = [vp]
    lib.jbp_check_us_oscillation.argtypes = [i, ctypes.c_ulonglong, ll, ctypes.POINTER(ll), ctypes.POINTER(ll)]
    lib.jbp_simulate_mixed.argtypes = [vp, i, ctypes.POINTER(COptions), vp, vp, vp, d, ctypes.POINTER(CStats), vp]
    lib.jbp_decode_errors_device.argtypes = [vp, ctypes.POINTER(COptions), ll, vp, d, vp, vp, ctypes.POINTER(CStats),
                                             vp]
    lib.jbp_sample_errors.argtypes = [vp, ctypes.c_uint64, ll, ll, d, i, vp]
    lib.jbp_sample_reference_errors.argtypes = [i, ctypes.c_uint64, ll, ll, d, vp, i]
    lib.jbp_default_options.argtypes = [ctypes.POINTER(COptions)]
    lib.jbp_default_options.restype = None
    fp = ctypes.c_float
    lib.jbp_mlp_param_count.restype = i
    lib.jbp_mlp_grad.argtypes = [vp, vp, ll, vp, vp, fp, vp, ctypes.POINTER(d)]
    lib.jbp_mlp_train.argtypes = [vp, vp, ll, vp, vp, i, i, fp, fp, ctypes.c_uint64, vp]
    lib.jbp_mlp_infer.argtypes = [vp, vp, ll, vp, vp]
    lib.jbp_set_flip_model.argtypes = [vp, vp]
    lib.jbp_collect_stall_states.argtypes = [vp, ctypes.POINTER(COptions), ctypes.c_uint64, ll, ll, d, i, ll, vp, vp,
                                             ctypes.POINTER(ll), ctypes.POINTER(CStats)]
    if path is None:
        _lib = lib
    return lib


def _check(lib, rc, stats=None):
    if rc != 0:
        raise JbpError(rc, lib.jbp_last_error().decode(errors="replace"),
                       stats.as_dict() if (rc in (5, 6) and stats is not None) else None)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def sample_reference_errors(n, seed, first_trial, ntrials, p, threads=0):
    """Errors of the reference stream (mt19937_64 per trial) sampled on the host."""
    lib = load_library()
    err = np.empty((ntrials, n), np.uint8)
    _check(lib, lib.jbp_sample_reference_errors(n, seed, first_trial, ntrials, p, _ptr(err), threads))
    return err


class Decoder:
    """One code on one GPU (the C context jbp_ctx)."""

    def __init__(self, handle, lib):
        self._h = handle
        self._lib = lib
        n, mx, mz, rx, rz, ng = (ctypes.c_int() for _ in range(6))
        _check(lib, lib.jbp_code_info(handle, *(ctypes.byref(v) for v in (n, mx, mz, rx, rz, ng))))
        self.n, self.mx, self.mz = n.value, mx.value, mz.value
        self.rank_x, self.rank_z, self.ets_groups = rx.value, rz.value, ng.value

    @classmethod
    def from_params(cls, params=DEFAULT_PARAMS, ets_dir="default", device=0):
        lib = load_library()
        if ets_dir == "default":
            ets_dir = str(Path(params).with_suffix(""))
        h = ctypes.c_void_p()
        _check(lib, lib.jbp_create_from_params(str(params).encode(), ets_dir.encode() if ets_dir else None, device,
                                               ctypes.byref(h)))
        return cls(h, lib)

    @classmethod
    def from_checks(cls, n, x_off, x_var, z_off, z_var, device=0):
        lib = load_library()
        arrs = [np.ascontiguousarray(a, np.int32) for a in (x_off, x_var, z_off, z_var)]
        h = ctypes.c_void_p()
        _check(lib, lib.jbp_create_from_checks(n, len(arrs[0]) - 1, _ptr(arrs[0]), _ptr(arrs[1]), len(arrs[2]) - 1,
                                               _ptr(arrs[2]), _ptr(arrs[3]), device, ctypes.byref(h)))
        return cls(h, lib)

    def close(self):
        if self._h:
            self._lib.jbp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def checks(self, side):
        m = self.mx if side == 0 else self.mz
        off = np.zeros(m + 1, np.int32)
        _check(self._lib, self._lib.jbp_code_checks(self._h, side, _ptr(off), None))
        var = np.zeros(int(off[-1]), np.int32)
        _check(self._lib, self._lib.jbp_code_checks(self._h, side, None, _ptr(var)))
        return off, var

    def simulate(self, seed, ntrials, p, opts=None, first_trial=1, sampler="philox", per_trial=True, hist=False):
        opts = opts or Options()
        st = CStats()
        res = np.zeros(ntrials, TRIAL_DTYPE) if per_trial else None
        h = np.zeros(opts.max_iter + 1, np.int64) if hist else None
        co = opts.to_c()
        _check(self._lib, self._lib.jbp_simulate(self._h, ctypes.byref(co), seed, first_trial, ntrials, p,
                                                 SAMPLER[sampler], ctypes.byref(st), _ptr(res), _ptr(h)), st)
        out = st.as_dict()
        if hist:
            out["hist"] = h
        return out, res

    def sample_errors(self, seed, first_trial, ntrials, p, sampler="philox"):
        """Errors drawn by a device sampler (the streams simulate() decodes)."""
        err = np.zeros((ntrials, self.n), np.uint8)
        _check(self._lib, self._lib.jbp_sample_errors(self._h, seed, first_trial, ntrials, p, SAMPLER[sampler],
                                                      _ptr(err)))
        return err

    def decode_errors(self, err, p, opts=None, want_est=True):
        err = np.ascontiguousarray(err, np.uint8).reshape(-1, self.n)
        opts = opts or Options()
        t = err.shape[0]
        est = np.zeros((t, self.n), np.uint8) if want_est else None
        res = np.zeros(t, TRIAL_DTYPE)
        st = CStats()
        co = opts.to_c()
        _check(self._lib, self._lib.jbp_decode_errors(self._h, ctypes.byref(co), t, _ptr(err), p, _ptr(est),
                                                      _ptr(res), ctypes.byref(st)), st)
        return st.as_dict(), res, est

    def autotune(self, p, opts=None, probe_trials=16384):
        """Fastest launch configuration (engine, slots, iterations per graph) for these options:
        returns (Options, trials/s of the probe)."""
        opts = opts or Options()
        co = opts.to_c()
        best = COptions()
        rate = ctypes.c_double()
        _check(self._lib, self._lib.jbp_autotune(self._h, ctypes.byref(co), p, probe_trials, ctypes.byref(best),
                                                 ctypes.byref(rate)))
        inv = {v: k for k, v in ENGINE.items()}
        from dataclasses import replace
        return replace(opts, engine=inv[best.engine], slots=best.slots, iters_per_launch=best.iters_per_launch,
                       check_interval=best.check_interval), rate.value

    def decode_errors_llr(self, err, p, opts=None):
        """decode_errors plus the final LLRs (trials x n x 2: x bit, z bit; natural log of
        P(1)/P(0)) -- those of the last variable update when opts.check_warmup >= max_iter."""
        err = np.ascontiguousarray(err, np.uint8).reshape(-1, self.n)
        opts = opts or Options()
        t = err.shape[0]
        llr = np.zeros((t, self.n, 2), np.float32)
        res = np.zeros(t, TRIAL_DTYPE)
        st = CStats()
        co = opts.to_c()
        _check(self._lib, self._lib.jbp_decode_errors_llr(self._h, ctypes.byref(co), t, _ptr(err), p, _ptr(llr),
                                                          _ptr(res), ctypes.byref(st)))
        return st.as_dict(), res, llr

    def decode_syndromes(self, sx, sz, p, opts=None, want_est=True):
        sx = np.ascontiguousarray(sx, np.uint8).reshape(-1, self.mx)
        sz = np.ascontiguousarray(sz, np.uint8).reshape(-1, self.mz)
        opts = opts or Options()
        t = sx.shape[0]
        est = np.zeros((t, self.n), np.uint8) if want_est else None
        res = np.zeros(t, TRIAL_DTYPE)
        st = CStats()
        co = opts.to_c()
        _check(self._lib, self._lib.jbp_decode_syndromes(self._h, ctypes.byref(co), t, _ptr(sx), _ptr(sz), p,
                                                         _ptr(est), _ptr(res), ctypes.byref(st)), st)
        return st.as_dict(), res, est

    def decode_errors_device(self, d_err_ptr, ntrials, p, d_est_ptr, d_res_ptr, opts=None, stream=0):
        """Device-resident decode: pointers are device addresses (ints), ordered on `stream`."""
        opts = opts or Options()
        st = CStats()
        co = opts.to_c()
        _check(self._lib, self._lib.jbp_decode_errors_device(self._h, ctypes.byref(co), ntrials,
                                                             ctypes.c_void_p(d_err_ptr), p,
                                                             ctypes.c_void_p(d_est_ptr) if d_est_ptr else None,
                                                             ctypes.c_void_p(d_res_ptr), ctypes.byref(st),
                                                             ctypes.c_void_p(stream)))
        return st.as_dict()


    # ------------------------------------------------------------ learned flip proposal

    def request_abort(self):
        """Stops the run in progress on this decoder (call from another thread), or the next run:
        it raises JbpError with code 6 and the counters of the trials that finished."""
        _check(self._lib, self._lib.jbp_request_abort(self._h))

    def set_flip_model(self, params):
        """Model used when Options.learned_from > 0 (None removes it)."""
        if params is None:
            _check(self._lib, self._lib.jbp_set_flip_model(self._h, None))
            return
        prm = np.ascontiguousarray(params, np.float32)
        if prm.size != MLP_PARAMS:
            raise ValueError(f"flip model has {prm.size} parameters, this library's network takes {MLP_PARAMS}")
        _check(self._lib, self._lib.jbp_set_flip_model(self._h, _ptr(prm)))

    def mlp_grad(self, params, x, y, pos_weight=1.0):
        """GPU gradient and mean loss of the flip-proposal MLP on samples (x: n x MLP_IN, y: n x 2)."""
        prm = np.ascontiguousarray(params, np.float32)
        x = np.ascontiguousarray(x, np.float32)
        if x.ndim != 2 or x.shape[1] != MLP_IN:
            raise ValueError(f"features must be n x {MLP_IN}")
        y = np.ascontiguousarray(y, np.float32)
        g = np.zeros(MLP_PARAMS, np.float32)
        loss = ctypes.c_double()
        _check(self._lib, self._lib.jbp_mlp_grad(self._h, _ptr(prm), len(x), _ptr(x), _ptr(y), pos_weight, _ptr(g),
                                                 ctypes.byref(loss)))
        return g, loss.value

    def mlp_train(self, params, x, y, epochs=10, batch=4096, lr=1e-3, pos_weight=1.0, seed=1):
        """Adam training on the GPU; returns (params, per-epoch mean loss)."""
        prm = np.array(params, np.float32)
        x = np.ascontiguousarray(x, np.float32)
        if x.ndim != 2 or x.shape[1] != MLP_IN:
            raise ValueError(f"features must be n x {MLP_IN}")
        y = np.ascontiguousarray(y, np.float32)
        hist = np.zeros(max(1, epochs), np.float64)
        _check(self._lib, self._lib.jbp_mlp_train(self._h, _ptr(prm), len(x), _ptr(x), _ptr(y), epochs, batch, lr,
                                                  pos_weight, seed, _ptr(hist)))
        return prm, hist[:epochs]

    def mlp_infer(self, params, x):
        """BF16 tensor-core inference (the decoder's fused kernel code): logits n x 2."""
        prm = np.ascontiguousarray(params, np.float32)
        x = np.ascontiguousarray(x, np.float32)
        if x.ndim != 2 or x.shape[1] != MLP_IN:
            raise ValueError(f"features must be n x {MLP_IN}")
        out = np.zeros((len(x), 2), np.float32)
        _check(self._lib, self._lib.jbp_mlp_infer(self._h, _ptr(prm), len(x), _ptr(x), _ptr(out)))
        return out

    def collect_stall_states(self, seed, ntrials, p, opts, capacity, first_trial=1, sampler="philox"):
        """Features and labels of the qubits of stalled BP states (training data)."""
        x = np.zeros((capacity, MLP_IN), np.float32)
        y = np.zeros((capacity, 2), np.float32)
        cnt = ctypes.c_longlong()
        st = CStats()
        co = opts.to_c()
        _check(self._lib, self._lib.jbp_collect_stall_states(self._h, ctypes.byref(co), seed, first_trial, ntrials, p,
                                                             SAMPLER[sampler], capacity, _ptr(x), _ptr(y),
                                                             ctypes.byref(cnt), ctypes.byref(st)))
        return x[:cnt.value], y[:cnt.value], st.as_dict()


def measure_sfu(device=0):
    """Measured special-function throughput of a GPU, G results/s: {"ex2", "lg2", "rcp"}."""
    lib = load_library()
    r = [ctypes.c_double() for _ in range(3)]
    _check(lib, lib.jbp_measure_sfu(device, *[ctypes.byref(x) for x in r]))
    return {"ex2": r[0].value, "lg2": r[1].value, "rcp": r[2].value}


def debug_fail_allocation(after):
    """Test hook: the allocation `after` allocations from now (0 = the next) fails once with
    JbpError; after < 0 turns the hook off."""
    lib = load_library()
    _check(lib, lib.jbp_debug_fail_allocation(int(after)))


def check_us_oscillation(n, seed=1, device=0):
    """Device self-check of the two forms of the us-signal oscillation test against the rule as
    the reference states it: (mismatches, histories the rule accepts)."""
    lib = load_library()
    bad, fired = ctypes.c_longlong(), ctypes.c_longlong()
    _check(lib, lib.jbp_check_us_oscillation(device, seed, n, ctypes.byref(bad), ctypes.byref(fired)))
    return bad.value, fired.value


def check_reciprocal(n, seed=1, device=0):
    """Device self-check of the FP64 kernels' branch-free reciprocal against correctly rounded
    division on n divisors: (mismatches, index of the first or -1)."""
    lib = load_library()
    bad, first = ctypes.c_longlong(), ctypes.c_longlong()
    _check(lib, lib.jbp_check_reciprocal(device, seed, n, ctypes.byref(bad), ctypes.byref(first)))
    return bad.value, first.value


def graph_checks(n, x_off, x_var, z_off, z_var):
    """Start-up graph checks of a CSS code given as check lists, on the host (no GPU):
    {"odd_pairs": X/Z check pairs with an odd overlap (0 = orthogonal), "girth_x", "girth_z"}."""
    lib = load_library()
    arr = [np.ascontiguousarray(a, np.int32) for a in (x_off, x_var, z_off, z_var)]
    odd, gx, gz = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int()
    _check(lib, lib.jbp_graph_checks(n, len(arr[0]) - 1, _ptr(arr[0]), _ptr(arr[1]), len(arr[2]) - 1, _ptr(arr[2]),
                                     _ptr(arr[3]), ctypes.byref(odd), ctypes.byref(gx), ctypes.byref(gz)))
    return {"odd_pairs": odd.value, "girth_x": gx.value, "girth_z": gz.value}


def simulate_mixed(decoders, ntrials, p, opts=None, seeds=None, first_trial=None, per_trial=False):
    """Mixed-size Monte Carlo in one kernel launch over the codes of several decoders on one
    device (jbp_simulate_mixed): code i decodes ntrials[i] Philox trials of seeds[i] from
    first_trial[i].  Plain BP in FP32 (opts.precision "fp32", or "fp16" message storage).
    Returns (list of stats, list of per-trial records or None)."""
    k = len(decoders)
    lib = decoders[0]._lib
    opts = opts or Options(precision="fp32", enable_pp=False)
    ntrials = [int(t) for t in (ntrials if hasattr(ntrials, "__len__") else [ntrials] * k)]
    seeds = np.asarray(seeds if seeds is not None else [11 + i for i in range(k)], np.uint64)
    first = np.asarray(first_trial if first_trial is not None else [1] * k, np.int64)
    ntr = np.asarray(ntrials, np.int64)
    if len(seeds) != k or len(first) != k or len(ntr) != k:
        raise ValueError("one seed, first trial and trial count per decoder")
    ctxs = (ctypes.c_void_p * k)(*[d._h for d in decoders])
    stats = (CStats * k)()
    res = [np.zeros(t, TRIAL_DTYPE) for t in ntrials] if per_trial else None
    ptrs = (ctypes.c_void_p * k)(*[r.ctypes.data for r in res]) if per_trial else None
    co = opts.to_c()
    _check(lib, lib.jbp_simulate_mixed(ctxs, k, ctypes.byref(co), _ptr(seeds), _ptr(first), _ptr(ntr), p, stats,
                                       ptrs))
    return [s.as_dict() for s in stats], res


MLP_IN = 8        # features per qubit of the flip-proposal MLP (include/jbp_b200.h)
MLP_PARAMS = 4866
FLIP_MODEL_PATH = DATA_DIR / "flip_mlp_params.npy"


def mlp_init(seed=0):
    """He-initialised parameters of the flip-proposal MLP (W1, b1, W2, b2, W3, b3)."""
    rng = np.random.default_rng(seed)
    w1 = rng.normal(0, (2 / MLP_IN) ** 0.5, (64, MLP_IN))
    w2 = rng.normal(0, (2 / 64) ** 0.5, (64, 64))
    w3 = rng.normal(0, (1 / 64) ** 0.5, (2, 64))
    return np.concatenate([w1.ravel(), np.zeros(64), w2.ravel(), np.zeros(64), w3.ravel(), np.full(2, -3.0)]).astype(
        np.float32)


def load_flip_model(path=FLIP_MODEL_PATH):
    """The trained flip-proposal parameters shipped with the package (None if absent)."""
    p = Path(path)
    return np.load(p).astype(np.float32) if p.exists() else None


def paired_ler_difference(fail_a, fail_b, z=1.96):
    """LER(a) - LER(b) on the same trials with its 95% interval (paired Wald interval from the
    discordant trials: d = (n10 - n01) / n, var = (n10 + n01 - (n10 - n01)^2 / n) / n^2).
    fail_a, fail_b: boolean arrays of per-trial failures.  Returns (d, lo, hi, n10, n01)."""
    a = np.asarray(fail_a, bool)
    b = np.asarray(fail_b, bool)
    n = a.size
    if n == 0 or b.size != n:
        raise ValueError("two failure arrays of the same nonzero length")
    n10 = int((a & ~b).sum())
    n01 = int((~a & b).sum())
    d = (n10 - n01) / n
    half = z * max(0.0, n10 + n01 - (n10 - n01) ** 2 / n) ** 0.5 / n
    return d, d - half, d + half, n10, n01


def wilson_interval(n, k, z=1.96):
    """Wilson score interval (jointbp_ets.cpp:4388-4399)."""
    if n <= 0:
        return None
    ph = k / n
    z2 = z * z
    den = 1.0 + z2 / n
    center = (ph + z2 / (2.0 * n)) / den
    half = z * ((ph * (1.0 - ph) + z2 / (4.0 * n)) / n) ** 0.5 / den
    return max(0.0, center - half), min(1.0, center + half)
