"""ctypes bindings to the CPU oracle (test infrastructure only).

* ``Oracle``    -- oracle/_ref/libjbp_oracle.so, this project's C restatement of the
                   reference decoder (oracle/jbp_oracle.c).
* ``Reference`` -- oracle/_ref/libjbp_ref.so, a harness over the unmodified reference
                   source (oracle/ref_harness.cpp); present only where the reference
                   sources could be compiled.

Nothing in the product imports this module.
"""
import ctypes
import os
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
REF_DIR = ROOT / "oracle" / "_ref"
DATA_DIR = ROOT / "joint_bp_plus_pp_b200" / "data"
PARAMS = DATA_DIR / "H_P768_J3_L12_dmax3_nc0-3_1-2_seed11579811919164041.txt"
ETS_DIR = DATA_DIR / "H_P768_J3_L12_dmax3_nc0-3_1-2_seed11579811919164041"

REC_FIELDS = ("iterations bp_ok syndrome_ok success exact stab_equiv pp_in_decode pp_in_ets pp_in_flip "
              "ets_pp_ok flip_pp_ok osd_pp_ok used_any used6 used12 ets_applied_post pp_success_this "
              "osd_success").split()


class TrialRecord(ctypes.Structure):
    _fields_ = [("trial_idx", ctypes.c_longlong)] + [(n, ctypes.c_int) for n in REC_FIELDS]

    def as_dict(self):
        d = {"trial_idx": self.trial_idx}
        d.update({n: getattr(self, n) for n in REC_FIELDS})
        return d


class _Code(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("m", ctypes.c_int * 2), ("e", ctypes.c_int * 2), ("P", ctypes.c_int),
                ("chk_off", ctypes.c_void_p * 2), ("chk_var", ctypes.c_void_p * 2),
                ("var_off", ctypes.c_void_p * 2), ("var_edge", ctypes.c_void_p * 2)]


class _Result(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("iterations syndrome_ok bp_ok pp_success pp_success_ets "
                                            "pp_success_flip pp_used_ets_any pp_used_ets6 pp_used_ets12").split()] + \
               [("ets_label_mask", ctypes.c_uint)]


class _Basis(ctypes.Structure):
    _fields_ = [("words", ctypes.c_int), ("rank", ctypes.c_int), ("rows", ctypes.c_void_p),
                ("pivot", ctypes.c_void_p), ("order", ctypes.c_void_p)]


_ETS_SET_BYTES = 1 << 16  # opaque jbo_ets_set storage (struct is ~2 KB)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _u64(x):
    return ctypes.c_ulonglong(int(x) & 0xFFFFFFFFFFFFFFFF)


class Oracle:
    """This project's C restatement of the reference decoder."""

    def __init__(self, params=PARAMS, ets_dir=ETS_DIR, load_ets=True):
        path = REF_DIR / "libjbp_oracle.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run `make -C oracle oracle`")
        self.lib = lib = ctypes.CDLL(str(path))
        lib.jbo_work_new.restype = ctypes.c_void_p
        lib.jbo_work_new.argtypes = [ctypes.c_void_p]
        lib.jbo_trial_seed.restype = ctypes.c_ulonglong
        lib.jbo_trial_seed.argtypes = [ctypes.c_ulonglong, ctypes.c_ulonglong]
        lib.jbo_sample.argtypes = [ctypes.c_ulonglong, ctypes.c_longlong, ctypes.c_double, ctypes.c_int, ctypes.c_void_p]
        lib.jbo_decode.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                           ctypes.c_double, ctypes.c_int] + [ctypes.c_void_p] * 4
        lib.jbo_simulate_trial.argtypes = [ctypes.c_void_p] * 5 + [ctypes.c_ulonglong, ctypes.c_longlong,
                                                                   ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                                                   ctypes.c_double, ctypes.c_int, ctypes.c_int] + \
            [ctypes.c_void_p] * 3
        lib.jbo_wilson.argtypes = [ctypes.c_longlong, ctypes.c_longlong, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p]
        lib.jbo_error_trial.argtypes = [ctypes.c_void_p] * 6 + [ctypes.c_longlong, ctypes.c_double, ctypes.c_int,
                                                               ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                                               ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        self.code = _Code()
        if params is not None:
            rc = lib.jbo_code_from_params(str(params).encode(), ctypes.byref(self.code))
            if rc:
                raise RuntimeError(f"jbo_code_from_params failed: {rc}")
            self._post_code(load_ets, ets_dir)

    @classmethod
    def from_checks(cls, n, xoff, xvar, zoff, zvar):
        o = cls(params=None)
        xoff, xvar, zoff, zvar = (np.ascontiguousarray(a, np.int32) for a in (xoff, xvar, zoff, zvar))
        rc = o.lib.jbo_code_from_checks(n, len(xoff) - 1, _ptr(xoff), _ptr(xvar), len(zoff) - 1, _ptr(zoff),
                                        _ptr(zvar), ctypes.byref(o.code))
        if rc:
            raise RuntimeError("jbo_code_from_checks failed")
        o._post_code(False, None)
        return o

    def _post_code(self, load_ets, ets_dir):
        lib = self.lib
        self.n = self.code.n
        self.m = (self.code.m[0], self.code.m[1])
        self.work = lib.jbo_work_new(ctypes.byref(self.code))
        self.ets = ctypes.create_string_buffer(_ETS_SET_BYTES)
        if load_ets and ets_dir is not None:
            lib.jbo_ets_set_load_dir(str(ets_dir).encode(), self.code.P, self.ets)
        self.bx, self.bz = _Basis(), _Basis()
        lib.jbo_basis_build(ctypes.byref(self.code), 0, ctypes.byref(self.bx))
        lib.jbo_basis_build(ctypes.byref(self.code), 1, ctypes.byref(self.bz))

    def checks(self, side):
        m, e = self.code.m[side], self.code.e[side]
        off = np.ctypeslib.as_array((ctypes.c_int * (m + 1)).from_address(self.code.chk_off[side])).copy()
        var = np.ctypeslib.as_array((ctypes.c_int * e).from_address(self.code.chk_var[side])).copy()
        return off, var

    def ets_groups(self):
        """[(label, size, count_x, count_z)] in load order."""
        out = []
        ng = self.lib.jbo_ets_info(self.ets, -1, None, None, None, None)
        for g in range(ng):
            size, cx, cz = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
            label = ctypes.create_string_buffer(8)
            self.lib.jbo_ets_info(self.ets, g, ctypes.byref(size), label, ctypes.byref(cx), ctypes.byref(cz))
            out.append((label.value.decode(), size.value, cx.value, cz.value))
        return out

    def sample(self, seed, trial_idx, p):
        err = np.zeros(self.n, np.uint8)
        self.lib.jbo_sample(_u64(seed), trial_idx, p, self.n, _ptr(err))
        return err

    def syndrome(self, err):
        err = np.ascontiguousarray(err, np.uint8)
        sx = np.zeros(self.m[0], np.uint8)
        sz = np.zeros(self.m[1], np.uint8)
        self.lib.jbo_syndrome(ctypes.byref(self.code), 0, _ptr(err), _ptr(sx))
        self.lib.jbo_syndrome(ctypes.byref(self.code), 1, _ptr(err), _ptr(sz))
        return sx, sz

    def decode(self, sx, sz, p, max_iter, flip_hist=5, freeze_syn=False, damping=0.0, enable_pp=False,
               want_llr=False):
        sx = np.ascontiguousarray(sx, np.uint8)
        sz = np.ascontiguousarray(sz, np.uint8)
        est = np.zeros(self.n, np.uint8)
        lx = np.zeros(self.n, np.float64) if want_llr else None
        lz = np.zeros(self.n, np.float64) if want_llr else None
        res = _Result()
        self.lib.jbo_decode(ctypes.byref(self.code), self.ets, self.work, _ptr(sx), _ptr(sz), p, max_iter,
                            flip_hist, int(freeze_syn), damping, int(enable_pp), _ptr(est),
                            _ptr(lx) if want_llr else None, _ptr(lz) if want_llr else None, ctypes.byref(res))
        out = {f: getattr(res, f) for f, _ in _Result._fields_}
        out["est"] = est
        if want_llr:
            out["abs_llr_x"], out["abs_llr_z"] = lx, lz
        return out

    def simulate_trial(self, seed, trial_idx, p, max_iter, flip_hist=5, damping=0.0, freeze_syn=False,
                       enable_pp=False, want_vectors=False):
        rec = TrialRecord()
        err = np.zeros(self.n, np.uint8) if want_vectors else None
        est = np.zeros(self.n, np.uint8) if want_vectors else None
        self.lib.jbo_simulate_trial(ctypes.byref(self.code), self.ets, ctypes.byref(self.bx), ctypes.byref(self.bz),
                                    self.work, _u64(seed), trial_idx, p, max_iter, flip_hist, damping,
                                    int(freeze_syn), int(enable_pp), ctypes.byref(rec),
                                    _ptr(err) if want_vectors else None, _ptr(est) if want_vectors else None)
        d = rec.as_dict()
        if want_vectors:
            d["err"], d["est"] = err, est
        return d

    def error_trial(self, err, p, max_iter, flip_hist=5, damping=0.0, freeze_syn=False, enable_pp=False):
        """The simulate-loop body on a known error: record and final estimate."""
        err = np.ascontiguousarray(err, np.uint8)
        rec = TrialRecord()
        est = np.zeros(self.n, np.uint8)
        self.lib.jbo_error_trial(ctypes.byref(self.code), self.ets, ctypes.byref(self.bx), ctypes.byref(self.bz),
                                 self.work, _ptr(err), 0, p, max_iter, flip_hist, damping, int(freeze_syn),
                                 int(enable_pp), ctypes.byref(rec), _ptr(est))
        d = rec.as_dict()
        d["est"] = est
        return d

    def classify(self, err, est):
        """(syndrome_ok, exact, stab_equiv, success) of a final estimate against the true error
        (jointbp_ets.cpp:6199-6211): the x-part of the residual must lie in rowspace(Hz) and the
        z-part in rowspace(Hx)."""
        err = np.ascontiguousarray(err, np.uint8)
        est = np.ascontiguousarray(est, np.uint8)
        sx, sz = self.syndrome(err)
        ex, ez = self.syndrome(est)
        ok = bool((sx == ex).all() and (sz == ez).all())
        exact = bool((err == est).all())
        stab = False
        if ok:
            words = (self.n + 63) // 64
            stab = True
            for part, basis in ((1, self.bz), (2, self.bx)):
                bits = np.zeros(words * 64, np.uint8)
                bits[:self.n] = ((err ^ est) & part) != 0
                vec = np.packbits(bits.reshape(-1, 8)[:, ::-1], axis=1).reshape(-1).view(np.uint64).copy()
                if not self.lib.jbo_in_row_space(ctypes.byref(basis), _ptr(vec)):
                    stab = False
                    break
        return ok, exact, stab, ok and stab

    def wilson(self, n, k, z=1.96):
        lo, hi = ctypes.c_double(), ctypes.c_double()
        self.lib.jbo_wilson(n, k, z, ctypes.byref(lo), ctypes.byref(hi))
        return lo.value, hi.value


class Reference:
    """Harness over the unmodified reference source (oracle/_ref/libjbp_ref.so)."""

    def __init__(self, params=PARAMS):
        path = REF_DIR / "libjbp_ref.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run `make -C oracle reference` where the reference sources exist")
        self.lib = lib = ctypes.CDLL(str(path))
        lib.ref_sample.argtypes = [ctypes.c_ulonglong, ctypes.c_longlong, ctypes.c_double, ctypes.c_void_p]
        lib.ref_bp_decode.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_simulate_trial.argtypes = [ctypes.c_ulonglong, ctypes.c_longlong, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        lib.ref_error_trial.argtypes = [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        if lib.ref_init(str(params).encode(), None) != 0:
            raise RuntimeError("ref_init failed")
        self.n = lib.ref_nvars()
        self.m = (lib.ref_mx(), lib.ref_mz())

    def sample(self, seed, trial_idx, p):
        err = np.zeros(self.n, np.int32)
        self.lib.ref_sample(_u64(seed), trial_idx, p, _ptr(err))
        return err.astype(np.uint8)

    def bp_decode(self, sx, sz, p, max_iter, damping=0.0, freeze_syn=False, want_llr=False):
        sx = np.ascontiguousarray(sx, np.int32)
        sz = np.ascontiguousarray(sz, np.int32)
        est = np.zeros(self.n, np.int32)
        ok = ctypes.c_int()
        lx = np.zeros(self.n) if want_llr else None
        lz = np.zeros(self.n) if want_llr else None
        it = self.lib.ref_bp_decode(_ptr(sx), _ptr(sz), p, max_iter, damping, int(freeze_syn), _ptr(est),
                                    ctypes.byref(ok), _ptr(lx) if want_llr else None, _ptr(lz) if want_llr else None)
        out = {"iterations": it, "syndrome_ok": ok.value, "est": est.astype(np.uint8)}
        if want_llr:
            out["abs_llr_x"], out["abs_llr_z"] = lx, lz
        return out

    def simulate_trial(self, seed, trial_idx, p, max_iter, flip_hist=5, damping=0.0, freeze_syn=False,
                       enable_pp=False, want_vectors=False):
        rec = TrialRecord()
        err = np.zeros(self.n, np.int32)
        est = np.zeros(self.n, np.int32)
        self.lib.ref_simulate_trial(_u64(seed), trial_idx, p, max_iter, flip_hist, damping, int(freeze_syn),
                                    int(enable_pp), ctypes.byref(rec), _ptr(err), _ptr(est))
        d = rec.as_dict()
        if want_vectors:
            d["err"], d["est"] = err.astype(np.uint8), est.astype(np.uint8)
        return d


    def error_trial(self, err, p, max_iter, flip_hist=5, damping=0.0, freeze_syn=False, enable_pp=False):
        e = np.ascontiguousarray(err, np.int32)
        rec = TrialRecord()
        est = np.zeros(self.n, np.int32)
        self.lib.ref_error_trial(_ptr(e), 0, p, max_iter, flip_hist, damping, int(freeze_syn), int(enable_pp),
                                 ctypes.byref(rec), _ptr(est))
        d = rec.as_dict()
        d["est"] = est.astype(np.uint8)
        return d


def reference_available():
    return (REF_DIR / "libjbp_ref.so").exists()
