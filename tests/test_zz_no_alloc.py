"""GPU test of jbp_decode_syndromes_noalloc, the allocation-free decode entry point.

That entry point serves callers that cannot call cudaMalloc while they decode: programs
whose device memory belongs to another allocator, and decoding loops that must not
allocate after start-up.  Everything it needs besides its inputs and outputs lives in a
fixed device array inside the library.  The test calls it through the C ABI on device
buffers and compares it with jbp_decode_syndromes, which allocates its own buffers, on two
calls in a row; the array keeps the previous call's contents, so the second call also shows
that each call starts from a clean state.  The file name makes pytest collect it last.
"""
import ctypes

import numpy as np
import pytest

from conftest import load_sim_case

pytestmark = pytest.mark.gpu


def syndromes(dec, err):
    out = []
    for side in (0, 1):
        off, var = dec.checks(side)
        bits = (err >> side) & 1                      # x-bit for side 0, z-bit for side 1
        dc = int(off[1] - off[0])
        out.append((bits[:, var].reshape(err.shape[0], -1, dc).sum(axis=2) % 2).astype(np.uint8))
    return out


def run_noalloc(dec, opts, sx, sz, p):
    import torch
    from joint_bp_plus_pp_b200 import TRIAL_DTYPE
    lib = dec._lib
    lib.jbp_decode_syndromes_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p]
    t = sx.shape[0]
    d_sx = torch.from_numpy(np.ascontiguousarray(sx)).cuda()
    d_sz = torch.from_numpy(np.ascontiguousarray(sz)).cuda()
    d_est = torch.full((t, dec.n), 0xFF, dtype=torch.uint8, device="cuda")
    d_res = torch.zeros((t, TRIAL_DTYPE.itemsize), dtype=torch.uint8, device="cuda")
    co = opts.to_c()
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.jbp_decode_syndromes_noalloc(dec._h, ctypes.byref(co), t, d_sx.data_ptr(), d_sz.data_ptr(), p,
                                          d_est.data_ptr(), d_res.data_ptr(), stream)
    torch.cuda.synchronize()
    assert rc == 0, lib.jbp_last_error()
    res = np.frombuffer(d_res.cpu().numpy().tobytes(), dtype=TRIAL_DTYPE)
    return res, d_est.cpu().numpy()


def check_same(dec, opts, err, p):
    """The allocation-free call runs the slot engine's kernels, so the allocating call it is
    compared with runs the slot engine too (engine AUTO could pick the trial-resident kernels
    for FP16, whose arithmetic differs slightly)."""
    from dataclasses import replace
    sx, sz = syndromes(dec, err)
    _, exp_res, exp_est = dec.decode_syndromes(sx, sz, p, replace(opts, engine="slots"))
    res, est = run_noalloc(dec, opts, sx, sz, p)
    assert (est == exp_est).all()
    for f in ("iterations", "syndrome_ok", "bp_ok", "success"):
        assert (res[f] == exp_res[f]).all(), f


def test_noalloc_matches_allocating_entry_point_twice(decoder):
    from joint_bp_plus_pp_b200 import Options, sample_reference_errors
    meta, errs, _ = load_sim_case("p050_mi50_nopp_s1")
    # first call: FP64 (bit-exact path) on the reference's golden trials
    check_same(decoder, Options(precision="fp64", max_iter=50, enable_pp=False), errs[:16], meta["p"])
    # second call: other trials and another precision, through the same scratch array
    err2 = sample_reference_errors(decoder.n, 77, 1, 40, 0.06)
    check_same(decoder, Options(precision="fp32", max_iter=40, enable_pp=False), err2, 0.06)
    # third call: FP16 message storage (the slot engine's FP16 kernels)
    err3 = sample_reference_errors(decoder.n, 78, 1, 48, 0.05)
    check_same(decoder, Options(precision="fp16", max_iter=40, enable_pp=False), err3, 0.05)


def test_noalloc_leaves_the_callers_device_current(decoder):
    """The call selects the context's device for its own work and restores the caller's
    current device before it returns."""
    import torch
    from joint_bp_plus_pp_b200 import Options, sample_reference_errors
    before = torch.cuda.current_device()
    err = sample_reference_errors(decoder.n, 79, 1, 8, 0.05)
    check_same(decoder, Options(precision="fp32", max_iter=20, enable_pp=False), err, 0.05)
    assert torch.cuda.current_device() == before


def test_noalloc_rejects_requests_beyond_its_scratch(decoder):
    import torch
    from joint_bp_plus_pp_b200 import Options
    lib = decoder._lib
    lib.jbp_decode_syndromes_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p]
    from joint_bp_plus_pp_b200 import TRIAL_DTYPE
    co = Options(precision="fp64", max_iter=10, enable_pp=False).to_c()
    # buffers of the full size of the request, so that even a call that were not rejected
    # would stay inside them
    t = 4096
    d_sx = torch.zeros((t, decoder.mx), dtype=torch.uint8, device="cuda")
    d_sz = torch.zeros((t, decoder.mz), dtype=torch.uint8, device="cuda")
    d_res = torch.zeros((t, TRIAL_DTYPE.itemsize), dtype=torch.uint8, device="cuda")
    rc = lib.jbp_decode_syndromes_noalloc(decoder._h, ctypes.byref(co), t, d_sx.data_ptr(), d_sz.data_ptr(), 0.05,
                                          None, d_res.data_ptr(), None)
    assert rc == 1
    assert b"scratch" in lib.jbp_last_error()
