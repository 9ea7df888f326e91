"""C-ABI library checks that need no GPU: it loads, exports every declared symbol, and its
host-side pieces (reference-stream sampler, error paths) behave."""
import ctypes
import json
import re
import subprocess
import zlib
from pathlib import Path

import numpy as np
import pytest

from conftest import GOLDEN, ROOT

INCLUDE = ROOT / "include"
LIBDIR = ROOT / "joint_bp_plus_pp_b200" / "lib"


def declared_functions(header):
    text = re.sub(r"/\*.*?\*/", "", header.read_text(), flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r"^\s*#[^\n]*", "", text, flags=re.M)
    names = re.findall(r"\b([A-Za-z_][A-Za-z0-9_]*)\s*\([^;{]*\)\s*;", text)
    return sorted(set(n for n in names if not n.startswith("__")))


def exported(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", str(lib)], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if line.strip()}


def test_dropin_library_exports_the_reference_boundary():
    """lib/libjointbp_cuda.so exports the three jointbp_cuda.h functions with the reference's
    C++ signatures (jointbp_cuda.h:46-62), so the reference host program links against it."""
    lib = LIBDIR / "libjointbp_cuda.so"
    assert lib.exists(), "run python -m joint_bp_plus_pp_b200.build"
    out = subprocess.run(["nm", "-DC", "--defined-only", str(lib)], capture_output=True, text=True,
                         check=True).stdout
    sigs = {re.sub(r"^\S+\s+\S+\s+", "", l) for l in out.splitlines() if "cuda_bp_" in l}
    s = "std::__cxx11::basic_string<char, std::char_traits<char>, std::allocator<char> >*"
    v = "std::vector<int, std::allocator<int> > const&"
    assert f"cuda_bp_create(CudaBPGraph const&, int, {s})" in sigs
    assert "cuda_bp_destroy(CudaBPContext*)" in sigs
    assert (f"cuda_bp_decode(CudaBPContext*, {v}, {v}, CudaMsg const&, int, int, int, bool, bool, bool, double, "
            f"CudaBPResult&, {s})") in sigs
    for name in declared_functions(INCLUDE / "jointbp_cuda.h"):
        assert any(x.startswith(name + "(") for x in sigs), name
    ctypes.CDLL(str(lib))


def test_library_exports_all_declared_symbols():
    lib = LIBDIR / "libjbp_b200.so"
    assert lib.exists(), "run python -m joint_bp_plus_pp_b200.build"
    decl = declared_functions(INCLUDE / "jbp_b200.h")
    assert "jbp_simulate" in decl and "jbp_decode_errors" in decl
    missing = [d for d in decl if d not in exported(lib)]
    assert not missing, missing
    ctypes.CDLL(str(lib))


def test_shim_exports_reference_boundary():
    lib = LIBDIR / "libjointbp_cuda.so"
    if not lib.exists():
        pytest.skip("shim not built")
    syms = exported(lib)
    # C++ symbols of jointbp_cuda.h (Itanium mangling of the reference signatures)
    for name in ("cuda_bp_create", "cuda_bp_destroy", "cuda_bp_decode"):
        assert any(name in s for s in syms), name


def test_version_and_error_strings():
    from joint_bp_plus_pp_b200 import load_library
    lib = load_library()
    assert b"sm_100a" in lib.jbp_version()
    h = ctypes.c_void_p()
    rc = lib.jbp_create_from_params(b"/nonexistent/params.txt", None, 0, ctypes.byref(h))
    assert rc == 3 and b"cannot open" in lib.jbp_last_error()
    assert not h.value


def test_host_reference_sampler_matches_golden():
    from joint_bp_plus_pp_b200 import sample_reference_errors
    kat = json.loads((GOLDEN / "kat.json").read_text())
    for key, exp in kat["sampler"].items():
        seed, p, idx = key.split(":")
        e = sample_reference_errors(9216, int(seed), int(idx), 1, float(p), threads=1)[0]
        assert zlib.crc32(e.tobytes()) & 0xFFFFFFFF == exp["crc"], key


def test_host_reference_sampler_threads_agree():
    from joint_bp_plus_pp_b200 import sample_reference_errors
    a = sample_reference_errors(9216, 106, 1, 24, 0.04, threads=1)
    b = sample_reference_errors(9216, 106, 1, 24, 0.04, threads=5)
    assert (a == b).all()


def test_no_gpu_is_an_error_not_a_fallback():
    """Without a usable device the library reports a CUDA error; it never decodes on the CPU."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from joint_bp_plus_pp_b200 import Decoder, JbpError
    with pytest.raises(JbpError) as ei:
        Decoder.from_params()
    assert ei.value.code == 2


def test_noalloc_entry_point_rejects_bad_options_before_any_cuda_call():
    """jbp_decode_syndromes_noalloc checks its options with the same rules as the other entry
    points before it touches a device: an unknown precision, an out-of-range prior entry or an
    error rate outside (0, 1) is JBP_ERR_ARG, an engine other than AUTO or SLOTS (it runs the
    slot engine's kernels only) is JBP_ERR_UNSUPPORTED, with no context needed to see it."""
    from joint_bp_plus_pp_b200 import Options, load_library
    lib = load_library()
    f = lib.jbp_decode_syndromes_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]

    def call(p=0.05, **kw):
        co = Options(max_iter=10, enable_pp=False, **kw).to_c()
        return f(None, ctypes.byref(co), 32, None, None, p, None, None, None)

    co = Options(max_iter=10, enable_pp=False).to_c()
    co.precision = 7
    assert f(None, ctypes.byref(co), 32, None, None, 0.05, None, None, None) == 1
    assert b"unknown precision" in lib.jbp_last_error()
    co = Options(max_iter=10, enable_pp=False).to_c()
    co.use_prior = 1
    co.prior[:] = [0.9, 0.05, 1.5, 0.05]
    assert f(None, ctypes.byref(co), 32, None, None, 0.05, None, None, None) == 1
    assert b"prior" in lib.jbp_last_error()
    assert call(p=1.5) == 1 and b"p must be" in lib.jbp_last_error()
    assert call(engine="resident") == 4 and b"slot engine" in lib.jbp_last_error()
    assert call(engine="table") == 4
    # valid options and no context: an argument error, still before any CUDA call
    assert call(precision="fp32", engine="slots") == 1 and b"invalid argument" in lib.jbp_last_error()
