"""Builds the native parts of joint_bp_plus_pp_b200 in-tree with nvcc for sm_100a.

Outputs (next to this file, under lib/ and bin/):
  lib/libjbp_b200.so      the C-ABI library (include/jbp_b200.h)
  lib/libjointbp_cuda.so  drop-in for the reference's jointbp_cuda.h boundary
  bin/jointbp_b200        the command-line driver (the reference CLI surface)

    python -m joint_bp_plus_pp_b200.build [--jobs N] [--force]
"""
import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "lib"
BIN = PKG / "bin"
INCLUDE = ROOT / "include"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                  "-Xptxas", "-warn-spills", f"-I{INCLUDE}"]
HOSTFLAGS = ["-O2", "-std=c++17", "-fPIC", f"-I{INCLUDE}"]

LIB_SOURCES = ["code_model.cpp", "engine.cu", "capi.cu", "noalloc.cu", "learned.cu", "peaks.cu"]
SHIM_SOURCES = ["jointbp_cuda_shim.cpp"]
CLI_SOURCES = ["cli.cpp"]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def cuda_home():
    return str(Path(nvcc()).resolve().parent.parent)


def host_cxx():
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("g++ not found")


# Register spills of the trial-resident kernels above this (bytes of spill stores) fail the
# build: their 768-thread blocks run at 80 registers per thread, and spills in the BP loop
# have cost more than half of the throughput before.
RESIDENT_SPILL_LIMIT = 512


def check_resident_spills(log):
    """Raises if a k_resident instantiation reports more spill stores than the limit."""
    import re
    cur = None
    for line in log.splitlines():
        m = re.search(r"Function properties for (\S*k_resident\S*)", line)
        if m:
            cur = m.group(1)
            continue
        m = re.search(r"(\d+) bytes spill stores", line)
        if cur and m:
            if int(m.group(1)) > RESIDENT_SPILL_LIMIT:
                raise RuntimeError(f"{cur}: {m.group(1)} bytes of register spill stores "
                                   f"(limit {RESIDENT_SPILL_LIMIT})")
            cur = None


def _compile(src, force):
    out = OBJ / (Path(src).name + ".o")
    srcp = CSRC / src
    deps = [srcp] + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.hpp")) + list(INCLUDE.glob("*.h"))
    if not force and out.exists() and all(out.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return out, None
    if src.endswith(".cu"):
        cmd = [nvcc()] + NVFLAGS + (["-Xptxas", "-v"] if src == "engine.cu" else []) + ["-c", str(srcp), "-o", str(out)]
    else:
        cmd = [host_cxx()] + HOSTFLAGS + [f"-I{cuda_home()}/include", "-c", str(srcp), "-o", str(out)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if src == "engine.cu":
        try:
            check_resident_spills(r.stdout + r.stderr)
        except RuntimeError:
            out.unlink(missing_ok=True)
            raise
    return out, (r.stdout + r.stderr).strip() or None


def _link(objs, out, shared=True, extra=()):
    cmd = [nvcc()] + ARCH + (["-shared"] if shared else []) + [str(o) for o in objs] + ["-o", str(out),
                                                                                         "-lcudart"] + list(extra)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")


def build(jobs=None, force=False, verbose=False):
    OBJ.mkdir(exist_ok=True)
    LIB.mkdir(exist_ok=True)
    BIN.mkdir(exist_ok=True)
    sources = [s for s in LIB_SOURCES + SHIM_SOURCES + CLI_SOURCES if (CSRC / s).exists()]
    with ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
        results = list(ex.map(lambda s: _compile(s, force), sources))
    objs = {Path(o).name.rsplit(".", 1)[0]: o for o, _ in results}
    if verbose:
        for (o, log) in results:
            if log:
                print(f"--- {o.name}\n{log}")
    lib = LIB / "libjbp_b200.so"
    _link([objs[s] for s in LIB_SOURCES], lib)
    if all((CSRC / s).exists() for s in SHIM_SOURCES):
        _link([objs[s] for s in SHIM_SOURCES], LIB / "libjointbp_cuda.so",
              extra=[f"-L{LIB}", "-ljbp_b200", "-Xlinker", "-rpath,$ORIGIN"])
    if all((CSRC / s).exists() for s in CLI_SOURCES):
        _link([objs[s] for s in CLI_SOURCES], BIN / "jointbp_b200", shared=False,
              extra=[f"-L{LIB}", "-ljbp_b200", "-Xlinker", "-rpath,$ORIGIN/../lib"])
    return lib


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.jobs, a.force, a.verbose))


if __name__ == "__main__":
    sys.exit(main())
