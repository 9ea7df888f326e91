"""Generates the golden fixtures in tests/golden/ from the reference itself.

Runs in a container that has the reference sources (built into oracle/_ref/ by
`make -C oracle`): the per-trial records come from the harness over the unmodified
reference decoder (oracle/_ref/libjbp_ref.so), the run summaries from the unmodified
reference CLI (oracle/_ref/jointbp_ets).  The fixtures are small JSON/NPZ files that
travel with the repository; the GPU tests read them without the reference present.

    python tests/golden/make_golden.py [--quick]
"""
import argparse
import hashlib
import json
import re
import subprocess
import sys
import zlib
from pathlib import Path

import ctypes

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
from oracle_bind import ETS_DIR, PARAMS, REF_DIR, Reference  # noqa: E402

# (name, seed, p, max_iter, enable_pp, flip_hist, trials, vectors_for_first[, freeze_syn])
SIM_CASES = [
    ("p050_mi50_nopp_s1", 1, 0.05, 50, False, 5, range(1, 201), 16),
    ("p040_mi1000_nopp_s106", 106, 0.04, 1000, False, 5, range(1, 101), 16),
    ("p050_mi200_pp_s305", 305, 0.05, 200, True, 5, range(1, 41), 40),
    ("p060_mi120_pp_s7", 7, 0.06, 120, True, 5, range(1, 25), 24),
    ("p055_mi150_pp_fh0_s11", 11, 0.055, 150, True, 0, range(1, 21), 20),
    ("p055_mi60_nopp_frz_s21", 21, 0.055, 60, False, 5, range(1, 121), 32, True),
    ("p060_mi130_pp_frz_s23", 23, 0.06, 130, True, 5, range(1, 25), 24, True),
]


def crc(a):
    return zlib.crc32(np.ascontiguousarray(a, np.uint8).tobytes()) & 0xFFFFFFFF


def run_cli(args):
    exe = REF_DIR / "jointbp_ets"
    out = subprocess.run([str(exe), "--params", str(PARAMS)] + args, capture_output=True, text=True,
                         cwd=str(PARAMS.parent), check=False)
    line = [l for l in out.stdout.splitlines() if l.startswith("trials=")]
    return out.returncode, line[-1] if line else None, out.stdout


def parse_summary(line):
    d = {}
    for k, v in re.findall(r"(\w+)=(\[[^\]]*\]|\S+)", line):
        d[k] = v
    return d


# Sampled trials on which in-loop post-processing saves the decode (seed, p, max_iter, trial):
# flip at 2001/78, 2001/550, 2002/130, 2002/629, 2002/1042; OSD on the others.
PP_SAVED_TRIALS = [(2001, 0.05, 130, 78), (2001, 0.05, 130, 550), (2002, 0.055, 130, 130),
                   (2002, 0.055, 130, 133), (2002, 0.055, 130, 169), (2002, 0.055, 130, 311),
                   (2002, 0.055, 130, 355), (2002, 0.055, 130, 358), (2002, 0.055, 130, 629),
                   (2002, 0.055, 130, 693), (2002, 0.055, 130, 773), (2002, 0.055, 130, 999),
                   (2002, 0.055, 130, 1042)]


def sparse(v):
    nz = np.nonzero(v)[0]
    return [[int(i), int(v[i])] for i in nz]


def ets_entries(path, P):
    """(side, vars, unsat checks) of each line of an ETS file; ids are block * P + offset."""
    out = []
    for ln in path.read_text().splitlines():
        m_v, m_u = re.search(r"vars=(\S+)", ln), re.search(r"unsat=(\S+)", ln)
        if not m_v or not m_u:
            continue
        ids = lambda s: [int(t[1:].split(":")[0]) * P + int(t.split(":")[1]) for t in s.split(",")]
        out.append((ln.split()[0], ids(m_v.group(1)), ids(m_u.group(1))))
    return out


def stage_trials(ref):
    """Per-trial reference records on errors that make post-processing act.

    Constructed cases put one ETS entry's variables in error (Pauli X, Z or Y, whichever
    leaves exactly that entry's two checks unsatisfied on its side) and decode with a small
    iteration cap, so the in-loop ETS, flip and OSD stages and the post-BP ETS all fire.
    Sampled cases are the PP_SAVED_TRIALS plus the first post-processed failures of seed 2002.
    """
    cases = []
    P = 768
    for path in sorted(ETS_DIR.glob("ets_*.txt")):
        for side, vs, uc in ets_entries(path, P)[:3]:
            for st in (1, 2, 3):
                e = np.zeros(ref.n, np.uint8)
                e[sorted(set(vs))] = st
                sx = np.zeros(ref.m[0], np.int32)
                sz = np.zeros(ref.m[1], np.int32)
                ref.lib.ref_syndrome(e.astype(np.int32).ctypes.data_as(ctypes.c_void_p),
                                     sx.ctypes.data_as(ctypes.c_void_p), sz.ctypes.data_as(ctypes.c_void_p))
                s = sx if side == "X" else sz
                if sorted(np.nonzero(s)[0].tolist()) != sorted(uc):
                    continue
                for mi in (1, 2, 5, 20):
                    d = ref.error_trial(e, 0.05, mi, flip_hist=5, enable_pp=True)
                    est = d.pop("est")
                    cases.append({"label": f"{path.stem}:{side}:{st}", "p": 0.05, "max_iter": mi, "flip_hist": 5,
                                  "err": sparse(e), "est": sparse(est), "record": d})
    fails = 0
    sampled = list(PP_SAVED_TRIALS)
    for t in range(1, 400):
        if fails >= 8:
            break
        d = ref.simulate_trial(2002, t, 0.055, 130, enable_pp=True)
        if not d["success"] and d["pp_in_decode"]:
            sampled.append((2002, 0.055, 130, t))
            fails += 1
    for seed, p, mi, t in sampled:
        d = ref.simulate_trial(seed, t, p, mi, flip_hist=5, enable_pp=True, want_vectors=True)
        e, est = d.pop("err"), d.pop("est")
        cases.append({"label": f"seed{seed}:trial{t}", "p": p, "max_iter": mi, "flip_hist": 5,
                      "err": sparse(e), "est": sparse(est), "record": d})
    (HERE / "pp_stage_trials.json").write_text(json.dumps(cases))
    print("stage trials", len(cases), "ets_pp", sum(c["record"]["ets_pp_ok"] for c in cases),
          "flip_pp", sum(c["record"]["flip_pp_ok"] for c in cases),
          "osd", sum(c["record"]["osd_success"] for c in cases),
          "post", sum(c["record"]["ets_applied_post"] for c in cases), flush=True)


def simulate_cases(ref, cases):
    """Per-trial reference records (and the first vectors) of seeded simulate runs."""
    for case in cases:
        name, seed, p, mi, pp, fh, trials, nvec = case[:8]
        frz = bool(case[8]) if len(case) > 8 else False
        recs, errs, ests = [], [], []
        for k, t in enumerate(trials):
            d = ref.simulate_trial(seed, t, p, mi, flip_hist=fh, enable_pp=pp, freeze_syn=frz, want_vectors=True)
            e, s = d.pop("err"), d.pop("est")
            d["err_crc"], d["est_crc"] = crc(e), crc(s)
            recs.append(d)
            if k < nvec:
                errs.append(e)
                ests.append(s)
        meta = {"seed": seed, "p": p, "max_iter": mi, "enable_pp": pp, "flip_hist": fh, "freeze_syn": frz,
                "records": recs}
        (HERE / f"sim_{name}.json").write_text(json.dumps(meta))
        np.savez_compressed(HERE / f"vec_{name}.npz", err=np.array(errs, np.uint8), est=np.array(ests, np.uint8))
        print(name, "failures", sum(1 - r["success"] for r in recs), "pp", sum(r["pp_success_this"] for r in recs),
              flush=True)


def cli_summaries(quick):
    """Run Summary lines of the unmodified reference CLI (cli_summaries.json)."""
    summaries = {}
    cli_cases = [("p050_mi50_nopp_s1_t200", ["--simulate", "--p", "0.05", "--trials", "200", "--max-iter", "50",
                                             "--no-pp", "--seed", "1", "--report-every", "0"]),
                 ("p050_mi200_pp_s305_t40", ["--simulate", "--p", "0.05", "--trials", "40", "--max-iter", "200",
                                             "--flip-hist", "5", "--seed", "305", "--report-every", "0"]),
                 ("p055_mi60_nopp_frz_s21_t60", ["--simulate", "--p", "0.055", "--trials", "60", "--max-iter", "60",
                                                 "--no-pp", "--freeze-syn", "--seed", "21", "--report-every", "0"]),
                 ("p050_mi50_nopp_s1_t20", ["--simulate", "--p", "0.05", "--trials", "20", "--max-iter", "50",
                                            "--no-pp", "--seed", "1", "--report-every", "0"])]
    if not quick:
        cli_cases.append(("p050_mi50_nopp_s1_t1000", ["--simulate", "--p", "0.05", "--trials", "1000",
                                                      "--max-iter", "50", "--no-pp", "--seed", "1",
                                                      "--report-every", "0"]))
    for name, a in cli_cases:
        rc, line, _ = run_cli(a)
        summaries[name] = {"args": a, "rc": rc, "summary": parse_summary(line) if line else None}
        print(name, line, flush=True)
    (HERE / "cli_summaries.json").write_text(json.dumps(summaries, indent=1))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true", help="skip the 1000-trial CLI summary")
    ap.add_argument("--stage-only", action="store_true", help="regenerate only pp_stage_trials.json")
    ap.add_argument("--cli-only", action="store_true", help="regenerate only cli_summaries.json")
    ap.add_argument("--sim", action="append", default=[], help="regenerate only these simulate cases")
    args = ap.parse_args()
    ref = Reference()
    lib = ref.lib
    if args.stage_only:
        stage_trials(ref)
        return
    if args.cli_only:
        cli_summaries(args.quick)
        return
    if args.sim:
        simulate_cases(ref, [c for c in SIM_CASES if c[0] in args.sim])
        return

    # --- code known answers (README start-up block) ---
    cnt = np.zeros(64, np.int32)
    labels = ctypes.create_string_buffer(32 * 8)
    ng = lib.ref_ets_counts(cnt.ctypes.data_as(ctypes.c_void_p), 32, labels, 8)
    groups = []
    for i in range(ng):
        groups.append({"label": labels.raw[i * 8:(i + 1) * 8].split(b"\0")[0].decode(),
                       "x": int(cnt[2 * i]), "z": int(cnt[2 * i + 1])})
    xchk = np.zeros(ref.m[0] * 12, np.int32)
    zchk = np.zeros(ref.m[1] * 12, np.int32)
    lib.ref_checks(0, xchk.ctypes.data_as(ctypes.c_void_p))
    lib.ref_checks(1, zchk.ctypes.data_as(ctypes.c_void_p))
    kat = {"n": ref.n, "mx": ref.m[0], "mz": ref.m[1], "rank_x": lib.ref_rank_x(), "rank_z": lib.ref_rank_z(),
           "girth_x": lib.ref_girth(0), "girth_z": lib.ref_girth(1), "ets_groups": groups,
           "x_checks_sha256": hashlib.sha256(xchk.tobytes()).hexdigest(),
           "z_checks_sha256": hashlib.sha256(zchk.tobytes()).hexdigest()}
    kat["k"] = kat["n"] - kat["rank_x"] - kat["rank_z"]

    # --- sampler goldens ---
    samp = {}
    for seed, p, idxs in ((106, 0.04, (1, 2, 3, 1000, 999999)), (1, 0.05, (1, 7)), (2 ** 63 + 5, 0.01, (4,))):
        for i in idxs:
            e = ref.sample(seed, i, p)
            samp[f"{seed}:{p}:{i}"] = {"crc": crc(e), "weight": int((e != 0).sum()),
                                       "counts": [int((e == s).sum()) for s in range(4)]}
    kat["sampler"] = samp
    (HERE / "kat.json").write_text(json.dumps(kat, indent=1))

    simulate_cases(ref, SIM_CASES)

    # --- |LLR| goldens (last-iteration |LLR| of plain BP; they order the OSD columns) ---
    llr = {}
    for seed, p, t, mi in ((305, 0.05, 19, 30), (1, 0.05, 3, 12)):
        e = ref.sample(seed, t, p)
        sx = np.zeros(ref.m[0], np.int32)
        sz = np.zeros(ref.m[1], np.int32)
        lib.ref_syndrome(e.astype(np.int32).ctypes.data_as(ctypes.c_void_p), sx.ctypes.data_as(ctypes.c_void_p),
                         sz.ctypes.data_as(ctypes.c_void_p))
        r = ref.bp_decode(sx, sz, p, mi, want_llr=True)
        llr[f"s{seed}_t{t}_mi{mi}"] = (r["abs_llr_x"], r["abs_llr_z"], r["est"], r["iterations"])
    np.savez_compressed(HERE / "llr_golden.npz",
                        **{k + "_x": v[0] for k, v in llr.items()}, **{k + "_z": v[1] for k, v in llr.items()},
                        **{k + "_est": v[2] for k, v in llr.items()},
                        **{k + "_iters": np.array([v[3]]) for k, v in llr.items()})

    cli_summaries(args.quick)
    stage_trials(ref)


if __name__ == "__main__":
    main()
