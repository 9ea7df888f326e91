"""GPU tests of the host-side failure paths: allocation failures injected on the host
(jbp_debug_fail_allocation) and runs stopped from another host thread (jbp_request_abort).

Nothing here faults, traps or hangs a GPU.  An injected allocation failure is a
cudaErrorMemoryAllocation returned by the library's allocation wrapper without calling the CUDA
runtime; an abort is a store to a pinned host word that the persistent kernels read between
trials (and the slot engine's loop condition reads every iteration), after which they claim no
further trial and return.  Each test then decodes on the same context to show that it is still
usable and decodes exactly as before.
"""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cfgs():
    from joint_bp_plus_pp_b200 import Options
    return {
        "slots_fp64_pp": Options(precision="fp64", engine="slots", max_iter=300, enable_pp=True),
        "resident_fp32_learned": Options(precision="fp32", engine="resident", max_iter=300, enable_pp=True,
                                         learned_from=6),
        "table_fp32": Options(precision="fp32", engine="table", max_iter=300, enable_pp=False),
        # calls of two syndromes each: pinned staging and the single-trial FP64 path
        "single_fp64_syndromes": Options(precision="fp64", max_iter=300, enable_pp=False),
    }


def _syndromes(dec, err):
    out = []
    for side in (0, 1):
        off, var = dec.checks(side)
        bits = (err >> side) & 1
        dc = int(off[1] - off[0])
        out.append((bits[:, var].reshape(err.shape[0], -1, dc).sum(axis=2) % 2).astype(np.uint8))
    return out


def _run(dec, opts):
    if opts.engine == "auto" and opts.precision == "fp64" and not opts.enable_pp:
        err = dec.sample_errors(106, 3, 8, 0.045)
        sx, sz = _syndromes(dec, err)
        recs, ests = [], []
        for i in range(0, 8, 2):
            st, r, e = dec.decode_syndromes(sx[i:i + 2], sz[i:i + 2], 0.045, opts)
            assert st["slots"] == 1   # the single-trial path ran
            recs.append(r)
            ests.append(e)
        return np.concatenate(ests), np.concatenate(recs)
    return dec.simulate(106, 1024, 0.045, opts, first_trial=3)


@pytest.mark.parametrize("name", ["slots_fp64_pp", "resident_fp32_learned", "table_fp32", "single_fp64_syndromes"])
def test_every_allocation_failure_is_reported_and_recovered(name):
    """The k-th allocation of creating a context and running it fails, for every k until the
    path completes: each failure comes back as JBP_ERR_CUDA "out of memory" (never a crash or a
    wrong result), and a context that was created decodes the same trials as a clean one."""
    from joint_bp_plus_pp_b200 import Decoder, JbpError, debug_fail_allocation, load_flip_model
    opts = _cfgs()[name]
    params = load_flip_model() if opts.learned_from > 0 else None
    ref = Decoder.from_params()
    if params is not None:
        ref.set_flip_model(params)
    _, want = _run(ref, opts)
    ref.close()
    failures = 0
    for k in range(400):
        debug_fail_allocation(k)
        dec = None
        try:
            dec = Decoder.from_params()
            if params is not None:
                dec.set_flip_model(params)
            _, got = _run(dec, opts)
            debug_fail_allocation(-1)
            assert (got == want).all()
            break   # k is past the path's last allocation: nothing failed
        except JbpError as e:
            debug_fail_allocation(-1)
            assert e.code == 2 and "out of memory" in str(e), str(e)
            failures += 1
            if dec is not None:
                if params is not None:
                    dec.set_flip_model(params)
                _, got = _run(dec, opts)
                assert (got == want).all(), k
        finally:
            debug_fail_allocation(-1)
            if dec is not None:
                dec.close()
    else:
        pytest.fail("the path never completed")
    assert failures >= 5, failures


def _abort_after(dec, delay, fn):
    """Runs fn() on a host thread and asks dec to abort after `delay` seconds; returns the
    JbpError fn raised (or None) and the wall time of fn."""
    out = {}

    def body():
        t0 = time.perf_counter()
        try:
            fn()
            out["err"] = None
        except Exception as e:  # noqa: BLE001 - returned to the test
            out["err"] = e
        out["wall"] = time.perf_counter() - t0

    th = threading.Thread(target=body)
    th.start()
    time.sleep(delay)
    dec.request_abort()
    th.join(timeout=120)
    assert not th.is_alive(), "the run did not stop"
    return out["err"], out["wall"]


@pytest.mark.parametrize("engine,prec,pp", [("resident", "fp32", True), ("resident", "fp16", False),
                                            ("table", "fp32", False), ("slots", "fp64", False)])
def test_abort_from_another_thread(decoder, engine, prec, pp):
    """A run of far more trials than fit in the wait stops soon after the request, returns
    JBP_ERR_ABORTED with the counters of the trials that finished, and the context then decodes
    the same trials as before; the request does not outlive the run it stopped."""
    from joint_bp_plus_pp_b200 import Options
    opts = Options(precision=prec, engine=engine, max_iter=1000, enable_pp=pp)
    _, before = decoder.simulate(106, 2048, 0.04, opts, first_trial=7)
    big = 200_000_000
    err, wall = _abort_after(decoder, 0.5, lambda: decoder.simulate(106, big, 0.04, opts, per_trial=False))
    assert err is not None and err.code == 6, err
    assert "aborted by request" in str(err)
    st = err.stats
    assert st is not None and 0 < st["trials"] < big // 10, st
    assert st["failures"] <= st["trials"] and st["total_iters"] >= st["trials"]
    assert wall < 20, wall
    _, after = decoder.simulate(106, 2048, 0.04, opts, first_trial=7)
    assert (after == before).all()


def test_abort_before_a_run_stops_that_run_only(decoder):
    """A request made while nothing runs stops the next run at once; the one after is whole."""
    from joint_bp_plus_pp_b200 import JbpError, Options
    opts = Options(precision="fp32", engine="resident", max_iter=1000, enable_pp=True)
    decoder.request_abort()
    with pytest.raises(JbpError) as ei:
        decoder.simulate(106, 10_000_000, 0.04, opts, per_trial=False)
    assert ei.value.code == 6
    assert ei.value.stats["trials"] < 10_000_000
    st, _ = decoder.simulate(106, 4096, 0.04, opts, per_trial=False)
    assert st["trials"] == 4096


def test_cli_interrupt_prints_partial_summary(tmp_path):
    """SIGINT to the command-line driver during --simulate: exit status 130 and a Run Summary
    of the trials decoded before the interrupt."""
    import signal
    import subprocess
    from pathlib import Path
    exe = Path(__file__).resolve().parents[1] / "joint_bp_plus_pp_b200" / "bin" / "jointbp_b200"
    params = Path(__file__).resolve().parents[1] / "joint_bp_plus_pp_b200" / "data" / \
        "H_P768_J3_L12_dmax3_nc0-3_1-2_seed11579811919164041.txt"
    proc = subprocess.Popen([str(exe), "--params", str(params), "--simulate", "--cuda", "--p", "0.04",
                             "--trials", "2000000000", "--max-iter", "1000", "--seed", "106", "--batch", "1000000000"],
                            stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, cwd=str(params.parent))
    time.sleep(8.0)   # context creation, then decoding
    proc.send_signal(signal.SIGINT)
    out, err = proc.communicate(timeout=120)
    assert proc.returncode == 130, (proc.returncode, err[-2000:])
    assert "interrupted:" in err
    line = [ln for ln in out.splitlines() if ln.startswith("trials=")]
    assert line, out[-2000:]
    trials = int(line[-1].split()[0].split("=")[1])
    assert 0 < trials < 2_000_000_000, line[-1]
