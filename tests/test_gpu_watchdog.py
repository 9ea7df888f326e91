"""GPU tests of the run budget (jbp_options.watchdog_ms), the device-side counterpart of the
reference's "CUDA failure becomes a status and a message" contract (jointbp_cuda.cu:565-573).

The persistent kernels (trial-resident, table-driven / mixed) read the GPU's global timer
between trials and every 16 BP iterations; when the budget has run out a block claims no
further trial, abandons the one it decodes and returns, so the launch ends on its own and the
host reports JBP_ERR_TIMEOUT with the counters of the trials that did finish.  The slot engine
checks the same budget on the host between CUDA-graph launches.  No GPU fault is involved:
the budget is simply set far below the run's length (1 ms for about a second of work), and
each test then decodes on the same context to show that it is still usable.
"""
import pytest

pytestmark = pytest.mark.gpu

BIG = 1_000_000


def expect_timeout(fn):
    from joint_bp_plus_pp_b200 import JbpError
    with pytest.raises(JbpError) as ei:
        fn()
    e = ei.value
    assert e.code == 5, str(e)
    assert "watchdog" in str(e)
    assert e.stats is not None
    return e.stats


def same_after(decoder, opts, p):
    """Decodes 2,048 trials before and after the timed-out run: identical records."""
    _, before = decoder.simulate(106, 2048, p, opts, first_trial=7)
    return lambda: (decoder.simulate(106, 2048, p, opts, first_trial=7)[1] == before).all()


@pytest.mark.parametrize("prec", ["fp32", "fp16"])
def test_resident_run_budget(decoder, prec):
    from dataclasses import replace
    from joint_bp_plus_pp_b200 import Options
    opts = Options(precision=prec, engine="resident", max_iter=1000, enable_pp=True)
    check = same_after(decoder, opts, 0.04)
    st = expect_timeout(lambda: decoder.simulate(106, BIG, 0.04, replace(opts, watchdog_ms=1), per_trial=False))
    # a partial count: some trials finished, far from all, and every counter is consistent
    assert 0 < st["trials"] < BIG // 2, st["trials"]
    assert st["kernel_launches"] == 1
    assert st["failures"] <= st["trials"] and st["total_iters"] >= st["trials"]
    assert check()
    # a budget the run fits in changes nothing
    s2, r2 = decoder.simulate(106, 2048, 0.04, replace(opts, watchdog_ms=60_000), first_trial=7)
    assert s2["trials"] == 2048


def test_table_engine_run_budget(decoder):
    from dataclasses import replace
    from joint_bp_plus_pp_b200 import Options
    opts = Options(precision="fp32", engine="table", max_iter=1000, enable_pp=False)
    check = same_after(decoder, opts, 0.04)
    st = expect_timeout(lambda: decoder.simulate(106, BIG, 0.04, replace(opts, watchdog_ms=1), per_trial=False))
    assert 0 < st["trials"] < BIG // 2
    assert check()


def test_mixed_launch_run_budget():
    from joint_bp_plus_pp_b200 import Decoder, JbpError, Options, simulate_mixed
    from joint_bp_plus_pp_b200.codes import hgp_code
    decs = [Decoder.from_checks(*hgp_code(nc, i + 1), device=0) for i, nc in enumerate((32, 64))]
    opts = Options(precision="fp32", max_iter=200, enable_pp=False)
    with pytest.raises(JbpError) as ei:
        simulate_mixed(decs, [BIG, BIG], 0.04, Options(precision="fp32", max_iter=200, enable_pp=False,
                                                         watchdog_ms=1))
    assert ei.value.code == 5
    st, _ = simulate_mixed(decs, [512, 512], 0.04, opts)
    assert [s["trials"] for s in st] == [512, 512]


def test_slot_engine_run_budget(decoder):
    from dataclasses import replace
    from joint_bp_plus_pp_b200 import Options
    opts = Options(precision="fp64", engine="slots", max_iter=1000, enable_pp=False)
    check = same_after(decoder, opts, 0.04)
    st = expect_timeout(lambda: decoder.simulate(106, BIG, 0.04, replace(opts, watchdog_ms=1), per_trial=False))
    assert 0 <= st["trials"] < BIG // 2
    assert check()
