"""The build's guard against register spills in the trial-resident kernels."""
import pytest

from joint_bp_plus_pp_b200.build import RESIDENT_SPILL_LIMIT, check_resident_spills

LOG = """ptxas info    : Function properties for _ZN3jbp10k_residentILi768ELi3ELi12ENS_9StoreHalfELb1ELb1EEEvNS_7ResCodeENS_6ResRunE
    4416 bytes stack frame, {} bytes spill stores, 328 bytes spill loads
ptxas info    : Function properties for _ZN3jbp9k_var_llrIfLi12ELi3ELb0EEEvNS_7DevCodeENS_6DevRunENS_7DevMsgsEf
    0 bytes stack frame, 4000 bytes spill stores, 0 bytes spill loads"""


def test_spill_guard_passes_small_spills_and_other_kernels():
    check_resident_spills(LOG.format(RESIDENT_SPILL_LIMIT))


def test_spill_guard_rejects_spilling_resident_kernels():
    with pytest.raises(RuntimeError, match="spill"):
        check_resident_spills(LOG.format(RESIDENT_SPILL_LIMIT + 4))
