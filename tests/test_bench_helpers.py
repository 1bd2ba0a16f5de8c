"""Host-side helpers of bench.py, without a GPU: the committed ncu summaries
it reports beside its own timing, and its command line."""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402

KERNELS = ("kCreateMD", "kCreateLS", "kCreateT3", "kT5Eval")


@pytest.mark.parametrize("kernel", KERNELS)
def test_committed_dram_traffic(kernel):
    """Every kernel the bench may name as dominant has measured DRAM bytes,
    with the capture's provenance."""
    traffic, source = bench.committed_traffic(kernel)
    assert traffic is not None and 1e8 < traffic < 1e10
    assert "ncu" in source and "64" in source


@pytest.mark.parametrize("kernel", KERNELS)
def test_committed_issue_slots(kernel):
    ipc, frac, source = bench.committed_issue_slots(kernel)
    assert 0 < ipc <= 4 and frac == pytest.approx(ipc / 4, abs=0.01)
    assert "ncu" in source


def test_unknown_kernel_has_no_committed_figures():
    assert bench.committed_traffic("kNoSuchKernel") == (None, None)
    assert bench.committed_issue_slots("kNoSuchKernel") == (None, None, None)


def test_event_sets_option():
    assert bench.parse_args([]).sets == 2
    assert bench.parse_args(["--sets", "1"]).sets == 1
    with pytest.raises(SystemExit):
        bench.parse_args(["--sets", "5"])
