"""The bounded device-side waits of the row pipeline, driven to their limit without a fault.

lbm_test_stall_next_step makes the producer of the next step's launch leave one work item's stage
unfilled (no copy is issued for it, so nothing is in flight and nothing can fault) and gives every
mbarrier wait of that launch a ~1 ms limit.  The consumers waiting for that stage time out, then the
producer; the launch returns, lbm_sync reports LBM_ERR_TIMEOUT once and clears the error word, and the
context stays usable: re-set populations step on and match the oracle."""
import numpy as np
import pytest

from helpers import O, cavity3d, channel2d, lb, mrt_cavity, oracle_problem, rel_l2

pytestmark = pytest.mark.gpu

TIMEOUT = -8


def _stalled_then_clean(d, m, F0, steps, item=0, storage=None):
    if storage is not None:
        d.storage = storage
    with lb.Lattice(d, m) as lat:
        lat.set_kernel(lb.KERNEL_ROWS)
        lat.set_populations(F0)
        lat.step(1)  # prepares the row pipeline (and checks a clean step first)
        assert lb.lib().lbm_sync(lat._h) == 0
        lat.test_stall_next_step(item=item, wait_clocks=1 << 21)
        lat.set_populations(F0)
        lat.step(3)  # the first launch stalls, the next two run normally
        rc = lb.lib().lbm_sync(lat._h)
        assert rc == TIMEOUT, rc
        assert b"row-pipeline wait" in lb.lib().lbm_last_error()
        assert lb.lib().lbm_sync(lat._h) == 0  # the error word was cleared
        # the context is still usable: a clean run from F0 matches the oracle
        lat.set_populations(F0)
        lat.step(steps)
        assert lb.lib().lbm_sync(lat._h) == 0
        return lat.get_populations(np.float64)


def test_stalled_stage_times_out_and_the_context_recovers_mrt():
    d, m, F0 = mrt_cavity(n=32, u_lid=0.05, basis=lb.MRT_GRAM_SCHMIDT)
    F = _stalled_then_clean(d, m, F0, 40)
    Fo, _, _ = O.run(oracle_problem(d, m), F0, 40)
    assert rel_l2(F, Fo) < 1e-5


def test_stalled_late_item_times_out_bgk3d():
    # an item of a later round of the persistent CTAs (the producer has issued earlier stages)
    d, m, F0 = cavity3d(n=(64, 48, 40), u_lid=0.1, omega=1.3)
    F = _stalled_then_clean(d, m, F0, 20, item=300)
    Fo, _, _ = O.run(oracle_problem(d, m), F0, 20)
    assert rel_l2(F, Fo) < 1e-5


def test_stalled_row_segment_times_out_d2q9():
    # rows wider than 1024 cells: the segmented kernel
    d, m, F0 = channel2d(2048, 40, 0.05, 100.0, 300, 20, 6, config_mode=True, seed=1, noise=1e-4)
    F = _stalled_then_clean(d, m, F0, 30, item=5, storage=lb.F16S)
    d64, m64, _ = channel2d(2048, 40, 0.05, 100.0, 300, 20, 6, config_mode=True, seed=1, noise=1e-4,
                            storage=lb.F64)
    with lb.Lattice(d64, m64) as lat:
        lat.set_populations(F0)
        lat.step(30)
        F64 = lat.get_populations(np.float64)
    assert rel_l2(F, F64) < 1e-3


def test_stall_needs_the_row_pipeline_and_sane_limits():
    d, m, F0 = cavity3d(n=(32, 32, 32))
    with lb.Lattice(d, m) as lat:
        with pytest.raises(lb.LbmError) as e:
            lat.test_stall_next_step(0, 1 << 21)  # AUTO family: not pinned to the row pipeline
        assert e.value.code == -7
        lat.set_kernel(lb.KERNEL_ROWS)
        with pytest.raises(lb.LbmError):
            lat.test_stall_next_step(0, 10)  # below 2^10 clocks
        with pytest.raises(lb.LbmError):
            lat.test_stall_next_step(-1, 1 << 21)
