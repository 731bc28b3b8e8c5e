"""Bounded waits that run out reach the host as error words, without a GPU
fault: a test kernel polls an mbarrier that nothing completes (a short,
bounded poll count), records a timeout in the grid's error word and returns;
the host reads it (cn_grid_device_error), the synchronising entry points
return CN_ERR_DEVICE, and the context keeps working."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CN_ERR_DEVICE = 11


def _timeout(cn, g, polls=256):
    from cubismnova_b200 import _lib
    _lib.check(_lib.lib().cn_debug_wait_timeout(g.handle, polls, None))


def test_timeout_sets_the_error_word_and_clears(cn):
    g = cn.Grid.Cartesian((1, 1, 1), (8, 8, 8))
    assert g.device_error() == 0
    _timeout(cn, g)
    assert g.device_error(clear=False) == 1
    assert g.device_error() == 1  # read and clear
    assert g.device_error() == 0


def test_synchronising_stage_reports_the_error_then_recovers(cn):
    nb, n = (2, 2, 2), (16, 16, 16)
    U = cn.Grid.Cartesian(nb, n, ncomp=5)
    cn.workloads.euler_pulse(U)
    w1, w2 = cn.euler.like(U), cn.euler.like(U)
    dt = cn.euler.cfl_dt(U, 0.3)
    _timeout(cn, U)
    with pytest.raises(cn._lib.CnError) as e:
        cn.euler.rk3_stage(U, U, None, w1, 1, dt, want_sums=True)
    assert e.value.status == CN_ERR_DEVICE
    # the word was cleared by the failing call; the same stage now succeeds
    # and gives the result of a stage on a fresh copy of the state
    assert U.device_error() == 0
    s1 = cn.euler.rk3_stage(U, U, None, w1, 1, dt, want_sums=True)
    s2 = cn.euler.rk3_stage(U, U, None, w2, 1, dt, want_sums=True)
    assert np.array_equal(np.array(s1), np.array(s2))
    for c in range(5):
        assert np.array_equal(w1.download(c), w2.download(c))
    assert U.device_error() == 0
