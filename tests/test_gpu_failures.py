"""Failure paths on the GPU, made on the host or by bounded device loops:
nothing here faults, traps or hangs a GPU."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_step_before_tables_is_a_state_error(grlbm, W):
    case = W.curved_shell(nx_=16, ny_=16, n_dir=8, steps=1)
    with grlbm.Radiation(case) as r:
        with pytest.raises(grlbm.GrlbmError) as e:
            r.step(1)
        assert e.value.code == 3


def test_rk45_substep_cap_reports_and_context_survives(grlbm, W):
    """A backtrace that exceeds max_substeps stops, is counted, and the call
    returns GRLBM_ERR_NONCONVERGED after finishing the others; a rebuild with
    the normal cap then works on the same context."""
    case = W.curved_shell(nx_=24, ny_=24, n_dir=16, steps=2)
    with grlbm.Radiation(case) as r:
        r.set_fields(case["fields"])
        with pytest.raises(grlbm.GrlbmError) as e:
            r.update_fourier_coefficients(1e-12, max_substeps=1)
        assert e.value.code == 5
        assert r.stats()["rk_nonconverged"] > 0
        r.update_fourier_coefficients(case["rk_tol"])
        assert r.stats()["rk_nonconverged"] == 0
        r.step(2)
        assert np.isfinite(r.moments_if()["E"]).all()


def test_bad_host_arguments(grlbm, W):
    case = W.curved_shell(nx_=8, ny_=8, n_dir=8, steps=1)
    with grlbm.Radiation(case) as r:
        import ctypes as C
        assert grlbm.lib().grlbm_set_intensity(r.h, None) == 1
        assert grlbm.lib().grlbm_step(r.h, -1) == 1
        assert grlbm.lib().grlbm_update_fourier_coefficients(r.h, -1.0, 0) == 1
        assert "rk_tol" in grlbm.lib().grlbm_last_error(r.h).decode()


def test_staging_wait_runs_out_and_returns(grlbm, W):
    """The precision step's staging wait has a time limit: a wait on an
    mbarrier phase that nothing completes returns after the limit (and the
    context stays usable); with one arrival it returns at once."""
    out = grlbm.selftest_staging_wait(arrive=False, limit_us=2000)
    assert out["completed"] is False
    assert 2000 <= out["waited_us"] < 1e6
    out = grlbm.selftest_staging_wait(arrive=True, limit_us=2000)
    assert out["completed"] is True and out["waited_us"] < 2000
    case = W.curved_shell(nx_=24, ny_=24, n_dir=16, n_fourier=5, steps=2)
    res = grlbm.run(case, 1)
    assert np.isfinite(res["E"]).all()
    with pytest.raises(grlbm.GrlbmError) as e:
        grlbm.selftest_staging_wait(arrive=False, limit_us=0)
    assert e.value.code == 1
