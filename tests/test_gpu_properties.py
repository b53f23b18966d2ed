"""Size-independent properties checked at the full benchmark sizes, where
the oracle would take too long: exact linearity in the sources, bitwise
determinism, the FP64 energy reduction, and the error of the FP32 precision
form against the FP64 form (pinned to the oracle at smaller sizes)."""
import numpy as np
import pytest
from conftest import rel_l2

pytestmark = pytest.mark.gpu


def scaled(case, factor):
    c = dict(case)
    f = dict(case["fields"])
    f["eta"] = f["eta"] * factor
    f["initial_I"] = f["initial_I"] * factor
    c["fields"] = f
    return c


@pytest.mark.parametrize("precision", [0, 1])
def test_linearity_in_emission_full_size(precision, grlbm, W):
    """The step is linear in (I, eta) for fixed opacities; scaling both by 2 is
    exact in binary floating point, so the state doubles bit for bit."""
    case = W.curved_scatter(steps=60)
    a = grlbm.run(case, precision)
    b = grlbm.run(scaled(case, 2.0), precision)
    for k in ("E", "Fx", "Fy", "I"):
        assert np.array_equal(2.0 * a[k], b[k]), k
    assert a["max_iterations"] == b["max_iterations"]


@pytest.mark.parametrize("precision", [0, 1])
def test_determinism_full_size(precision, grlbm, W):
    case = W.curved_shell(steps=100)
    a = grlbm.run(case, precision)
    b = grlbm.run(case, precision)
    for k in ("E", "Fx", "Fy", "I", "coefX"):
        assert np.array_equal(a[k], b[k]), k


def test_energy_reduction_fp64(grlbm, W):
    case = W.curved_shell(steps=50)
    res = grlbm.run(case)
    nx, ny = res["nx"], res["ny"]
    E = res["E"].reshape(ny, nx)[1:-1, 1:-1]
    assert abs(res["energy"] - E.sum()) <= 1e-12 * abs(E).sum()


@pytest.mark.parametrize("maker,steps", [("curved_shell", 1000), ("curved_scatter", 2000)])
def test_precision_form_error_full_size(maker, steps, grlbm, W):
    """FP32 intensities and stream/collide arithmetic with Kahan-compensated
    moments, on FP64 geodesic tables: relative L2 error <= 1e-5 on E and F
    against the FP64 form after the full run."""
    case = W.make_case(maker, steps=steps)
    ref = grlbm.run(case, 0)
    res = grlbm.run(case, 1)
    for k in ("E", "Fx", "Fy"):
        err = rel_l2(res[k], ref[k])
        assert err <= 1e-5, f"{k}: {err:.3e}"
    assert abs(res["energy"] - ref["energy"]) <= 1e-5 * abs(ref["energy"])


def test_precision_form_against_oracle(grlbm, W, oracle):
    case = W.curved_scatter(nx_=120, ny_=120, n_dir=32, n_fourier=9, steps=60)
    ref = oracle.run(case, "oracle")
    res = grlbm.run(case, 1)
    for k in ("E", "Fx", "Fy"):
        assert rel_l2(res[k], ref[k]) <= 1e-5, k
