"""Adaptive streaming (FlatAdaptive, CurvedAdaptive; src/Radiation.cpp:361-378,
415-452, 513-575) against the reference itself, compiled from its sources
(the oracle's C restatement covers the fixed types only):

- flat adaptive streaming, with a beam of intensities and with von Mises
  moment sources in a moving, anisotropically scattering fluid, is
  bit-identical -- the stencil rotations use the reference's polynomial
  trigonometry, which the library reproduces exactly;
- curved adaptive streaming evaluates the Fourier series of the geodesic
  tables at run-time angles with the GPU's cos/sin instead of the C
  library's, so it matches within 1e-11 (tables taken from the reference).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


def run_ours(grlbm, case, ref=None):
    with grlbm.Radiation(case, grlbm.PLAIN_FP64) as r:
        r.set_fields(case["fields"])
        r.set_initial_data(case["fields"])
        r.load_initial_data()
        if ref is not None:
            r.set_coefficients(ref)
        else:
            r.update_fourier_coefficients(case["rk_tol"])
        r.step(int(case["n_steps"]))
        out = dict(r.moments_if())
        out["I"] = r.intensity()
    return out


def flat_cases(W):
    beam = W.flat_beam(nx_=40, ny_=30, n_dir=16, steps=25)
    beam["streaming_type"] = W.FLAT_ADAPTIVE
    moving = W.moving_scatter(nx_=30, ny_=26, n_dir=20, steps=12, metric_kind=W.MINKOWSKI,
                              streaming_type=W.FLAT_ADAPTIVE)
    return [beam, moving]


@pytest.mark.parametrize("k", [0, 1])
def test_flat_adaptive_is_bit_identical(grlbm, W, oracle, k):
    if not oracle.available("ref_strict"):
        pytest.skip("the reference build is absent")
    case = flat_cases(W)[k]
    ref = oracle.run(case, "ref_strict")
    ours = run_ours(grlbm, case)
    for key in ("E", "Fx", "Fy", "Pxx", "Pxy", "Pyy", "I"):
        assert np.array_equal(ours[key], ref[key]), (key, rel_l2(ours[key], ref[key]))


@pytest.mark.parametrize("kw", [
    dict(nx_=40, ny_=36, n_dir=16, n_fourier=5, steps=20),
    dict(nx_=37, ny_=23, n_dir=12, n_fourier=64, steps=10),  # ragged rows, 12 directions, the largest Fourier order
])
def test_curved_adaptive_matches_reference(grlbm, W, oracle, kw):
    if not oracle.available("ref_strict"):
        pytest.skip("the reference build is absent")
    case = W.curved_shell(**kw)
    case["streaming_type"] = W.CURVED_ADAPTIVE
    ref = oracle.run(case, "ref_strict")
    ours = run_ours(grlbm, case, ref)
    for key in ("E", "Fx", "Fy"):
        assert rel_l2(ours[key], ref[key]) <= 1e-11, (key, rel_l2(ours[key], ref[key]))


def precision_cases(W):
    """Adaptive cases for the precision form: the flat beam, a moving
    anisotropically scattering fluid (flat and curved), and curved shells
    (the second with ragged rows, 12 directions and the largest Fourier
    order)."""
    beam = W.flat_beam(nx_=40, ny_=30, n_dir=16, steps=25)
    beam["streaming_type"] = W.FLAT_ADAPTIVE
    shell = W.curved_shell(nx_=48, ny_=40, n_dir=24, n_fourier=7, steps=20)
    shell["streaming_type"] = W.CURVED_ADAPTIVE
    wide = W.curved_shell(nx_=37, ny_=23, n_dir=12, n_fourier=64, steps=10)
    wide["streaming_type"] = W.CURVED_ADAPTIVE
    return [beam,
            W.moving_scatter(nx_=30, ny_=26, n_dir=20, steps=12, metric_kind=W.MINKOWSKI,
                             streaming_type=W.FLAT_ADAPTIVE),
            W.moving_scatter(nx_=30, ny_=26, n_dir=20, steps=12, streaming_type=W.CURVED_ADAPTIVE),
            shell, wide]


@pytest.mark.parametrize("k", [0, 1, 2, 3, 4])
def test_precision_form_adaptive_against_plain(grlbm, W, k):
    """Adaptive streaming in the precision form (FP32 stream and moment-space
    collide, FP32 Fourier basis) against the plain form on the same tables:
    the precision form's tolerance."""
    case = precision_cases(W)[k]
    ref = grlbm.run(case, grlbm.PLAIN_FP64)
    res = grlbm.run(case, grlbm.PRECISION_FP32)
    for key in ("E", "Fx", "Fy"):
        assert rel_l2(res[key], ref[key]) <= 2e-5, (key, rel_l2(res[key], ref[key]))


def test_precision_form_adaptive_from_set_coefficients(grlbm, W):
    """Coefficients handed in through grlbm_set_fourier_coefficients (as a
    caller of the reference may set coefficientsS/X/Y/Cx/Cy) feed the
    precision form's FP32 copy as well: the same run as with the tables built
    in place, within the precision form's tolerance of the plain form."""
    case = W.curved_shell(nx_=37, ny_=23, n_dir=12, n_fourier=7, steps=10)
    case["streaming_type"] = W.CURVED_ADAPTIVE
    with grlbm.prepare(case, grlbm.PLAIN_FP64) as p:
        coef = p.coefficients()
        p.step(int(case["n_steps"]))
        ref = dict(p.moments_if())
    with grlbm.Radiation(case, grlbm.PRECISION_FP32) as r:
        r.set_fields(case["fields"])
        r.set_initial_data(case["fields"])
        r.load_initial_data()
        r.set_coefficients(coef)
        r.step(int(case["n_steps"]))
        res = dict(r.moments_if())
    for key in ("E", "Fx", "Fy"):
        assert rel_l2(res[key], ref[key]) <= 2e-5, (key, rel_l2(res[key], ref[key]))
