"""Parity of the CUDA path (through the C-ABI) with the reference: the plain
FP64 form must match to relative L2 <= 1e-12 on E and F (and every other
output), on the golden vectors and, at larger sizes, on the oracle."""
import numpy as np
import pytest
from conftest import GOLDEN_NAMES, rel_l2

pytestmark = pytest.mark.gpu
TOL = 1e-12
MOMENTS = ("E", "Fx", "Fy", "Pxx", "Pxy", "Pyy")
LF = ("E_LF", "Fx_LF", "Fy_LF", "Pxx_LF", "Pxy_LF", "Pyy_LF", "F_LF")
COEF = ("coefS", "coefX", "coefY", "coefCx", "coefCy")


def check(res, ref, keys, tol=TOL):
    for k in keys:
        err = rel_l2(res[k], ref[k])
        assert err <= tol, f"{k}: rel L2 {err:.3e} > {tol:g}"


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_plain_fp64_matches_reference_golden(name, grlbm, cases, golden):
    g = golden(name)
    ref = {k[len("ref_strict_"):]: v for k, v in g.items() if k.startswith("ref_strict_")}
    res = grlbm.run(cases[name])
    check(res, ref, MOMENTS + LF + ("I",) + COEF)
    assert res["max_iterations"] == int(ref["max_iterations"])
    assert abs(res["average_iterations"] - float(ref["average_iterations"])) < 1e-12


@pytest.mark.parametrize("maker,kw,steps", [
    ("curved_shell", dict(nx_=200, ny_=200, n_dir=32, n_fourier=5), 40),
    ("curved_scatter", dict(nx_=160, ny_=160, n_dir=64, n_fourier=16), 20),
    ("flat_beam", dict(nx_=100, ny_=100, n_dir=20), 500),
])
def test_plain_fp64_matches_oracle_at_scale(maker, kw, steps, grlbm, W, oracle):
    case = W.make_case(maker, steps=steps, **kw)
    ref = oracle.run(case, "oracle")
    res = grlbm.run(case)
    check(res, ref, MOMENTS + ("I",) + LF + COEF)
    assert res["max_iterations"] == ref["max_iterations"]


@pytest.mark.parametrize("kw", [
    dict(nx_=37, ny_=23, n_dir=12, n_fourier=5),      # ragged interior, partial blocks
    dict(nx_=2, ny_=2, n_dir=8, n_fourier=3),         # smallest grid
    dict(nx_=30, ny_=18, n_dir=200, n_fourier=7),     # widest FP64 stencil (200 KB shared memory)
    dict(nx_=21, ny_=21, n_dir=64, n_fourier=32),     # many harmonics
])
def test_edge_shapes_match_oracle(kw, grlbm, W, oracle):
    case = W.curved_scatter(steps=5, **kw)
    ref = oracle.run(case, "oracle")
    res = grlbm.run(case)
    check(res, ref, MOMENTS + ("I",) + COEF)


def test_chunked_steps_equal_single_steps(grlbm, W):
    """Graph-replayed chunks of steps give the same state as one launch per step."""
    case = W.curved_scatter(nx_=40, ny_=40, n_dir=16, n_fourier=5, steps=70)
    with grlbm.prepare(case) as a, grlbm.prepare(case) as b:
        a.step(70)
        for _ in range(70):
            b.step(1)
        assert np.array_equal(a.intensity(), b.intensity())
        ma, mb = a.moments_if(), b.moments_if()
        for k in MOMENTS:
            assert np.array_equal(ma[k], mb[k])
