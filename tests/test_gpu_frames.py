"""RunSimulation with frame output: grlbm_run_simulation against the
reference's own RunSimulation writing its CSV frames (initial, every write
period, final) for the flat beam, whose steps are bit-identical: the frame
files must match byte for byte, names included."""
import os

import pytest

pytestmark = pytest.mark.gpu


def test_run_simulation_frames_match_reference(grlbm, W, oracle, tmp_path):
    if not oracle.available("ref_strict"):
        pytest.skip("the reference build is absent")
    case = W.flat_beam(nx_=30, ny_=24, n_dir=12, steps=41)
    work = tmp_path / "ref" / "run"
    work.mkdir(parents=True)
    with grlbm.prepare(case) as r:
        dt = r.dt
        period = 7.5 * dt
        try:
            oracle.set_frames("ref_strict", period, str(work))
            oracle.run(case, "ref_strict", use_run_simulation=True)
        finally:
            oracle.set_frames("ref_strict", None, None)
        ours = tmp_path / "ours"
        steps = r.run_simulation((int(case["n_steps"]) - 0.5) * dt, period, str(ours) + "/")
    assert steps == int(case["n_steps"])
    ref_dir = tmp_path / "ref" / "output" / "ref_run" / "Moments"
    a, b = sorted(os.listdir(ours)), sorted(os.listdir(ref_dir))
    assert a == b and len(a) == 7  # initial, 5 periods, final
    for name in a:
        assert (ours / name).read_bytes() == (ref_dir / name).read_bytes(), name


@pytest.mark.parametrize("adaptive,precision", [(False, 0), (True, 0), (True, 1)])
def test_tables_rebuilt_every_step(grlbm, W, adaptive, precision):
    """Config::updateFourierHarmonics: with a static metric, rebuilding the
    tables before every step reproduces the tables-once run bit for bit (as
    it does in the reference); the table statistics show the rebuilds.  With
    CurvedAdaptive streaming the rebuild also refreshes the coefficient
    copies the adaptive stream reads (FP64 node-major, or FP32 about the node
    in the precision form)."""
    import numpy as np
    case = W.curved_shell(nx_=40, ny_=32, n_dir=16, n_fourier=5, steps=6)
    if adaptive:
        case["streaming_type"] = W.CURVED_ADAPTIVE
    with grlbm.prepare(case, precision) as a:
        a.step(6)
        Ea = a.moments_if()["E"]
    with grlbm.prepare(case, precision) as b:
        b.update_tables_each_step(True, case["rk_tol"])
        b.step(6)
        Eb = b.moments_if()["E"]
        assert b.stats()["table_ms"] > 0
    assert np.array_equal(Ea, Eb)


def test_adaptive_run_simulation_frames_match_reference(grlbm, W, oracle, tmp_path):
    """The same with FlatAdaptive streaming: the frames' moments use each
    node's rotated stencil, and the moments a frame computes feed the next
    rotation update, as in the reference."""
    if not oracle.available("ref_strict"):
        pytest.skip("the reference build is absent")
    case = W.flat_beam(nx_=30, ny_=24, n_dir=12, steps=23)
    case["streaming_type"] = W.FLAT_ADAPTIVE
    work = tmp_path / "ref" / "run"
    work.mkdir(parents=True)
    with grlbm.prepare(case) as r:
        period = 5.5 * r.dt
        try:
            oracle.set_frames("ref_strict", period, str(work))
            oracle.run(case, "ref_strict", use_run_simulation=True)
        finally:
            oracle.set_frames("ref_strict", None, None)
        ours = tmp_path / "ours"
        r.run_simulation((int(case["n_steps"]) - 0.5) * r.dt, period, str(ours) + "/")
    ref_dir = tmp_path / "ref" / "output" / "ref_run" / "Moments"
    a, b = sorted(os.listdir(ours)), sorted(os.listdir(ref_dir))
    assert a == b and len(a) >= 5
    for name in a:
        assert (ours / name).read_bytes() == (ref_dir / name).read_bytes(), name
