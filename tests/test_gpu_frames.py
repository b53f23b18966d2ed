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


def test_run_log_and_trace_match_reference(grlbm, W, oracle, tmp_path):
    """grlbm_write_log after grlbm_run_simulation against the Log.txt of the
    reference's own RunSimulation on the same flat beam (bit-identical
    steps): every line but the date and the timings is the same, the lambda
    iteration counts included.  A profile session around the run writes the
    reference profiler's Chrome-trace JSON, with the same event keys as the
    reference's own profileResults.json."""
    import json
    if not oracle.available("ref_strict"):
        pytest.skip("the reference build is absent")
    case = W.flat_beam(nx_=30, ny_=24, n_dir=12, steps=41)
    work = tmp_path / "ref" / "run"
    (work / "output" / "ref_run").mkdir(parents=True)  # where the reference's profiler writes
    with grlbm.prepare(case) as r:
        dt = r.dt
        try:
            oracle.set_frames("ref_strict", 7.5 * dt, str(work))
            oracle.run(case, "ref_strict", use_run_simulation=True)
        finally:
            oracle.set_frames("ref_strict", None, None)
        r.trace_begin(str(tmp_path / "ours" / "profileResults.json"))
        r.run_simulation((int(case["n_steps"]) - 0.5) * dt, 7.5 * dt, str(tmp_path / "ours" / "Moments") + "/")
        r.trace_end()
        r.write_log(str(tmp_path / "ours"))
    ref = (tmp_path / "ref" / "output" / "ref_run" / "Log.txt").read_text().splitlines()
    ours = (tmp_path / "ours" / "Log.txt").read_text().splitlines()
    timed = ("Creation Date", "Computation Time", "Benchmark")

    def fixed(lines):
        out, in_times = [], False
        for ln in lines:
            if ln == "Time measurements:":
                in_times = True
            elif ln.startswith("Computation Time"):
                in_times = False
            if not in_times and not ln.startswith(timed):
                out.append(ln)
        return out
    assert fixed(ours) == fixed(ref)
    assert any(ln.startswith("Total Time: ") for ln in ours)
    trace = json.loads((tmp_path / "ours" / "profileResults.json").read_text())
    ev = trace["traceEvents"]
    names = {e["name"] for e in ev}
    assert "Total Time" in names and any("WriteFrametoCsv" in n for n in names)
    assert all(e["dur"] >= 0 and e["ph"] == "X" and e["pid"] == 0 for e in ev)
    ref_json = work / "output" / "ref_run" / "profileResults.json"
    if ref_json.exists():
        rev = json.loads(ref_json.read_text())
        assert set(rev) == set(trace)
        assert {k for e in rev["traceEvents"] for k in e} == {k for e in ev for k in e}


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


@pytest.mark.parametrize("adaptive", [False, True])
def test_tables_rebuilt_every_step_match_reference(grlbm, W, oracle, adaptive):
    """Config::updateFourierHarmonics against the reference run with the same
    option (its own driver calls UpdateFourierCoefficients at the top of every
    step, src/Radiation.cpp:790-791): the plain form's moments and
    intensities within 1e-12 (the tables agree to 1e-13, not bit for bit:
    the reference's step-size control uses libm's pow), on a workload whose
    result is stable under last-bit changes (no scattering)."""
    import numpy as np
    if not oracle.available("ref_strict"):
        pytest.skip("the reference build is absent")
    case = W.curved_shell(nx_=40, ny_=32, n_dir=16, n_fourier=5, steps=6)
    if adaptive:
        case["streaming_type"] = W.CURVED_ADAPTIVE
    ref = oracle.run(case, "ref_strict", update_tables_each_step=True)
    with grlbm.prepare(case, 0) as r:
        r.update_tables_each_step(True, case["rk_tol"])
        r.step(6)
        m = r.moments_if()
        I = r.intensity()
    for k in ("E", "Fx", "Fy"):
        err = np.linalg.norm(m[k] - ref[k]) / np.linalg.norm(ref[k])
        assert err <= 1e-12, (k, err)
    assert np.linalg.norm(I - ref["I"]) <= 1e-12 * np.linalg.norm(ref["I"])


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
