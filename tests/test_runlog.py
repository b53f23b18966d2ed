"""Log.txt (Logger::Write, src/Logger.hh:48-97) without a GPU: the library's
writer (grlbm_host_write_log) against the file the reference's own
RunSimulation writes, compiled from its sources, for the same values --
line for line, except the two figures the reference derives from its
unrounded timings (computation time and MLUPS), which agree to the printed
digits."""
import re

import pytest


def parse_log(text):
    lines = text.splitlines()
    date = lines[0].split(": ", 1)[1]
    times, it = [], {}
    in_times = False
    for ln in lines:
        if ln.startswith("Max Lambda Itteration Count"):
            it["max"] = int(ln.split("=")[1])
        elif ln.startswith("Average Lambda Itteration Count"):
            it["avg"] = float(ln.split("=")[1])
        elif ln.startswith("Nt"):
            it["nt"] = int(ln.split("=")[1])
        elif ln == "Time measurements:":
            in_times = True
        elif ln.startswith("Computation Time"):
            in_times = False
        elif in_times and ln.endswith("s") and ": " in ln:
            name, val = ln.rsplit(": ", 1)
            times.append((name, float(val[:-1])))
    return date, times, it, lines


def figure(line):
    return float(re.findall(r"[-+0-9.eE]+", line.split(": ", 1)[1])[0])


@pytest.mark.parametrize("maker,kw", [
    ("flat_beam", dict(nx_=20, ny_=16, n_dir=12, steps=9)),
    ("curved_shell", dict(nx_=18, ny_=18, n_dir=16, n_fourier=5, steps=4)),
])
def test_log_file_matches_reference(grlbm, W, oracle, tmp_path, maker, kw):
    if not oracle.available("ref_strict"):
        pytest.skip("the reference build is absent")
    case = W.make_case(maker, **kw)
    work = tmp_path / "ref" / "run"
    work.mkdir(parents=True)
    try:
        oracle.set_frames("ref_strict", 1e9, str(work))
        oracle.run(case, "ref_strict", use_run_simulation=True)
    finally:
        oracle.set_frames("ref_strict", None, None)
    ref_text = (tmp_path / "ref" / "output" / "ref_run" / "Log.txt").read_text()
    date, times, it, ref_lines = parse_log(ref_text)
    assert any(n == "Total Time" for n, _ in times)
    grlbm.host_write_log(case, date, it["nt"], it["max"], it["avg"], times, str(tmp_path / "ours"))
    ours = (tmp_path / "ours" / "Log.txt").read_text().splitlines()
    assert len(ours) == len(ref_lines)
    for a, b in zip(ours, ref_lines):
        if a.startswith(("Computation Time", "Benchmark")):
            assert a.split(":")[0] == b.split(":")[0]
            assert abs(figure(a) - figure(b)) <= 1e-5 * abs(figure(b)), (a, b)
        else:
            assert a == b
