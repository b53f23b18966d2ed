"""Frame output: the library's CSV writer (grlbm_host_write_frame_csv) against
the reference's own Grid::WriteFrametoCsv (src/Grid.cpp:110-137) compiled
from its sources, byte for byte -- file name (Format(time, 3)) and content,
for values of every magnitude, signed zeros, and several frame times."""
import ctypes as C
import os

import numpy as np
import pytest


def test_frame_files_are_byte_identical(grlbm, W, oracle, tmp_path):
    if not oracle.available("ref_strict"):
        pytest.skip("the reference build is absent")
    case = W.flat_beam(nx_=13, ny_=9, n_dir=8, steps=1)
    nxy = (case["nx_"] + 2) * (case["ny_"] + 2)
    rng = np.random.default_rng(3)
    arrs = [rng.normal(size=nxy) * 10.0 ** rng.integers(-12, 12, size=nxy) for _ in range(4)]
    arrs[0][:5] = [0.0, -0.0, 1.0, -1e-300, 123456789.0]
    g = grlbm.grid_desc(case)
    D = C.POINTER(C.c_double)
    for t in (0.0, 0.5, 1.2345678, 100.0, -0.25):
        ours, ref = tmp_path / "ours", tmp_path / "ref"
        ref.mkdir(exist_ok=True)
        rc = grlbm.lib().grlbm_host_write_frame_csv(C.byref(g), t, *[a.ctypes.data_as(D) for a in arrs],
                                                    (str(ours) + "/").encode(), b"frame")
        assert rc == 0, grlbm.lib().grlbm_last_error(None)
        oracle.write_frame("ref_strict", case, t, *arrs, str(ref) + "/", "frame")
        a, b = sorted(os.listdir(ours)), sorted(os.listdir(ref))
        assert a == b and len(a) >= 1
        for name in a:
            assert (ours / name).read_bytes() == (ref / name).read_bytes(), name
