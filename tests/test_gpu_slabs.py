"""Slab decomposition on one GPU: three contexts of the same problem, each
stepping one band of interior rows (grlbm_set_rows) and building the tables
of its band's cells only, exchange the rows next to their bands through
grlbm_copy_rows before every step -- the exchange a multi-GPU run does over
NCCL, here as device copies between contexts -- and step their bands in
parts (grlbm_step_rows_async: inner rows, then the edge rows, as a rank
does around its exchange).  The bands together must reproduce the
whole-grid run bit for bit, in every form: each cell's arithmetic is the
same, only where it runs differs."""
import importlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1, 2])
@pytest.mark.parametrize("maker,kw", [
    ("curved_scatter", dict(nx_=64, ny_=45, n_dir=16, n_fourier=9, steps=12)),
    ("moving_scatter", dict(nx_=40, ny_=33, n_dir=24, n_fourier=5, steps=10)),
    ("flat_beam", dict(nx_=50, ny_=31, n_dir=20, steps=15)),
])
def test_bands_reproduce_whole_grid(grlbm, W, precision, maker, kw):
    import torch
    S = importlib.import_module("2dradiation_b200.slabs")
    case = W.make_case(maker, **kw)
    steps = int(case["n_steps"])
    with grlbm.prepare(case, precision) as whole:
        whole.step(steps)
        ref = whole.moments_if()
        refI = whole.intensity().reshape(whole.nxy, whole.nd)
        ref_energy = whole.energy()
    world = 3
    bands = S.partition(int(case["ny_"]), world)
    rads = [grlbm.prepare(case, precision, rows=b) for b in bands]
    try:
        g = max(r.departure_rows() for r in rads)
        assert 1 <= g <= min(b - a for a, b in bands)
        dtype = torch.float32 if precision == 1 else torch.float64
        buf = torch.empty(g * rads[0].row_bytes() // dtype.itemsize, dtype=dtype, device="cuda")
        for _ in range(steps):
            for k in range(world - 1):
                lo_of_next = bands[k + 1][0]
                # rank k's top rows -> rank k+1's lower ghost rows
                rads[k].copy_rows(lo_of_next - g, g, buf.data_ptr(), True)
                rads[k].sync()
                rads[k + 1].copy_rows(lo_of_next - g, g, buf.data_ptr(), False)
                rads[k + 1].sync()
                # rank k+1's bottom rows -> rank k's upper ghost rows
                rads[k + 1].copy_rows(lo_of_next, g, buf.data_ptr(), True)
                rads[k + 1].sync()
                rads[k].copy_rows(lo_of_next, g, buf.data_ptr(), False)
                rads[k].sync()
            for r, (lo, hi) in zip(rads, bands):
                parts = [(lo + g, hi - g), (lo, min(lo + g, hi)), (max(hi - g, lo + g), hi)]
                for a, b in parts:
                    if a < b:
                        r.step_rows_async(a, b, False)
                r.step_rows_async(hi, hi, True)
                r.sync()
        nx = rads[0].nx
        for r, (lo, hi) in zip(rads, bands):
            m = r.moments_if()
            I = r.intensity().reshape(r.nxy, r.nd)
            rows = slice(lo * nx, hi * nx)
            for k in ("E", "Fx", "Fy", "Pxx", "Pxy", "Pyy"):
                assert np.array_equal(m[k][rows], ref[k][rows]), (k, lo, hi)
            assert np.array_equal(I[rows], refI[rows])
        # the bands' energies (grlbm_energy over each band) add up to the whole grid's
        total = sum(r.energy() for r in rads)
        assert abs(total - ref_energy) <= 1e-12 * abs(ref_energy)
    finally:
        for r in rads:
            r.close()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("maker,kw,kind", [
    ("curved_scatter", dict(nx_=48, ny_=40, n_dir=16, n_fourier=9, steps=10), "curved"),
    ("moving_scatter", dict(nx_=36, ny_=31, n_dir=24, n_fourier=5, steps=8), "curved"),
    ("flat_beam", dict(nx_=40, ny_=31, n_dir=20, steps=12), "flat"),
])
def test_adaptive_bands_reproduce_whole_grid(grlbm, W, precision, maker, kw, kind):
    """Adaptive streaming in bands (plain and precision forms): before every
    step the three contexts exchange, besides the intensities' ghost rows,
    those rows' rotation angles and the moment row next to each band
    (grlbm_copy_node_rows), then step their bands whole.  The bands together
    reproduce the whole-grid run bit for bit."""
    import torch
    S = importlib.import_module("2dradiation_b200.slabs")
    case = dict(W.make_case(maker, **kw),
                streaming_type=W.CURVED_ADAPTIVE if kind == "curved" else W.FLAT_ADAPTIVE)
    steps = int(case["n_steps"])
    with grlbm.prepare(case, precision) as whole:
        whole.step(steps)
        ref = whole.moments_if()
        refI = whole.intensity()
    world = 3
    bands = S.partition(int(case["ny_"]), world)
    rads = [grlbm.prepare(case, precision, rows=b) for b in bands]
    try:
        g = max(r.departure_rows() for r in rads)
        assert 1 <= g <= min(b - a for a, b in bands)
        dtype = torch.float32 if precision == 1 else torch.float64
        fields = [(None, g, rads[0].row_bytes()), (grlbm.ROWS_ANGLES, g, rads[0].node_row_bytes(grlbm.ROWS_ANGLES)),
                  (grlbm.ROWS_MOMENTS, 1, rads[0].node_row_bytes(grlbm.ROWS_MOMENTS))]
        buf = torch.empty(max(rows * nb for _, rows, nb in fields) // 4, dtype=torch.float32, device="cuda")

        def copy(r, what, j, n, to_buffer):
            if what is None:
                r.copy_rows(j, n, buf.data_ptr(), to_buffer)
            else:
                r.copy_node_rows(what, j, n, buf.data_ptr(), to_buffer)
            r.sync()

        for _ in range(steps):
            for k in range(world - 1):
                lo_next = bands[k + 1][0]
                for what, rows, _ in fields:
                    copy(rads[k], what, lo_next - rows, rows, True)   # rank k's top rows
                    copy(rads[k + 1], what, lo_next - rows, rows, False)
                    copy(rads[k + 1], what, lo_next, rows, True)      # rank k+1's bottom rows
                    copy(rads[k], what, lo_next, rows, False)
            for r in rads:
                r.step_async(1)
                r.sync()
        nx = rads[0].nx
        for r, (lo, hi) in zip(rads, bands):
            m = r.moments_if()
            rows = slice(lo * nx, hi * nx)
            for q in ("E", "Fx", "Fy", "Pxx", "Pxy", "Pyy"):
                assert np.array_equal(m[q][rows], ref[q][rows]), (q, lo, hi)
            I = r.intensity().reshape(r.nxy, r.nd)
            assert np.array_equal(I[rows], refI.reshape(r.nxy, r.nd)[rows])
    finally:
        for r in rads:
            r.close()


def test_band_tables_cover_the_band_only(grlbm, W):
    """Tables built for one band do not serve a wider one: stepping it is
    refused until they are rebuilt."""
    case = W.make_case("curved_shell", nx_=32, ny_=30, n_dir=12, n_fourier=5, steps=2)
    with grlbm.prepare(case, 1, rows=(5, 12)) as r:
        r.step(1)
        r.set_rows(1, 31)
        with pytest.raises(grlbm.GrlbmError) as e:
            r.step(1)
        assert e.value.code == 3
        r.update_fourier_coefficients(case["rk_tol"])
        r.step(1)
