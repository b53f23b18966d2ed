"""Seeded input generation shared by every side of the parity tests."""
import numpy as np


def test_splitmix64_known_answers(W):
    # reference values of splitmix64 from state 0 (Steele, Lea & Flood 2014)
    z = W.splitmix64(0, 3)
    assert [int(v) for v in z] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_uniform_and_normal_ranges(W):
    u = W.uniform(5, 100000)
    assert u.min() >= 0.0 and u.max() < 1.0 and abs(u.mean() - 0.5) < 0.01
    z = W.normal(5, 100000)
    assert abs(z.mean()) < 0.02 and abs(z.std() - 1.0) < 0.02


def test_benchmark_workload_shapes(W):
    c = W.flat_beam()
    assert (c["nx_"], c["ny_"], c["n_dir"], c["n_steps"]) == (100, 100, 20, 500)
    c = W.curved_shell(steps=1)
    assert (c["nx_"], c["n_dir"], c["n_fourier"], c["n_steps"], c["excision"], c["rk_tol"]) == (200, 32, 5, 1, 2.4, 1e-10)
    c = W.curved_scatter(nx_=40, ny_=40, steps=1)
    f = c["fields"]
    assert f["kappa0"].min() >= 0 and f["kappa0"].max() <= 2
    assert np.all(f["kappaA"] > 0)


def test_grid_coordinates_follow_reference(W):
    X, Y, dx, dy = W.grid_coords(100, 100, (-1, -1), (1, 1))
    # x(i) = (start - dx) + i*dx (src/Grid.cpp:20, 48-51): not exactly -1 at i = 1
    assert dx == 2.0 / 99 and X[1] == (-1.0 - dx) + 1.0 * dx and Y[(100 + 2) * 1] == (-1.0 - dy) + dy
