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


def test_batch_replicas_deal_every_problem_once_and_balance(grlbm, W):
    """The multi-GPU batched form deals the 64 benchmark problems to the ranks
    as independent replicas: every problem exactly once, the same deal on
    every rank, and no rank's estimated cost above the lightest's by more
    than the costliest single problem."""
    cases = W.batch_instances(count=64, seed=10, steps=2)
    assert grlbm.share_problems(cases, 1) == [list(range(64))]
    for world in (2, 3, 4, 8):
        deal = grlbm.share_problems(cases, world)
        assert deal == grlbm.share_problems(cases, world)
        assert sorted(k for part in deal for k in part) == list(range(64))
        loads = [sum(grlbm.batch_cost(cases[k]) for k in part) for part in deal]
        assert max(loads) - min(loads) <= max(grlbm.batch_cost(c) for c in cases)
    with_more_ranks = grlbm.share_problems(cases[:3], 5)
    assert sorted(len(p) for p in with_more_ranks) == [0, 0, 1, 1, 1]


def test_batch_cost_orders_forms_as_measured(grlbm, W):
    """The cost model the batch's launch shares use: curved streaming above
    flat, and the forms in the order of their measured step times."""
    shell = W.curved_shell(nx_=40, ny_=40, n_dir=16, steps=2)
    flat = dict(shell, streaming_type=W.FLAT_FIXED)
    adaptive = dict(shell, streaming_type=W.CURVED_ADAPTIVE)
    c = grlbm.batch_cost
    assert c(shell) == 1.6 * c(flat) and c(shell) == 40 * 40 * 64 * 1.6
    assert c(shell) < c(shell, grlbm.FAST_FP64) < c(shell, grlbm.PLAIN_FP64) < c(adaptive, grlbm.PLAIN_FP64)
    assert c(adaptive) < c(adaptive, grlbm.PLAIN_FP64)
