"""Batched steps (grlbm_batch_*): problems of different forms, grid sizes,
direction counts and streaming types advanced together -- by one persistent
launch per step (FP32 fixed streaming) or by their own steps launched
concurrently -- must each match their single-problem run bit for bit, across
graph-replayed and single steps, after autotuning (which must leave every
problem as it was), and when a problem is also stepped on its own between
batch steps."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_batch_matches_single_problems(grlbm, W):
    cases = W.batch_instances(count=7, seed=12, sizes=(24, 37, 64), dirs=(8, 16, 32), steps=40)
    assert len({c["n_dir"] for c in cases}) > 1 and len({c["streaming_type"] for c in cases}) > 1
    P = grlbm.PRECISION_FP32
    ref = []
    for k, c in enumerate(cases):
        with grlbm.prepare(c, P) as r:
            r.step(37 + 6 + (1 if k == 0 else 0))
            ref.append((r.moments_if()["E"], r.intensity(), r.stats()["average_iterations"]))
    probs = [grlbm.prepare(c, P) for c in cases]
    try:
        with grlbm.Batch(probs) as b:
            choice = b.autotune(3)
            assert -8 <= choice["blocks_per_sm"]
            b.step(37)          # one 32-step graph and 5 single launches
            probs[0].step(1)    # a problem stepped on its own in between
            b.step(6)
        for k, (r, (E, I, it)) in enumerate(zip(probs, ref)):
            assert np.array_equal(r.moments_if()["E"], E), k
            assert np.array_equal(r.intensity(), I), k
            assert r.stats()["average_iterations"] == it, k
    finally:
        for r in probs:
            r.close()


@pytest.mark.parametrize("shape", [(0, True), (-1, True), (-3, False), (1, False), (5, True)])
def test_batch_shapes_match_single_problems(grlbm, W, shape):
    """Each launch shape, set explicitly: the concurrent launches on the
    problems' own grids (0) and on shares of one and three GPUs' worth of
    resident blocks (-1, -3), and the persistent launch at 1 and 5 blocks per
    SM (capped at the occupancy limit); -9 is refused."""
    cases = W.batch_instances(count=5, seed=21, sizes=(24, 37, 64), dirs=(8, 16, 32), steps=40)
    P = grlbm.PRECISION_FP32
    ref = []
    for c in cases:
        with grlbm.prepare(c, P) as r:
            r.step(35)
            ref.append(r.intensity())
    probs = [grlbm.prepare(c, P) for c in cases]
    try:
        with grlbm.Batch(probs) as b:
            bps, lf = shape
            try:
                b.set_shape(bps, lf)
            except grlbm.GrlbmError:
                assert bps > 1  # above this kernel's occupancy limit
                b.set_shape(1, lf)
            b.step(35)  # one 32-step graph and 3 single steps
            with pytest.raises(grlbm.GrlbmError) as e:
                b.set_shape(-9, True)
            assert e.value.code == 1
        for k, (r, I) in enumerate(zip(probs, ref)):
            assert np.array_equal(r.intensity(), I), k
    finally:
        for r in probs:
            r.close()


def _mixed_cases(grlbm, W):
    """One small problem of every form and streaming type, and beams that keep
    their source nodes active: (case, precision) pairs."""
    P32, P64, F64 = grlbm.PRECISION_FP32, grlbm.PLAIN_FP64, grlbm.FAST_FP64
    shell = W.curved_shell(nx_=30, ny_=26, n_dir=12, n_fourier=5, steps=40)
    flat = next(c for c in W.batch_instances(count=8, seed=3, sizes=(24,), dirs=(8,), steps=40)
                if c["streaming_type"] == W.FLAT_FIXED)
    beam = W.flat_beam(nx_=20, ny_=18, n_dir=8, steps=40)
    shell_ad, flat_ad = dict(shell), dict(flat)
    shell_ad["streaming_type"] = W.CURVED_ADAPTIVE
    flat_ad["streaming_type"] = W.FLAT_ADAPTIVE
    return [(shell, P32), (flat, P32), (shell_ad, P32), (flat_ad, P64), (shell, P64), (shell, F64), (beam, P32),
            (beam, F64), (flat, F64)]


def test_mixed_batch_matches_single_problems(grlbm, W):
    """Problems of every form in one batch -- FP32 fixed streaming (flat and
    curved), FP32 and plain FP64 adaptive streaming, plain and fast FP64 fixed
    streaming, and beams that keep their source nodes active -- each
    bit-identical to its own run: in the default shape, after autotuning
    (which must leave every problem as it was) across a 32-step graph, and on
    the problems' own grids.  The persistent launch is refused for such a
    batch (GRLBM_ERR_UNSUPPORTED), and so is a problem that rebuilds its
    tables every step."""
    cases = _mixed_cases(grlbm, W)
    ref = []
    for c, P in cases:
        with grlbm.prepare(c, P) as r:
            r.step(40)
            ref.append((r.moments_if()["E"], r.intensity(), r.stats()["average_iterations"]))
    probs = [grlbm.prepare(c, P) for c, P in cases]
    try:
        with grlbm.Batch(probs) as b:
            b.step(5)               # the default shape: concurrent launches on shares
            choice = b.autotune(3)
            assert -8 <= choice["blocks_per_sm"] <= 0
            b.step(32)              # one 32-step graph
            with pytest.raises(grlbm.GrlbmError) as e:
                b.set_shape(1, True)
            assert e.value.code == 4
            b.set_shape(0, True)
            b.step(3)
        for k, (r, (E, I, it)) in enumerate(zip(probs, ref)):
            assert np.array_equal(r.moments_if()["E"], E), k
            assert np.array_equal(r.intensity(), I), k
            assert r.stats()["average_iterations"] == it, k
    finally:
        for r in probs:
            r.close()
    c, P = cases[4]
    with grlbm.prepare(c, P) as r:
        r.update_tables_each_step(True, c["rk_tol"])
        with pytest.raises(grlbm.GrlbmError) as e:
            grlbm.Batch([r])
        assert e.value.code == 4


def test_contexts_of_different_direction_counts_coexist(grlbm, W):
    """Kernel launch limits are per process: creating a context with fewer
    directions must not break the launches of one with more."""
    big = W.batch_instances(count=1, seed=5, sizes=(24,), dirs=(64,), steps=3)[0]
    small = W.batch_instances(count=1, seed=6, sizes=(24,), dirs=(8,), steps=3)[0]
    for P in (grlbm.PRECISION_FP32, grlbm.PLAIN_FP64):
        with grlbm.prepare(big, P) as a, grlbm.prepare(small, P) as b:
            a.step(3)
            b.step(3)
            assert np.isfinite(a.moments_if()["E"]).all() and np.isfinite(b.moments_if()["E"]).all()


def test_batch_config5_instances_against_oracle(grlbm, W, oracle):
    """Four instances of the batched workload (64 seeded problems of grid
    sizes 64^2..512^2, 16/32/64 directions, flat or Schwarzschild, 500 steps)
    -- its smallest ones, one per direction count where the draw has one --
    stepped in one batch with the persistent launch, against the FP64
    oracle: E within 1e-5 (relative L2)."""
    allc = W.batch_instances(count=64, seed=10)
    picked = []
    for nd in (16, 32, 64):
        small = sorted((c for c in allc if c["n_dir"] == nd), key=lambda c: c["nx_"] * c["ny_"])
        picked += small[:1]
    rest = sorted((c for c in allc if all(c is not p for p in picked)), key=lambda c: c["nx_"] * c["ny_"] * c["n_dir"])
    picked += rest[:4 - len(picked)]
    assert len(picked) == 4 and len({c["n_dir"] for c in picked}) >= 2
    probs = [grlbm.prepare(c, grlbm.PRECISION_FP32) for c in picked]
    try:
        with grlbm.Batch(probs) as b:
            b.set_shape(1, True)
            b.step(int(picked[0]["n_steps"]))
        for c, r in zip(picked, probs):
            ref = oracle.run(c, "oracle", n_threads=0)
            err = float(np.linalg.norm(r.moments_if()["E"] - ref["E"]) / np.linalg.norm(ref["E"]))
            assert err <= 1e-5, (c["nx_"], c["n_dir"], err)
    finally:
        for r in probs:
            r.close()
