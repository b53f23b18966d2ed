"""The hand-written adjoint (grlbm_adjoint_*) against FP64 central finite
differences of the plain forward, through a thin torch.autograd.Function, on
a small version of the adjoint workload (Schwarzschild, Gaussian-sum eta and
kappaA, fluid at rest): loss 0.5 |E - E*|^2 of the final E, E* from a second
field set.  Also: the checkpointed forward is the plain forward bit for bit,
a scattering field's gradient is checked the same way, and flat streaming."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make(W, **kw):
    base = dict(nx_=40, ny_=36, n_dir=16, n_fourier=5, steps=23)
    base.update(kw)
    return W.adjoint_case(**base)


class Runner:
    """Plain forward of a case on a context whose tables are built once."""

    def __init__(self, grlbm, case):
        self.r = grlbm.prepare(case, grlbm.PLAIN_FP64)
        self.case = case
        self.I0 = np.zeros(self.r.nxy * self.r.nd)
        self.steps = int(case["n_steps"])

    def fields(self, **over):
        f = {k: v.copy() for k, v in self.case["fields"].items()}
        f.update(over)
        return f

    def iteration_total(self):
        st = self.r.stats()
        return round(st["average_iterations"] * st["steps"] * self.case["nx_"] * self.case["ny_"])

    def E(self, **over):
        before = self.iteration_total()
        self.r.set_fields(self.fields(**over))
        self.r.set_intensity(self.I0)
        self.r.step(self.steps)
        self.iterations = self.iteration_total() - before  # lambda-iteration cycles of this run
        return self.r.moments_if()["E"].copy()


def interior(case):
    nx, ny = case["nx_"] + 2, case["ny_"] + 2
    m = np.zeros((ny, nx), bool)
    m[1:-1, 1:-1] = True
    return m.ravel()


def autograd_fn(torch, run, adj):
    class RadiationE(torch.autograd.Function):
        @staticmethod
        def forward(ctx, eta, kappaA):
            run.r.set_fields(run.fields(eta=eta.detach().cpu().numpy(), kappaA=kappaA.detach().cpu().numpy()))
            run.r.set_intensity(run.I0)
            adj.forward(run.steps)
            return torch.from_numpy(run.r.moments_if()["E"].copy())

        @staticmethod
        def backward(ctx, gE):
            g = adj.backward(gE.detach().cpu().numpy())
            return torch.from_numpy(g["eta"]), torch.from_numpy(g["kappaA"])

    return RadiationE


def fd_check(run, L, f, name, cells, grad, rtol, min_checked=None, atol=1e-9):
    """Central differences with h = 1e-6 at `cells`.  The adjoint is that of
    the lambda iterations the forward ran; a perturbation that changes any
    cell's iteration count (the reference's exit test compares moments that
    can be rounding noise) leaves the map being differentiated, so such
    cells are skipped -- at least `min_checked` must remain."""
    h = 1e-6
    run.E()
    base = run.iterations
    checked = 0
    for c in cells:
        p = f[name].copy()
        p[c] += h
        Lp = L(run.E(**{name: p}))
        same = run.iterations == base
        p[c] -= 2 * h
        Lm = L(run.E(**{name: p}))
        same = same and run.iterations == base
        if not same:
            continue
        fd = (Lp - Lm) / (2 * h)
        assert abs(grad[c] - fd) <= rtol * abs(fd) + atol, (name, c, grad[c], fd)
        checked += 1
    assert checked >= (len(cells) if min_checked is None else min_checked), (name, checked)


@pytest.mark.parametrize("every", [5, 23])
def test_adjoint_matches_finite_differences(grlbm, W, every):
    import torch
    case = make(W)
    run = Runner(grlbm, case)
    mask = interior(case)
    Et = Runner(grlbm, make(W, seeds=(7, 8))).E()
    f = case["fields"]
    with grlbm.Adjoint(run.r, every) as adj:
        Fn = autograd_fn(torch, run, adj)
        eta = torch.tensor(f["eta"], requires_grad=True)
        ka = torch.tensor(f["kappaA"], requires_grad=True)
        E = Fn.apply(eta, ka)
        E_ref = run.E()
        assert np.array_equal(E.detach().numpy(), E_ref)  # the checkpointed forward is the plain forward
        loss = 0.5 * ((E - torch.from_numpy(Et))[torch.from_numpy(mask)] ** 2).sum()
        loss.backward()
    L = lambda E_: 0.5 * float(np.sum((E_ - Et)[mask] ** 2))
    rng = np.random.default_rng(9)
    cells = rng.choice(np.flatnonzero(mask & (f["eta"] > 1e-3)), 8, replace=False)
    fd_check(run, L, f, "eta", cells, eta.grad.numpy(), 2e-3)
    fd_check(run, L, f, "kappaA", cells, ka.grad.numpy(), 2e-3)


def test_adjoint_config4_full_size(grlbm, W):
    """The adjoint workload at its stated size: Schwarzschild 256^2 cells, 48
    directions, 200 steps, checkpoints every 20; the FP32 adjoint's gradients
    of eta and kappaA against FP64 central differences (h = 1e-6) of the
    plain forward on 32 random cells (seed 9) of the emitting region.  The
    absolute slack covers the differences' own rounding: the loss is ~4e3,
    so a relative 1e-15 in it is ~2e-6 in a difference quotient."""
    case = W.adjoint_case()
    assert (case["nx_"], case["ny_"], case["n_dir"], int(case["n_steps"])) == (256, 256, 48, 200)
    run = Runner(grlbm, case)
    mask = interior(case)
    Et = Runner(grlbm, W.adjoint_case(seeds=(7, 8))).E()
    f = case["fields"]
    with grlbm.Adjoint(run.r, 20) as adj:
        run.r.set_fields(run.fields())
        run.r.set_intensity(run.I0)
        adj.forward(run.steps)
        E = run.r.moments_if()["E"]
        g = adj.backward(np.where(mask, E - Et, 0.0))
    L = lambda E_: 0.5 * float(np.sum((E_ - Et)[mask] ** 2))
    rng = np.random.default_rng(9)
    cells = rng.choice(np.flatnonzero(mask & (f["eta"] > 1e-3)), 32, replace=False)
    fd_check(run, L, f, "eta", cells, g["eta"], 2e-3, atol=1e-5)
    fd_check(run, L, f, "kappaA", cells, g["kappaA"], 2e-3, atol=1e-5)


def test_adjoint_scattering_gradient(grlbm, W):
    """kappa0 > 0: the lambda iteration runs several cycles; the adjoint
    follows the recorded cycle counts."""
    case = make(W, steps=12)
    f = case["fields"]
    f["kappa0"][:] = 0.5 * f["kappaA"]
    run = Runner(grlbm, case)
    mask = interior(case)
    Et = Runner(grlbm, make(W, steps=12, seeds=(7, 8))).E()
    with grlbm.Adjoint(run.r, 5) as adj:
        run.r.set_fields(run.fields())
        run.r.set_intensity(run.I0)
        adj.forward(run.steps)
        E = run.r.moments_if()["E"]
        g = adj.backward(np.where(mask, E - Et, 0.0))
    L = lambda E_: 0.5 * float(np.sum((E_ - Et)[mask] ** 2))
    rng = np.random.default_rng(4)
    cells = rng.choice(np.flatnonzero(mask & (f["kappa0"] > 1e-2)), 12, replace=False)
    fd_check(run, L, f, "kappa0", cells, g["kappa0"], 2e-3, min_checked=4)
    fd_check(run, L, f, "eta", cells, g["eta"], 2e-3, min_checked=4)


def test_adjoint_flat_streaming(grlbm, W):
    case = W.adjoint_case(nx_=30, ny_=26, n_dir=12, steps=9)
    case["metric_kind"], case["streaming_type"], case["excision"] = W.MINKOWSKI, W.FLAT_FIXED, -1.0
    run = Runner(grlbm, case)
    mask = interior(case)
    f = case["fields"]
    Et = 0.5 * run.E()
    with grlbm.Adjoint(run.r, 4) as adj:
        run.r.set_fields(run.fields())
        run.r.set_intensity(run.I0)
        adj.forward(run.steps)
        E = run.r.moments_if()["E"]
        g = adj.backward(np.where(mask, E - Et, 0.0))
    L = lambda E_: 0.5 * float(np.sum((E_ - Et)[mask] ** 2))
    cells = np.random.default_rng(2).choice(np.flatnonzero(mask & (f["eta"] > 1e-3)), 5, replace=False)
    fd_check(run, L, f, "kappaA", cells, g["kappaA"], 2e-3)


def test_adjoint_rejects_moving_fluids(grlbm, W):
    case = W.moving_scatter(nx_=16, ny_=16, n_dir=8, steps=2)
    with grlbm.prepare(case, grlbm.PLAIN_FP64) as r:
        with pytest.raises(grlbm.GrlbmError) as e:
            grlbm.Adjoint(r)
        assert e.value.code == 4
