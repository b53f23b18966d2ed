"""Seeded synthetic workloads for the GR lattice-Boltzmann radiation step.

A *case* is a plain dict that fully describes one run of the reference's
``Radiation`` set-up (exe/main.cpp style): the ``Grid``, the ``Metric``
subclass, the two ``Stencil`` orders, the ``Config`` flags and every public
input buffer the caller writes (src/Radiation.h:28-39, 62-68).  The same dict
drives the product (through the C-ABI), the CPU restatement and the reference
build, so all three see identical inputs.

Random fields come from splitmix64 (one 64-bit draw per node, in node order
ij = i + j*nx over the whole grid including the halo) mapped to [0,1) by the
top 53 bits; normal variates use Box-Muller on consecutive pairs of draws.
The generator is written here in numpy so that every side reads the same
numbers; nothing depends on a library RNG.

Named workloads:
  flat_beam        100x100 cells, 20 directions, Minkowski, 500 steps: a beam
                   injected at the left boundary (|y| <= 0.1) on the two
                   directions that bracket angle 0 (the offset stencil has no
                   direction at exactly 0), kept active every step.
  curved_shell     200x200, 32 directions, Kerr-Schild M=1 a=0 on [-6,6]^2,
                   nF=5, 1000 steps, excision r <= 2.4, RK45 tol 1e-10;
                   emissivity 1 on the shell 3.8 <= r <= 4.2, absorption
                   U[0,0.5] (seed 2) inside r < 5.
  curved_scatter   400x400, 64 directions, same metric, nF=16, 2000 steps;
                   absorption lognormal exp(-1 + 0.5 z) (seed 3), scattering
                   U[0,2] (seed 4), emissivity a Gaussian blob (amplitude 1,
                   width 0.5) at (3,0).
Smaller variants (same domains and physics, fewer cells/directions/steps) are
built by ``make_case(name, **overrides)`` for the parity tests.
"""
from __future__ import annotations

import math

import numpy as np

MINKOWSKI, SCHWARZSCHILD, KERRSCHILD = 0, 1, 2
FLAT_FIXED, FLAT_ADAPTIVE, CURVED_FIXED, CURVED_ADAPTIVE = 0, 1, 2, 3
MOMENTS, INTENSITIES = 0, 1

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, n: int) -> np.ndarray:
    """n consecutive splitmix64 outputs for a given seed (uint64)."""
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + k * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        z = z ^ (z >> np.uint64(31))
    return z


def uniform(seed: int, n: int) -> np.ndarray:
    """n draws in [0,1): top 53 bits of splitmix64 times 2^-53."""
    return (splitmix64(seed, n) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed: int, n: int) -> np.ndarray:
    """n standard normal draws by Box-Muller on consecutive uniform pairs."""
    u = uniform(seed, 2 * n).reshape(n, 2)
    u1 = 1.0 - u[:, 0]  # (0,1]
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u[:, 1])


def grid_coords(nx_: int, ny_: int, start, end):
    """Node coordinates as the reference's Grid computes them
    (src/Grid.cpp:4-24, 48-55): x(i) = (start - dx) + i*dx, dx = L/(nx_-1)."""
    nx, ny = nx_ + 2, ny_ + 2
    dx = (end[0] - start[0]) / (nx - 1.0 - 2.0)
    dy = (end[1] - start[1]) / (ny - 1.0 - 2.0)
    startx = start[0] - dx
    starty = start[1] - dy
    x = startx + np.arange(nx, dtype=np.float64) * dx
    y = starty + np.arange(ny, dtype=np.float64) * dy
    X = np.broadcast_to(x[None, :], (ny, nx)).reshape(-1).copy()
    Y = np.broadcast_to(y[:, None], (ny, nx)).reshape(-1).copy()
    return X, Y, dx, dy


def _base(name, nx_, ny_, start, end, n_dir, n_fourier, steps, metric_kind,
          streaming_type, cfl=0.9, m=1.0, a=0.0, excision=2.4, rk_tol=1e-10,
          initial_data_type=INTENSITIES, keep=False):
    nxy = (nx_ + 2) * (ny_ + 2)
    z = np.zeros(nxy)
    fields = {k: z.copy() for k in ("kappa0", "kappa1", "kappaA", "eta", "ux", "uy",
                                    "initial_E_LF", "initial_Fx_LF", "initial_Fy_LF",
                                    "initial_Pxx_LF", "initial_Pxy_LF", "initial_Pyy_LF")}
    fields["is_initial"] = np.zeros(nxy, dtype=np.uint8)
    fields["initial_I"] = np.zeros(nxy * n_dir)
    return dict(name=name, nx_=nx_, ny_=ny_, start=tuple(start), end=tuple(end), cfl=cfl,
                metric_kind=metric_kind, m=m, a=a, excision=excision, n_dir=n_dir,
                n_fourier=n_fourier, streaming_type=streaming_type,
                initial_data_type=initial_data_type, keep_source_nodes_active=int(keep),
                n_steps=steps, rk_tol=rk_tol, fields=fields)


def flat_beam(nx_=100, ny_=100, n_dir=20, steps=500, n_fourier=5):
    c = _base("flat_beam", nx_, ny_, (-1, -1), (1, 1), n_dir, n_fourier, steps,
              MINKOWSKI, FLAT_FIXED, excision=-1.0, rk_tol=1e-4,
              initial_data_type=INTENSITIES, keep=True)
    X, Y, dx, dy = grid_coords(nx_, ny_, (-1, -1), (1, 1))
    nx = nx_ + 2
    i = np.arange(X.size) % nx
    src = (i <= 1) & (Y >= -0.1) & (Y <= 0.1)
    f = c["fields"]
    f["is_initial"][src] = 1
    I0 = f["initial_I"].reshape(-1, n_dir)
    I0[src, 0] = 1.0
    I0[src, n_dir - 1] = 1.0
    return c


def curved_shell(nx_=200, ny_=200, n_dir=32, n_fourier=5, steps=1000, rk_tol=1e-10,
                 excision=2.4, seed=2):
    c = _base("curved_shell", nx_, ny_, (-6, -6), (6, 6), n_dir, n_fourier, steps,
              KERRSCHILD, CURVED_FIXED, excision=excision, rk_tol=rk_tol)
    X, Y, _, _ = grid_coords(nx_, ny_, (-6, -6), (6, 6))
    r = np.sqrt(X * X + Y * Y)
    f = c["fields"]
    f["eta"][(r >= 3.8) & (r <= 4.2)] = 1.0
    ka = 0.5 * uniform(seed, X.size)
    f["kappaA"][:] = np.where(r < 5.0, ka, 0.0)
    return c


def curved_scatter(nx_=400, ny_=400, n_dir=64, n_fourier=16, steps=2000, rk_tol=1e-10,
                   excision=2.4, seeds=(3, 4)):
    c = _base("curved_scatter", nx_, ny_, (-6, -6), (6, 6), n_dir, n_fourier, steps,
              KERRSCHILD, CURVED_FIXED, excision=excision, rk_tol=rk_tol)
    X, Y, _, _ = grid_coords(nx_, ny_, (-6, -6), (6, 6))
    f = c["fields"]
    f["kappaA"][:] = np.exp(-1.0 + 0.5 * normal(seeds[0], X.size))
    f["kappa0"][:] = 2.0 * uniform(seeds[1], X.size)
    f["eta"][:] = np.exp(-((X - 3.0) ** 2 + Y ** 2) / (2.0 * 0.5 ** 2))
    return c


def moving_scatter(nx_=24, ny_=24, n_dir=16, n_fourier=5, steps=8, metric_kind=KERRSCHILD,
                   streaming_type=CURVED_FIXED, seed=11):
    """Exercises every term of Collide (src/Radiation.cpp:641-736): moving
    fluid (ux, uy != 0), anisotropic scattering (kappa1 != 0), emission and
    absorption, plus von Mises moment sources kept active every step
    (InitialDataType::Moments, src/Radiation.cpp:128-182)."""
    c = _base("moving_scatter", nx_, ny_, (-6, -6), (6, 6), n_dir, n_fourier, steps,
              metric_kind, streaming_type, excision=2.4, rk_tol=1e-6,
              initial_data_type=MOMENTS, keep=True)
    X, Y, _, _ = grid_coords(nx_, ny_, (-6, -6), (6, 6))
    n = X.size
    u = uniform(seed, 8 * n).reshape(8, n)
    f = c["fields"]
    f["kappa0"][:] = 1.5 * u[0]
    f["kappa1"][:] = 0.3 * u[1]
    f["kappaA"][:] = 0.5 * u[2]
    f["eta"][:] = np.exp(-((X - 3.0) ** 2 + (Y + 1.0) ** 2) / 2.0)
    f["ux"][:] = 0.3 * (u[3] - 0.5)
    f["uy"][:] = 0.3 * (u[4] - 0.5)
    src = (np.abs(X + 4.0) < 1.0) & (np.abs(Y - 3.0) < 1.0)
    f["is_initial"][src] = 1
    f["initial_E_LF"][src] = 1.0 + u[5][src]
    f["initial_Fx_LF"][src] = 0.5 * (u[6][src] - 0.2)
    f["initial_Fy_LF"][src] = 0.4 * (u[7][src] - 0.5)
    return c


WORKLOADS = {
    "flat_beam": flat_beam,
    "curved_shell": curved_shell,
    "curved_scatter": curved_scatter,
    "moving_scatter": moving_scatter,
}


def batch_instances(count=64, seed=10, sizes=(64, 128, 256, 512), dirs=(16, 32, 64), steps=500,
                    n_fourier=5, rk_tol=1e-10):
    """Independent problems of uneven size for the batched form: per instance
    a grid size from `sizes` (square), a direction count from `dirs`, and flat
    (Minkowski, flat streaming) or Schwarzschild M=1 (Kerr-Schild
    coordinates, curved streaming, excision r <= 2.4) at random, on
    [-6,6]^2.  Fields as the curved-shell problem (eta = 1 on 3.8 <= r <= 4.2,
    kappaA ~ U[0, 0.5) for r < 5) plus scattering kappa0 ~ U[0, 1) for r < 5,
    each instance with its own seeds; intensities start at zero."""
    u = uniform(seed, 3 * count).reshape(count, 3)
    out = []
    for k in range(count):
        n = int(sizes[min(int(u[k, 0] * len(sizes)), len(sizes) - 1)])
        nd = int(dirs[min(int(u[k, 1] * len(dirs)), len(dirs) - 1)])
        curved = u[k, 2] >= 0.5
        c = _base(f"batch{k}", n, n, (-6, -6), (6, 6), nd, n_fourier, steps,
                  KERRSCHILD if curved else MINKOWSKI, CURVED_FIXED if curved else FLAT_FIXED,
                  excision=2.4 if curved else -1.0, rk_tol=rk_tol)
        X, Y, _, _ = grid_coords(n, n, (-6, -6), (6, 6))
        r = np.sqrt(X * X + Y * Y)
        f = c["fields"]
        f["eta"][(r >= 3.8) & (r <= 4.2)] = 1.0
        f["kappaA"][:] = np.where(r < 5.0, 0.5 * uniform(1000 + 2 * k + seed, X.size), 0.0)
        f["kappa0"][:] = np.where(r < 5.0, uniform(1001 + 2 * k + seed, X.size), 0.0)
        out.append(c)
    return out


def gaussian_field(X, Y, seed, count=8, width=1.0, box=5.0):
    """Sum of `count` Gaussians of the given width with amplitudes U[0, 1) and
    centres U[-box, box)^2."""
    u = uniform(seed, 3 * count).reshape(count, 3)
    f = np.zeros_like(X)
    for a, cx, cy in u:
        f += a * np.exp(-((X - (2 * cx - 1) * box) ** 2 + (Y - (2 * cy - 1) * box) ** 2) / (2 * width * width))
    return f


def adjoint_case(nx_=256, ny_=256, n_dir=48, n_fourier=5, steps=200, seeds=(5, 6), rk_tol=1e-10):
    """Fields of the adjoint workload: Schwarzschild M = 1 (Kerr-Schild
    coordinates, excision r <= 2.4) on [-6,6]^2, eta and kappaA each a sum of
    8 Gaussians of width 1 (seeds[0], seeds[1]), no scattering, fluid at rest,
    intensities starting at zero.  The target of the loss comes from the same
    problem with seeds (7, 8)."""
    c = _base("adjoint", nx_, ny_, (-6, -6), (6, 6), n_dir, n_fourier, steps, KERRSCHILD, CURVED_FIXED,
              excision=2.4, rk_tol=rk_tol)
    X, Y, _, _ = grid_coords(nx_, ny_, (-6, -6), (6, 6))
    c["fields"]["eta"][:] = gaussian_field(X, Y, seeds[0])
    c["fields"]["kappaA"][:] = gaussian_field(X, Y, seeds[1])
    return c


def make_case(name: str, **overrides) -> dict:
    return WORKLOADS[name](**overrides)


def nxy(case: dict) -> int:
    return (int(case["nx_"]) + 2) * (int(case["ny_"]) + 2)
