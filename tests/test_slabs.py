"""Slab decomposition host logic on CPU: the band partition, and the ghost-row
exchange of 2dradiation_b200/slabs.py over gloo with two and three ranks,
driving a CPU stand-in for a context whose step reads `ghost` rows around
each cell.  Each step updates the band's inner rows while the exchange is
in flight and its edge rows after it.  The multi-rank runs must equal the
one-rank run bit for bit, as the GPU runs do (tests/test_gpu_slabs.py)."""
import importlib
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def slabs():
    return importlib.import_module("2dradiation_b200.slabs")


def test_partition_covers_rows_once():
    part = slabs().partition
    for ny_, world in [(10, 1), (10, 2), (11, 3), (400, 8), (7, 7)]:
        bands = part(ny_, world)
        assert bands[0][0] == 1 and bands[-1][1] == ny_ + 1
        assert all(b[1] == c[0] for b, c in zip(bands, bands[1:]))
        assert max(b - a for a, b in bands) - min(b - a for a, b in bands) <= 1
    with pytest.raises(ValueError):
        part(3, 4)


class CpuRows:
    """A context stand-in: state[d][j][i] over the whole grid; a step updates
    the band's interior rows from rows within `ghost` of each cell."""

    def __init__(self, nx, ny, nd, ghost, band, seed):
        rng = np.random.default_rng(seed)
        self.state = torch.from_numpy(rng.uniform(size=(nd, ny, nx)))
        self.nx, self.ny, self.nd, self.ghost, self.band = nx, ny, nd, ghost, band
        self.row_elems = nx * nd
        self.dtype = torch.float64
        self.stream = None

    def buffer(self, rows):
        return torch.empty(rows * self.row_elems, dtype=self.dtype)

    def copy_rows(self, j, n, buf, to_buffer):
        view = buf.view(self.nd, n, self.nx)
        if to_buffer:
            view.copy_(self.state[:, j:j + n, :])
        else:
            self.state[:, j:j + n, :] = view

    def energy(self):
        lo, hi = self.band
        return float(self.state[:, lo:hi, 1:-1].sum())

    def _rows(self, new, j_first, j_end):
        g, s = self.ghost, self.state
        for j in range(j_first, j_end):
            rows = [min(max(j + k, 0), self.ny - 1) for k in range(-g, g + 1)]
            mix = sum((k + 2.0) * torch.roll(s[:, r, :], shifts=k, dims=1) for k, r in enumerate(rows))
            new[:, j, 1:-1] = (0.5 * s[:, j, 1:-1] + 0.5 * mix[:, 1:-1] / mix.abs().max())

    def step(self, n=1):
        for _ in range(n):
            new = self.state.clone()
            self._rows(new, *self.band)
            self.state = new

    def step_rows(self, j_first, j_end, finish):
        """One step in parts (grlbm_step_rows_async): rows [j_first, j_end)
        of the next state from the current one; finish swaps them in."""
        if getattr(self, "_next", None) is None:
            self._next = self.state.clone()
        self._rows(self._next, j_first, j_end)
        if finish:
            self.state, self._next = self._next, None


class CpuAdaptiveRows(CpuRows):
    """An adaptive-streaming stand-in: besides the intensities, per-node
    angles and six moment planes.  A step first turns each band cell's angle
    from the flux averaged over its 3x3 neighbourhood (the previous moments),
    then streams from rows within `ghost` weighted by the source rows'
    previous angles, then takes the band's moments -- the dependencies of
    UpdateRotationMatrizes, the rotated gather and the collide."""

    adaptive = True

    def __init__(self, nx, ny, nd, ghost, band, seed):
        super().__init__(nx, ny, nd, ghost, band, seed)
        rng = np.random.default_rng(seed + 1)
        self.ang = torch.from_numpy(rng.uniform(size=(ny, nx)))
        self.mom = torch.from_numpy(rng.uniform(size=(6, ny, nx)))
        self.fields = [(1, nx, torch.float64), (2, 6 * nx, torch.float64)]

    def field_buffer(self, k, rows):
        return torch.empty(rows * self.fields[k][1], dtype=torch.float64)

    def copy_field_rows(self, k, j, n, buf, to_buffer):
        view = buf.view(n, self.nx) if k == 0 else buf.view(6, n, self.nx)
        src = self.ang[j:j + n, :] if k == 0 else self.mom[:, j:j + n, :]
        if to_buffer:
            view.copy_(src)
        else:
            src.copy_(view)

    def step(self, n=1):
        lo, hi = self.band
        g = self.ghost
        for _ in range(n):
            ang = self.ang.clone()
            flux = self.mom[1] + 2.0 * self.mom[2]
            for j in range(lo, hi):
                avg = sum(torch.roll(flux[j + b], shifts=a) for b in (-1, 0, 1) for a in (-1, 0, 1)) / 9.0
                ang[j, 1:-1] = torch.atan2(avg[1:-1], 1.0 + self.mom[0, j, 1:-1])
            new = self.state.clone()
            s = self.state
            for j in range(lo, hi):
                rows = [min(max(j + k, 0), self.ny - 1) for k in range(-g, g + 1)]
                mix = sum(torch.cos(self.ang[r, :]) * torch.roll(s[:, r, :], shifts=k, dims=1)
                          for k, r in enumerate(rows))
                new[:, j, 1:-1] = 0.5 * s[:, j, 1:-1] + 0.5 * torch.sin(ang[j, 1:-1]) * mix[:, 1:-1] / len(rows)
            self.state, self.ang = new, ang
            for q in range(6):
                self.mom[q, lo:hi, :] = new[:, lo:hi, :].sum(dim=0) * (q + 1.0) + new[q % self.nd, lo:hi, :]


def _worker(rank, world, port, nx, ny_, nd, ghost, steps, out, adaptive=False):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        S = slabs()
        band = S.partition(ny_, world)[rank]
        rows = (CpuAdaptiveRows if adaptive else CpuRows)(nx + 2, ny_ + 2, nd, ghost, band, seed=7)
        slab = S.Slab(rows, rank, world, ny_, ghost)
        slab.step(steps)
        out[rank] = rows.state[:, band[0]:band[1], :].clone()
        if adaptive:
            out[("ang", rank)] = rows.ang[band[0]:band[1], :].clone()
        out[("energy", rank)] = slab.energy()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("ghost,world,ny_", [(1, 2, 12), (2, 2, 12), (2, 3, 7), (3, 3, 11)])
def test_multi_rank_exchange_equals_one_rank(ghost, world, ny_):
    """(Bands of 2-4 rows with 2-3 ghost rows: the inner rows are empty or
    single, the edge row ranges meet or overlap the band's middle.)"""
    nx, nd, steps = 9, 3, 5
    S = slabs()
    single = CpuRows(nx + 2, ny_ + 2, nd, ghost, (1, ny_ + 1), seed=7)
    S.Slab(single, 0, 1, ny_, ghost).step(steps)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, world, port, nx, ny_, nd, ghost, steps, out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        got = torch.cat([out[r] for r in range(world)], dim=1)
        energies = [out[("energy", r)] for r in range(world)]
    assert torch.equal(got, single.state[:, 1:ny_ + 1, :])
    # the all-reduced energy is the same on every rank and is the whole grid's
    assert len(set(energies)) == 1
    assert abs(energies[0] - single.energy()) <= 1e-12 * abs(single.energy())


@pytest.mark.parametrize("ghost,world,ny_", [(1, 2, 8), (2, 3, 9)])
def test_adaptive_exchange_equals_one_rank(ghost, world, ny_):
    """Adaptive streaming's bands also exchange the ghost rows' angles and the
    moment row next to the band, and step after the exchange: the ranks'
    intensities and angles equal the one-rank run bit for bit."""
    nx, nd, steps = 7, 3, 4
    S = slabs()
    single = CpuAdaptiveRows(nx + 2, ny_ + 2, nd, ghost, (1, ny_ + 1), seed=7)
    S.Slab(single, 0, 1, ny_, ghost).step(steps)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, world, port, nx, ny_, nd, ghost, steps, out, True))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        got = torch.cat([out[r] for r in range(world)], dim=1)
        ang = torch.cat([out[("ang", r)] for r in range(world)], dim=0)
    assert torch.equal(got, single.state[:, 1:ny_ + 1, :])
    assert torch.equal(ang, single.ang[1:ny_ + 1, :])

