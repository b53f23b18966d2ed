"""Slab decomposition host logic on CPU: the band partition, and the ghost-row
exchange of 2dradiation_b200/slabs.py over gloo with two ranks, driving a
CPU stand-in for a context whose step reads `ghost` rows around each cell.
The two-rank run must equal the one-rank run bit for bit, as the GPU runs
do (tests/test_gpu_slabs.py)."""
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

    def step(self, n=1):
        g, (lo, hi) = self.ghost, self.band
        s = self.state
        new = s.clone()
        for j in range(lo, hi):
            rows = [min(max(j + k, 0), self.ny - 1) for k in range(-g, g + 1)]
            mix = sum((k + 2.0) * torch.roll(s[:, r, :], shifts=k, dims=1) for k, r in enumerate(rows))
            new[:, j, 1:-1] = (0.5 * s[:, j, 1:-1] + 0.5 * mix[:, 1:-1] / mix.abs().max())
        self.state = new


def _worker(rank, world, port, nx, ny_, nd, ghost, steps, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        S = slabs()
        band = S.partition(ny_, world)[rank]
        rows = CpuRows(nx + 2, ny_ + 2, nd, ghost, band, seed=7)
        slab = S.Slab(rows, rank, world, ny_, ghost)
        slab.step(steps)
        out[rank] = rows.state[:, band[0]:band[1], :].clone()
        out[("energy", rank)] = slab.energy()
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("ghost", [1, 2])
def test_two_rank_exchange_equals_one_rank(ghost):
    nx, ny_, nd, steps = 9, 12, 3, 5
    S = slabs()
    single = CpuRows(nx + 2, ny_ + 2, nd, ghost, (1, ny_ + 1), seed=7)
    S.Slab(single, 0, 1, ny_, ghost).step(steps)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, nx, ny_, nd, ghost, steps, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        got = torch.cat([out[0], out[1]], dim=1)
        energies = (out[("energy", 0)], out[("energy", 1)])
    assert torch.equal(got, single.state[:, 1:ny_ + 1, :])
    # the all-reduced energy is the same on both ranks and is the whole grid's
    assert energies[0] == energies[1]
    assert abs(energies[0] - single.energy()) <= 1e-12 * abs(single.energy())
