"""Slab decomposition of the radiation step: one process per GPU, each
stepping one band of interior node rows of the same grid, with the rows next
to each band exchanged between neighbouring ranks before every step.

The reference runs on one node with OpenMP only (Readme.txt:5-6); this is
the multi-GPU form of its time loop (src/Radiation.cpp:789-822).  Every step
only reads intensities within `ghost` node rows of the cell it updates (the
departure records bound it: grlbm_departure_rows), so a rank that holds its
band plus `ghost` up-to-date rows on each side steps its band exactly as a
single GPU would: the results are bit-identical to the single-GPU run.

Each rank keeps the whole grid in its context (tables are built for every
cell; rows outside band + ghosts go stale and are never read), so the state
is replicated and the work is divided.  The exchange is point-to-point over
torch.distributed: NCCL between GPUs (NVLink), gloo for the CPU tests.
"""
from __future__ import annotations

import torch
import torch.distributed as dist


def partition(ny_: int, world: int) -> list[tuple[int, int]]:
    """Interior node rows 1..ny_ split into `world` contiguous bands
    [j_first, j_end), the first ny_ % world bands one row taller."""
    if world < 1 or ny_ < world:
        raise ValueError(f"cannot split {ny_} rows over {world} ranks")
    base, extra = divmod(ny_, world)
    bands, j = [], 1
    for r in range(world):
        n = base + (1 if r < extra else 0)
        bands.append((j, j + n))
        j += n
    return bands


class RadiationRows:
    """Row access to a Radiation context's intensity state through the C-ABI
    (grlbm_copy_rows), for the exchange."""

    def __init__(self, rad, device: torch.device):
        self.rad = rad
        self.device = device
        self.row_bytes = rad.row_bytes()
        self.dtype = torch.float32 if rad.precision == 1 else torch.float64
        self.row_elems = self.row_bytes // (4 if rad.precision == 1 else 8)
        self.stream = torch.cuda.ExternalStream(rad.stream, device=device)

    def buffer(self, rows: int) -> torch.Tensor:
        return torch.empty(rows * self.row_elems, dtype=self.dtype, device=self.device)

    def copy_rows(self, j_first: int, n: int, buf: torch.Tensor, to_buffer: bool):
        self.rad.copy_rows(j_first, n, buf.data_ptr(), to_buffer)

    def step(self, n: int = 1):
        self.rad.step_async(n)

    def energy(self) -> float:
        return self.rad.energy()  # grlbm_energy: the band's interior cells


class Slab:
    """One rank's band and its exchange with the neighbouring bands.

    `state` provides row_elems, dtype, buffer(rows), copy_rows(j, n, buf,
    to_buffer), step(n) and a `stream` usable as torch.cuda.stream(...) (or
    None on CPU).  The band must be at least `ghost` rows high."""

    def __init__(self, state, rank: int, world: int, ny_: int, ghost: int, group=None):
        self.state, self.rank, self.world, self.group = state, rank, world, group
        self.bands = partition(ny_, world)
        self.band = self.bands[rank]
        self.ghost = ghost
        if world > 1 and min(b - a for a, b in self.bands) < ghost:
            raise ValueError(f"bands of {min(b - a for a, b in self.bands)} rows are thinner than the "
                             f"{ghost} ghost rows a step reads")
        g = ghost
        self.send_lo = state.buffer(g) if rank > 0 else None
        self.recv_lo = state.buffer(g) if rank > 0 else None
        self.send_hi = state.buffer(g) if rank < world - 1 else None
        self.recv_hi = state.buffer(g) if rank < world - 1 else None

    def _ops(self):
        lo, hi = self.band
        ops = []
        if self.rank > 0:
            ops.append(dist.P2POp(dist.isend, self.send_lo, self.rank - 1, self.group))
            ops.append(dist.P2POp(dist.irecv, self.recv_lo, self.rank - 1, self.group))
        if self.rank < self.world - 1:
            ops.append(dist.P2POp(dist.isend, self.send_hi, self.rank + 1, self.group))
            ops.append(dist.P2POp(dist.irecv, self.recv_hi, self.rank + 1, self.group))
        return ops

    def exchange(self):
        """Sends the `ghost` rows at each edge of the band to the neighbour
        and receives the neighbour's rows next to the band."""
        if self.world == 1 or self.ghost == 0:
            return
        lo, hi, g, st = self.band[0], self.band[1], self.ghost, self.state
        ctx = torch.cuda.stream(st.stream) if st.stream is not None else _Null()
        with ctx:
            if self.send_lo is not None:
                st.copy_rows(lo, g, self.send_lo, True)
            if self.send_hi is not None:
                st.copy_rows(hi - g, g, self.send_hi, True)
            for req in dist.batch_isend_irecv(self._ops()):
                req.wait()
            if self.recv_lo is not None:
                st.copy_rows(lo - g, g, self.recv_lo, False)
            if self.recv_hi is not None:
                st.copy_rows(hi, g, self.recv_hi, False)

    def step(self, n: int = 1):
        """n time steps of the band, each after a ghost-row exchange."""
        for _ in range(n):
            self.exchange()
            self.state.step(1)

    def energy(self) -> float:
        """The global energy: the bands' FP64 sums added by one all-reduce."""
        e = torch.tensor([self.state.energy()], dtype=torch.float64,
                         device=self.state.device if self.state.stream is not None else "cpu")
        if self.world > 1:
            dist.all_reduce(e, group=self.group)
        return float(e.item())


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


def open_slab(case: dict, precision: int, rank: int, world: int, device: int, group=None):
    """A Radiation context for `case` on `device`, restricted to this rank's
    band, with its exchange.  Returns (radiation, slab)."""
    G = __import__(__package__ or "2dradiation_b200")
    rad = G.prepare(case, precision, device=device)
    slab = Slab(RadiationRows(rad, torch.device("cuda", device)), rank, world, int(case["ny_"]),
                rad.departure_rows(), group)
    rad.set_rows(*slab.band)
    return rad, slab
