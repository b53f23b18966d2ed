"""Slab decomposition of the radiation step: one process per GPU, each
stepping one band of interior node rows of the same grid, with the rows next
to each band exchanged between neighbouring ranks before every step.

The reference runs on one node with OpenMP only (Readme.txt:5-6); this is
the multi-GPU form of its time loop (src/Radiation.cpp:789-822).  Every step
only reads intensities within `ghost` node rows of the cell it updates (the
departure records bound it: grlbm_departure_rows), so a rank that holds its
band plus `ghost` up-to-date rows on each side steps its band exactly as a
single GPU would: the results are bit-identical to the single-GPU run.

Each rank's context holds the grid's state, but builds the geodesic tables
of its band's cells only, and steps only its band (rows outside band +
ghosts go stale and are never read).  The exchange is point-to-point over
torch.distributed: NCCL between GPUs (NVLink), gloo for the CPU tests.  A
step overlaps it with the band's inner rows -- those whose gathers stay
within the band -- and updates the edge rows once the ghost rows are in:
with NCCL every wait is a dependency between CUDA streams, and the host never
waits on the GPU within a step.

Adaptive streaming (src/Radiation.cpp:361-378, 415-453, 513-575) also reads
the neighbours' rotation angles at the corners it gathers from and their
flux moments in the angle update's 3x3 average, so its bands exchange the
ghost rows' angles and the moment row next to the band too, and step the
whole band after the exchange.
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
        G = __import__(__package__ or "2dradiation_b200")
        self.adaptive = int(rad.case["streaming_type"]) in (G.FLAT_ADAPTIVE, G.CURVED_ADAPTIVE)
        # the other per-node fields of an adaptive band's exchange: (field, elements per row, dtype)
        self.fields = [(G.ROWS_ANGLES, rad.node_row_bytes(G.ROWS_ANGLES) // 8, torch.float64),
                       (G.ROWS_MOMENTS, rad.node_row_bytes(G.ROWS_MOMENTS) // self.dtype.itemsize,
                        self.dtype)] if self.adaptive else []

    def buffer(self, rows: int) -> torch.Tensor:
        return torch.empty(rows * self.row_elems, dtype=self.dtype, device=self.device)

    def copy_rows(self, j_first: int, n: int, buf: torch.Tensor, to_buffer: bool):
        self.rad.copy_rows(j_first, n, buf.data_ptr(), to_buffer)

    def field_buffer(self, k: int, rows: int) -> torch.Tensor:
        _, elems, dtype = self.fields[k]
        return torch.empty(rows * elems, dtype=dtype, device=self.device)

    def copy_field_rows(self, k: int, j_first: int, n: int, buf: torch.Tensor, to_buffer: bool):
        self.rad.copy_node_rows(self.fields[k][0], j_first, n, buf.data_ptr(), to_buffer)

    def step(self, n: int = 1):
        self.rad.step_async(n)

    def step_rows(self, j_first: int, j_end: int, finish: bool):
        self.rad.step_rows_async(j_first, j_end, finish)

    def energy(self) -> float:
        return self.rad.energy()  # grlbm_energy: the band's interior cells


class Slab:
    """One rank's band and its exchange with the neighbouring bands.

    `state` provides row_elems, dtype, buffer(rows), copy_rows(j, n, buf,
    to_buffer), step(n) and a `stream` usable as torch.cuda.stream(...) (or
    None on CPU); for adaptive streaming (state.adaptive) also `fields` and
    field_buffer(k, rows) / copy_field_rows(k, j, n, buf, to_buffer) for the
    rotation angles (field 0, `ghost` rows) and the moments (field 1, one
    row).  The band must be at least `ghost` rows high."""

    def __init__(self, state, rank: int, world: int, ny_: int, ghost: int, group=None):
        self.state, self.rank, self.world, self.group = state, rank, world, group
        self.bands = partition(ny_, world)
        self.band = self.bands[rank]
        self.ghost = ghost
        if world > 1 and min(b - a for a, b in self.bands) < ghost:
            raise ValueError(f"bands of {min(b - a for a, b in self.bands)} rows are thinner than the "
                             f"{ghost} ghost rows a step reads")
        g = ghost
        self.adaptive = bool(getattr(state, "adaptive", False))
        # per exchanged field (the intensities; for adaptive streaming also the
        # angles and the moments): rows, and send/receive buffers below and
        # above the band (None at the grid's edges)
        self.parts = [(None, g)] + ([(0, g), (1, 1)] if self.adaptive else [])
        self.bufs = []
        for k, rows in self.parts:
            make = (lambda n: state.buffer(n)) if k is None else (lambda n, k=k: state.field_buffer(k, n))
            self.bufs.append({side: (make(rows), make(rows)) if (side == "lo" and rank > 0) or
                              (side == "hi" and rank < world - 1) else None for side in ("lo", "hi")})

    def _copy(self, k, j, n, buf, to_buffer):
        if k is None:
            self.state.copy_rows(j, n, buf, to_buffer)
        else:
            self.state.copy_field_rows(k, j, n, buf, to_buffer)

    def _ops(self):
        ops = []
        for b in self.bufs:
            if b["lo"] is not None:
                ops.append(dist.P2POp(dist.isend, b["lo"][0], self.rank - 1, self.group))
                ops.append(dist.P2POp(dist.irecv, b["lo"][1], self.rank - 1, self.group))
            if b["hi"] is not None:
                ops.append(dist.P2POp(dist.isend, b["hi"][0], self.rank + 1, self.group))
                ops.append(dist.P2POp(dist.irecv, b["hi"][1], self.rank + 1, self.group))
        return ops

    def _send(self):
        """Packs the rows at each edge of the band and starts their exchange
        with the neighbours; returns the pending requests."""
        lo, hi = self.band
        for (k, rows), b in zip(self.parts, self.bufs):
            if b["lo"] is not None:
                self._copy(k, lo, rows, b["lo"][0], True)
            if b["hi"] is not None:
                self._copy(k, hi - rows, rows, b["hi"][0], True)
        return dist.batch_isend_irecv(self._ops())

    def _receive(self, reqs):
        """Waits for the exchange (NCCL: the state's stream waits) and
        unpacks the neighbours' rows next to the band."""
        lo, hi = self.band
        for req in reqs:
            req.wait()
        for (k, rows), b in zip(self.parts, self.bufs):
            if b["lo"] is not None:
                self._copy(k, lo - rows, rows, b["lo"][1], False)
            if b["hi"] is not None:
                self._copy(k, hi, rows, b["hi"][1], False)

    def exchange(self):
        """Sends the `ghost` rows at each edge of the band to the neighbour
        and receives the neighbour's rows next to the band."""
        if self.world == 1 or self.ghost == 0:
            return
        st = self.state
        with (torch.cuda.stream(st.stream) if st.stream is not None else _Null()):
            self._receive(self._send())

    def step(self, n: int = 1):
        """n time steps of the band.  Each starts the ghost-row exchange,
        updates the inner rows [lo + g, hi - g) meanwhile (their gathers
        read the band only), then, with the ghost rows in, the edge rows."""
        st = self.state
        if self.world == 1 or self.ghost == 0:
            st.step(n)
            return
        if self.adaptive:  # the angle update reads the moments next to the band: exchange, then step
            with (torch.cuda.stream(st.stream) if st.stream is not None else _Null()):
                for _ in range(n):
                    self._receive(self._send())
                    st.step(1)
            return
        lo, hi, g = self.band[0], self.band[1], self.ghost
        edges = [(lo, min(lo + g, hi)), (max(hi - g, lo + g), hi)]
        with (torch.cuda.stream(st.stream) if st.stream is not None else _Null()):
            for _ in range(n):
                reqs = self._send()
                if lo + g < hi - g:
                    st.step_rows(lo + g, hi - g, False)
                self._receive(reqs)
                for a, b in edges:
                    if a < b:
                        st.step_rows(a, b, False)
                st.step_rows(hi, hi, True)

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


def ghost_rows(local: int, device, world: int, group=None) -> int:
    """The ghost depth all ranks use: the largest of the ranks' own
    (grlbm_departure_rows over each band's cells)."""
    if world == 1:
        return local
    t = torch.tensor([local], dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return int(t.item())


def open_slab(case: dict, precision: int, rank: int, world: int, device: int, group=None):
    """A Radiation context for `case` on `device` that steps this rank's band
    and builds the tables of its cells only, with its exchange.  Returns
    (radiation, slab)."""
    G = __import__(__package__ or "2dradiation_b200")
    band = partition(int(case["ny_"]), world)[rank]
    rad = G.prepare(case, precision, device=device, rows=band)
    dev = torch.device("cuda", device)
    slab = Slab(RadiationRows(rad, dev), rank, world, int(case["ny_"]),
                ghost_rows(rad.departure_rows(), dev, world, group), group)
    return rad, slab
