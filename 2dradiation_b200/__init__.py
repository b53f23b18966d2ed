"""Python harness over the C-ABI of libgrlbm.so (include/grlbm.h).

The product is the shared library built from ``csrc/`` (host set-up in C++,
kernels and C-ABI in CUDA for sm_100a).  This module is the thin ctypes layer
the tests and the benchmark drive it with; it mirrors the reference's
``Radiation`` workflow (src/Radiation.h): construct, write the public input
buffers, ``LoadInitialData``, ``UpdateFourierCoefficients``, then time steps.

There is no CPU fallback: if ``libgrlbm.so`` is missing or no GPU is usable,
the calls raise.
"""
from __future__ import annotations

import ctypes as C
import importlib
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libgrlbm.so"

workloads = importlib.import_module(__name__ + ".workloads")

OK = 0
ERRORS = {1: "ARGUMENT", 2: "CUDA", 3: "STATE", 4: "UNSUPPORTED", 5: "NONCONVERGED", 6: "HOST"}
MINKOWSKI, SCHWARZSCHILD, KERRSCHILD = 0, 1, 2
FLAT_FIXED, FLAT_ADAPTIVE, CURVED_FIXED, CURVED_ADAPTIVE, GEODESIC_FIXED = 0, 1, 2, 3, 4
MOMENTS, INTENSITIES = 0, 1
PLAIN_FP64, PRECISION_FP32, FAST_FP64 = 0, 1, 2
ROWS_ANGLES, ROWS_MOMENTS = 1, 2  # grlbm_copy_node_rows fields


class GrlbmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"grlbm error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class GridDesc(C.Structure):
    _fields_ = [("nx_", C.c_int64), ("ny_", C.c_int64), ("startx", C.c_double), ("starty", C.c_double),
                ("endx", C.c_double), ("endy", C.c_double), ("cfl", C.c_double)]


class MetricDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("m", C.c_double), ("a", C.c_double), ("excision", C.c_double)]


class RunDesc(C.Structure):
    _fields_ = [("n_dir", C.c_int32), ("n_fourier", C.c_int32), ("streaming_type", C.c_int32),
                ("precision", C.c_int32), ("keep_source_nodes_active", C.c_int32),
                ("initial_data_type", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("steps", C.c_int64), ("max_iterations", C.c_int32), ("average_iterations", C.c_double),
                ("rk_substeps", C.c_int64), ("rk_nonconverged", C.c_int32),
                ("departures_off_grid", C.c_int32), ("table_ms", C.c_double),
                ("far_departures", C.c_int64)]


_D = C.POINTER(C.c_double)
_lib = None

# Every entry point of include/grlbm.h with its argument types.
SIGNATURES = {
    "grlbm_create": ([C.POINTER(GridDesc), C.POINTER(MetricDesc), C.POINTER(RunDesc), C.c_int32,
                      C.POINTER(C.c_void_p)], C.c_int),
    "grlbm_destroy": ([C.c_void_p], None),
    "grlbm_last_error": ([C.c_void_p], C.c_char_p),
    "grlbm_get_grid": ([C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), _D, _D, _D], C.c_int),
    "grlbm_set_fields": ([C.c_void_p] + [_D] * 6, C.c_int),
    "grlbm_set_initial_data": ([C.c_void_p, C.POINTER(C.c_uint8)] + [_D] * 7, C.c_int),
    "grlbm_load_initial_data": ([C.c_void_p], C.c_int),
    "grlbm_set_intensity": ([C.c_void_p, _D], C.c_int),
    "grlbm_get_intensity": ([C.c_void_p, _D], C.c_int),
    "grlbm_update_fourier_coefficients": ([C.c_void_p, C.c_double, C.c_int32], C.c_int),
    "grlbm_get_fourier_coefficients": ([C.c_void_p] + [_D] * 5, C.c_int),
    "grlbm_set_fourier_coefficients": ([C.c_void_p] + [_D] * 5, C.c_int),
    "grlbm_step": ([C.c_void_p, C.c_int32], C.c_int),
    "grlbm_step_async": ([C.c_void_p, C.c_int32], C.c_int),
    "grlbm_step_rows_async": ([C.c_void_p, C.c_int64, C.c_int64, C.c_int32], C.c_int),
    "grlbm_sync": ([C.c_void_p], C.c_int),
    "grlbm_stream": ([C.c_void_p], C.c_void_p),
    "grlbm_get_moments_if": ([C.c_void_p] + [_D] * 6, C.c_int),
    "grlbm_compute_moments_lf": ([C.c_void_p] + [_D] * 7, C.c_int),
    "grlbm_energy": ([C.c_void_p, _D], C.c_int),
    "grlbm_energy_noalloc": ([C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p], C.c_int),
    "grlbm_selftest_staging_wait": ([C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32),
                                     C.POINTER(C.c_double)], C.c_int),
    "grlbm_get_stats": ([C.c_void_p, C.POINTER(Stats)], C.c_int),
    "grlbm_batch_create": ([C.POINTER(C.c_void_p), C.c_int32, C.POINTER(C.c_void_p)], C.c_int),
    "grlbm_batch_destroy": ([C.c_void_p], None),
    "grlbm_batch_last_error": ([C.c_void_p], C.c_char_p),
    "grlbm_batch_step": ([C.c_void_p, C.c_int32], C.c_int),
    "grlbm_batch_autotune": ([C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
    "grlbm_batch_set_shape": ([C.c_void_p, C.c_int32, C.c_int32], C.c_int),
    "grlbm_adjoint_create": ([C.c_void_p, C.c_int32, C.POINTER(C.c_void_p)], C.c_int),
    "grlbm_adjoint_destroy": ([C.c_void_p], None),
    "grlbm_adjoint_last_error": ([C.c_void_p], C.c_char_p),
    "grlbm_adjoint_forward": ([C.c_void_p, C.c_int32], C.c_int),
    "grlbm_adjoint_backward": ([C.c_void_p, _D, _D, _D, _D], C.c_int),
    "grlbm_set_initial_flux_angle": ([C.c_void_p, _D], C.c_int),
    "grlbm_set_update_tables_each_step": ([C.c_void_p, C.c_int32, C.c_double, C.c_int32], C.c_int),
    "grlbm_host_write_frame_csv": ([C.POINTER(GridDesc), C.c_float, _D, _D, _D, _D, C.c_char_p, C.c_char_p],
                                   C.c_int),
    "grlbm_write_frame_csv": ([C.c_void_p, C.c_float, C.c_char_p, C.c_char_p], C.c_int),
    "grlbm_run_simulation": ([C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_int32, C.c_char_p,
                              C.POINTER(C.c_int64)], C.c_int),
    "grlbm_set_rows": ([C.c_void_p, C.c_int64, C.c_int64], C.c_int),
    "grlbm_row_bytes": ([C.c_void_p, C.POINTER(C.c_int64)], C.c_int),
    "grlbm_copy_rows": ([C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_int32], C.c_int),
    "grlbm_departure_rows": ([C.c_void_p, C.POINTER(C.c_int32)], C.c_int),
    "grlbm_node_row_bytes": ([C.c_void_p, C.c_int32, C.POINTER(C.c_int64)], C.c_int),
    "grlbm_copy_node_rows": ([C.c_void_p, C.c_int32, C.c_int64, C.c_int64, C.c_void_p, C.c_int32], C.c_int),
    "grlbm_set_tile_shape": ([C.c_void_p, C.c_int32, C.c_int32], C.c_int),
    "grlbm_write_log": ([C.c_void_p, C.c_char_p], C.c_int),
    "grlbm_host_write_log": ([C.POINTER(GridDesc), C.POINTER(MetricDesc), C.c_int32, C.c_int32, C.c_char_p,
                              C.c_int64, C.c_int32, C.c_double, C.POINTER(C.c_char_p), _D, C.c_int32,
                              C.c_char_p], C.c_int),
    "grlbm_trace_begin": ([C.c_void_p, C.c_char_p], C.c_int),
    "grlbm_trace_end": ([C.c_void_p], C.c_int),
    "grlbm_get_tile_shape": ([C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
    "grlbm_host_stencil": ([C.c_int32, C.c_int32, _D, _D, _D, _D, C.POINTER(C.c_int64), _D], C.c_int),
    "grlbm_host_flux_table": ([C.c_int32, C.POINTER(C.c_int32), _D, _D, _D, C.c_int32], C.c_int),
    "grlbm_host_metric_arrays": ([C.POINTER(GridDesc), C.POINTER(MetricDesc), _D], C.c_int),
    "grlbm_metric_array_count": ([], C.c_int32),
}


def lib() -> C.CDLL:
    """Load libgrlbm.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} is missing: run __graft_entry__.build()")
        L = C.CDLL(str(LIB_PATH))
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(_D)


def _check(rc: int, ctx=None):
    if rc != OK:
        msg = lib().grlbm_last_error(ctx)
        raise GrlbmError(rc, msg.decode() if msg else "")


def grid_desc(case: dict) -> GridDesc:
    return GridDesc(int(case["nx_"]), int(case["ny_"]), case["start"][0], case["start"][1],
                    case["end"][0], case["end"][1], case["cfl"])


def metric_desc(case: dict) -> MetricDesc:
    return MetricDesc(int(case["metric_kind"]), case["m"], case["a"], case["excision"])


# ------------------------------------------------------------- host helpers
def host_stencil(n: int, intensity: bool = True) -> dict:
    out = {k: np.zeros(n) for k in ("w", "phi", "cx", "cy")}
    ng = 10 * n if intensity else 0
    idx = np.zeros(max(4 * ng, 1), dtype=np.int64)
    wt = np.zeros(max(4 * ng, 1))
    _check(lib().grlbm_host_stencil(n, int(intensity), _p(out["w"]), _p(out["phi"]), _p(out["cx"]),
                                    _p(out["cy"]), idx.ctypes.data_as(C.POINTER(C.c_int64)), _p(wt)))
    out["ig_index"], out["ig_weight"] = idx[:4 * ng], wt[:4 * ng]
    return out


def host_flux_table(n: int) -> dict:
    size = C.c_int32(0)
    _check(lib().grlbm_host_flux_table(n, C.byref(size), None, None, None, 0))
    k = size.value
    a, s, z = np.zeros(k), np.zeros(k), np.zeros(k)
    _check(lib().grlbm_host_flux_table(n, C.byref(size), _p(a), _p(s), _p(z), k))
    return {"inputs": a, "sigma": s, "normalization": z}


def host_write_log(case: dict, date: str, time_steps: int, max_iterations: int, average_iterations: float,
                   times: list, directory: str):
    """Log.txt (Logger::Write's format) from given values, without a GPU."""
    names = (C.c_char_p * max(len(times), 1))(*[n.encode() for n, _ in times])
    secs = np.ascontiguousarray([t for _, t in times] or [0.0], dtype=np.float64)
    _check(lib().grlbm_host_write_log(C.byref(grid_desc(case)), C.byref(metric_desc(case)), int(case["n_dir"]),
                                      int(case["n_fourier"]), date.encode(), int(time_steps), int(max_iterations),
                                      float(average_iterations), names, _p(secs), len(times), directory.encode()))


def host_metric_arrays(case: dict) -> np.ndarray:
    nxy = workloads.nxy(case)
    n = lib().grlbm_metric_array_count()
    out = np.zeros(n * nxy)
    g, m = grid_desc(case), metric_desc(case)
    _check(lib().grlbm_host_metric_arrays(C.byref(g), C.byref(m), _p(out)))
    return out.reshape(n, nxy)


# ------------------------------------------------------------------ solver
class Radiation:
    """One problem resident on the GPU (a grlbm_ctx)."""

    def __init__(self, case: dict, precision: int = PLAIN_FP64, device: int = -1):
        self.case = case
        self.precision = precision
        self.nd = int(case["n_dir"])
        self.nf = int(case["n_fourier"])
        g, m = grid_desc(case), metric_desc(case)
        r = RunDesc(self.nd, self.nf, int(case["streaming_type"]), precision,
                    int(case["keep_source_nodes_active"]), int(case["initial_data_type"]))
        h = C.c_void_p()
        _check(lib().grlbm_create(C.byref(g), C.byref(m), C.byref(r), device, C.byref(h)))
        self.h = h
        nx, ny = C.c_int64(), C.c_int64()
        dx, dy, dt = C.c_double(), C.c_double(), C.c_double()
        _check(lib().grlbm_get_grid(h, C.byref(nx), C.byref(ny), C.byref(dx), C.byref(dy), C.byref(dt)), h)
        self.nx, self.ny, self.dx, self.dy, self.dt = nx.value, ny.value, dx.value, dy.value, dt.value
        self.nxy = self.nx * self.ny

    def close(self):
        if getattr(self, "h", None):
            lib().grlbm_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _c(self, rc):
        _check(rc, self.h)

    @property
    def stream(self) -> int:
        return lib().grlbm_stream(self.h) or 0

    def set_fields(self, f: dict):
        arr = [np.ascontiguousarray(f[k], dtype=np.float64) for k in ("kappa0", "kappa1", "kappaA", "eta", "ux", "uy")]
        self._c(lib().grlbm_set_fields(self.h, *[_p(a) for a in arr]))

    def set_initial_data(self, f: dict):
        mask = np.ascontiguousarray(f["is_initial"], dtype=np.uint8)
        arr = [np.ascontiguousarray(f[k], dtype=np.float64) for k in
               ("initial_I", "initial_E_LF", "initial_Fx_LF", "initial_Fy_LF", "initial_Pxx_LF",
                "initial_Pxy_LF", "initial_Pyy_LF")]
        self._c(lib().grlbm_set_initial_data(self.h, mask.ctypes.data_as(C.POINTER(C.c_uint8)),
                                             *[_p(a) for a in arr]))

    def load_initial_data(self):
        self._c(lib().grlbm_load_initial_data(self.h))

    def set_intensity(self, I: np.ndarray):
        I = np.ascontiguousarray(I, dtype=np.float64).reshape(-1)
        assert I.size == self.nxy * self.nd
        self._c(lib().grlbm_set_intensity(self.h, _p(I)))

    def intensity(self) -> np.ndarray:
        out = np.zeros(self.nxy * self.nd)
        self._c(lib().grlbm_get_intensity(self.h, _p(out)))
        return out

    def update_fourier_coefficients(self, rk_tol: float, max_substeps: int = 0):
        self._c(lib().grlbm_update_fourier_coefficients(self.h, rk_tol, max_substeps))

    def coefficients(self) -> dict:
        out = {k: np.zeros(self.nxy * self.nf) for k in ("coefS", "coefX", "coefY", "coefCx", "coefCy")}
        self._c(lib().grlbm_get_fourier_coefficients(self.h, *[_p(out[k]) for k in
                                                               ("coefS", "coefX", "coefY", "coefCx", "coefCy")]))
        return out

    def set_coefficients(self, coef: dict):
        arr = [np.ascontiguousarray(coef[k], dtype=np.float64) for k in ("coefS", "coefX", "coefY", "coefCx", "coefCy")]
        for a in arr:
            assert a.size == self.nxy * self.nf
        self._c(lib().grlbm_set_fourier_coefficients(self.h, *[_p(a) for a in arr]))

    def step(self, n: int):
        self._c(lib().grlbm_step(self.h, n))

    def step_async(self, n: int):
        self._c(lib().grlbm_step_async(self.h, n))

    def step_rows_async(self, j_first: int, j_end: int, finish: bool):
        """One step's update of node rows [j_first, j_end), enqueued without
        waiting; finish=True ends the step (grlbm_step_rows_async)."""
        self._c(lib().grlbm_step_rows_async(self.h, int(j_first), int(j_end), int(bool(finish))))

    def sync(self):
        self._c(lib().grlbm_sync(self.h))

    def moments_if(self, out: dict | None = None) -> dict:
        names = ("E", "Fx", "Fy", "Pxx", "Pxy", "Pyy")
        out = out if out is not None else {k: np.zeros(self.nxy) for k in names}
        self._c(lib().grlbm_get_moments_if(self.h, *[_p(out[k]) for k in names]))
        return out

    def moments_lf(self) -> dict:
        names = ("E_LF", "Fx_LF", "Fy_LF", "Pxx_LF", "Pxy_LF", "Pyy_LF", "F_LF")
        out = {k: np.zeros(self.nxy) for k in names}
        self._c(lib().grlbm_compute_moments_lf(self.h, *[_p(out[k]) for k in names]))
        return out

    def energy(self) -> float:
        v = C.c_double()
        self._c(lib().grlbm_energy(self.h, C.byref(v)))
        return v.value

    def update_tables_each_step(self, enabled: bool, rk_tol: float = 1e-4, max_substeps: int = 0):
        """Config::updateFourierHarmonics: rebuild the geodesic tables before every step."""
        self._c(lib().grlbm_set_update_tables_each_step(self.h, 1 if enabled else 0, rk_tol, max_substeps))

    # ---- frames and the simulation loop (Grid::WriteFrametoCsv, RunSimulation) ----
    def write_frame(self, time: float, directory: str, name: str = ""):
        self._c(lib().grlbm_write_frame_csv(self.h, time, directory.encode(), name.encode()))

    def run_simulation(self, sim_time: float, write_period: float, directory: str | None,
                       t0: float = 0.0, save_initial: bool = True) -> int:
        n = C.c_int64()
        self._c(lib().grlbm_run_simulation(self.h, t0, sim_time, write_period, 1 if save_initial else 0,
                                           directory.encode() if directory else None, C.byref(n)))
        return n.value

    # ---- Log.txt and the profile session (Logger::Write, Profiler::Session) ----
    def write_log(self, directory: str):
        self._c(lib().grlbm_write_log(self.h, directory.encode()))

    def trace_begin(self, path: str):
        self._c(lib().grlbm_trace_begin(self.h, path.encode()))

    def trace_end(self):
        self._c(lib().grlbm_trace_end(self.h))

    # ---- slab decomposition (one band of interior node rows per rank) ----
    def set_rows(self, j_first: int, j_end: int):
        self._c(lib().grlbm_set_rows(self.h, j_first, j_end))

    def row_bytes(self) -> int:
        v = C.c_int64()
        self._c(lib().grlbm_row_bytes(self.h, C.byref(v)))
        return v.value

    def copy_rows(self, j_first: int, n: int, buffer_ptr: int, to_buffer: bool):
        """Rows [j_first, j_first + n) of the state to/from a device buffer
        (stream-ordered on the context's stream)."""
        self._c(lib().grlbm_copy_rows(self.h, j_first, n, C.c_void_p(buffer_ptr), 1 if to_buffer else 0))

    # ---- tiles of the precision form's fixed streaming step ----
    def set_tile_shape(self, tile_x: int, tile_y: int):
        self._c(lib().grlbm_set_tile_shape(self.h, tile_x, tile_y))

    def tile_shape(self) -> tuple:
        x, y = C.c_int32(), C.c_int32()
        self._c(lib().grlbm_get_tile_shape(self.h, C.byref(x), C.byref(y)))
        return (x.value, y.value)

    def departure_rows(self) -> int:
        v = C.c_int32()
        self._c(lib().grlbm_departure_rows(self.h, C.byref(v)))
        return v.value

    def node_row_bytes(self, what: int) -> int:
        """Bytes of one node row of ROWS_ANGLES or ROWS_MOMENTS."""
        v = C.c_int64()
        self._c(lib().grlbm_node_row_bytes(self.h, what, C.byref(v)))
        return v.value

    def copy_node_rows(self, what: int, j_first: int, n: int, buffer_ptr: int, to_buffer: bool):
        """Rows [j_first, j_first + n) of the rotation angles (ROWS_ANGLES) or
        the moments (ROWS_MOMENTS) to/from a device buffer (stream-ordered on
        the context's stream)."""
        self._c(lib().grlbm_copy_node_rows(self.h, what, j_first, n, C.c_void_p(buffer_ptr),
                                           1 if to_buffer else 0))

    def stats(self) -> dict:
        s = Stats()
        self._c(lib().grlbm_get_stats(self.h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}


class Adjoint:
    """Gradients of a loss of the final E with respect to eta, kappaA and
    kappa0 by the hand-written adjoint (grlbm_adjoint_*) of a plain-form
    Radiation whose fields and tables are set."""

    def __init__(self, rad: "Radiation", checkpoint_every: int = 20):
        self.rad = rad
        h = C.c_void_p()
        rc = lib().grlbm_adjoint_create(rad.h, checkpoint_every, C.byref(h))
        if rc != OK:
            raise GrlbmError(rc, (lib().grlbm_adjoint_last_error(None) or b"").decode())
        self.h = h

    def _c(self, rc):
        if rc != OK:
            raise GrlbmError(rc, (lib().grlbm_adjoint_last_error(self.h) or b"").decode())

    def forward(self, n_steps: int):
        self._c(lib().grlbm_adjoint_forward(self.h, n_steps))

    def backward(self, dL_dE: np.ndarray) -> dict:
        n = self.rad.nxy
        g = {k: np.zeros(n) for k in ("eta", "kappaA", "kappa0")}
        d = np.ascontiguousarray(dL_dE, dtype=np.float64)
        self._c(lib().grlbm_adjoint_backward(self.h, _p(d), _p(g["eta"]), _p(g["kappaA"]), _p(g["kappa0"])))
        return g

    def close(self):
        if self.h:
            lib().grlbm_adjoint_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Several problems stepped together (grlbm_batch_*): the problems' own
    steps launched concurrently (any forms), or one persistent launch per
    step (FP32 fixed streaming without active sources).  The Radiation
    objects stay usable."""

    def __init__(self, problems: list):
        self.problems = list(problems)
        arr = (C.c_void_p * len(self.problems))(*[p.h for p in self.problems])
        h = C.c_void_p()
        rc = lib().grlbm_batch_create(arr, len(self.problems), C.byref(h))
        if rc != OK:
            raise GrlbmError(rc, (lib().grlbm_batch_last_error(None) or b"").decode())
        self.h = h

    def _c(self, rc):
        if rc != OK:
            raise GrlbmError(rc, (lib().grlbm_batch_last_error(self.h) or b"").decode())

    def step(self, n: int):
        self._c(lib().grlbm_batch_step(self.h, n))

    def set_shape(self, blocks_per_sm: int, largest_first: bool = True):
        """blocks_per_sm >= 1: the persistent launch; 0: each problem's own
        step, the problems' launches concurrent; -m (m = 1..8): the same
        with the tiled forms' grids cut to shares of m GPUs' worth of
        resident blocks (the default, -4)."""
        self._c(lib().grlbm_batch_set_shape(self.h, int(blocks_per_sm), int(bool(largest_first))))

    def autotune(self, trial_steps: int = 4) -> dict:
        bps, lf = C.c_int32(), C.c_int32()
        self._c(lib().grlbm_batch_autotune(self.h, trial_steps, C.byref(bps), C.byref(lf)))
        return {"blocks_per_sm": bps.value, "largest_first": bool(lf.value)}

    def close(self):
        if self.h:
            lib().grlbm_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_cost(case: dict, precision: int = PRECISION_FP32) -> float:
    """A problem's estimated step time in arbitrary units, as a batch's
    launch shares estimate it (grlbm_batch_set_shape): cells x (directions +
    48), x 1.6 for curved streaming, x the form's cost against the FP32
    fixed-streaming step (fast FP64 1.9, plain FP64 4.7, adaptive streaming
    4.9 in FP32 and 10.9 in plain FP64)."""
    st = int(case["streaming_type"])
    curved = st in (CURVED_FIXED, CURVED_ADAPTIVE)
    adaptive = st in (FLAT_ADAPTIVE, CURVED_ADAPTIVE)
    if precision == FAST_FP64:
        form = 1.9
    elif adaptive:
        form = 4.9 if precision == PRECISION_FP32 else 10.9
    else:
        form = 1.0 if precision == PRECISION_FP32 else 4.7
    return int(case["nx_"]) * int(case["ny_"]) * (int(case["n_dir"]) + 48.0) * (1.6 if curved else 1.0) * form


def share_problems(cases: list, world: int, precision: int = PRECISION_FP32) -> list:
    """Independent problems dealt to `world` GPUs as replicas, with no
    communication between them: largest estimated cost (batch_cost) first,
    each to the GPU with the least cost so far (the lower rank on a tie).
    Returns each rank's problem indices in ascending order; every rank
    computes the same deal."""
    if world < 1:
        raise ValueError("world must be at least 1")
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for k in sorted(range(len(cases)), key=lambda k: (-batch_cost(cases[k], precision), k)):
        r = min(range(world), key=lambda r: (load[r], r))
        load[r] += batch_cost(cases[k], precision)
        out[r].append(k)
    return [sorted(x) for x in out]


def selftest_staging_wait(arrive: bool, limit_us: int, device: int = -1) -> dict:
    """One block's bounded wait on an mbarrier phase that nothing (arrive
    False) or one thread (arrive True) completes: {"completed", "waited_us"}."""
    done, waited = C.c_int32(-1), C.c_double(0.0)
    _check(lib().grlbm_selftest_staging_wait(device, int(bool(arrive)), int(limit_us), C.byref(done),
                                             C.byref(waited)))
    return {"completed": bool(done.value), "waited_us": waited.value}


def prepare(case: dict, precision: int = PLAIN_FP64, device: int = -1, rows: tuple | None = None) -> Radiation:
    """Construct and load a case the way RunSimulation starts
    (src/Radiation.cpp:745-746): inputs, LoadInitialData, then the geodesic
    tables.  With `rows` = (j_first, j_end) the context steps that band of
    node rows and builds the tables of its cells only."""
    r = Radiation(case, precision, device)
    if rows is not None:
        r.set_rows(*rows)
    r.set_fields(case["fields"])
    r.set_initial_data(case["fields"])
    r.load_initial_data()
    r.update_fourier_coefficients(case["rk_tol"])
    return r


def run(case: dict, precision: int = PLAIN_FP64, steps: int | None = None) -> dict:
    """Whole run of a case; returns the same keys as the oracle's run()."""
    with prepare(case, precision) as r:
        r.step(int(case["n_steps"] if steps is None else steps))
        res = dict(r.moments_if())
        res.update(r.moments_lf())
        res["I"] = r.intensity()
        res.update(r.coefficients())
        st = r.stats()
        res["max_iterations"] = st["max_iterations"]
        res["average_iterations"] = st["average_iterations"]
        res["stats"] = st
        res["energy"] = r.energy()
        res["nx"], res["ny"] = r.nx, r.ny
    return res
