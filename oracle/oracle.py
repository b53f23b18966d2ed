"""ctypes front end for the CPU checkers in this directory.

Test infrastructure only: tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py load this module; the
product library never does.

Two libraries share one C entry-point shape (oracle/ref_api.h):

* ``liboracle.so`` -- ``oracle_run``: the C restatement of the reference's
  radiation step (oracle/grlbm_oracle.c), plain IEEE FP64;
* ``_ref/libref_{fast,strict}.so`` -- ``ref_run``: the reference itself,
  compiled from its own sources (oracle/Makefile).  ``_ref`` exists only where
  the reference tree was available at build time.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
N_METRIC_ARRAYS = 102

# Member order of the reference's src/Metric.h:19-65.
METRIC_NAMES = (
    "g00_ll g00_uu g01_ll g01_uu g02_ll g02_uu g11_ll g11_uu g12_ll g12_uu g22_ll g22_uu "
    "d0_g00_lll d1_g00_lll d2_g00_lll d0_g01_lll d1_g01_lll d2_g01_lll "
    "d0_g02_lll d1_g02_lll d2_g02_lll d0_g11_lll d1_g11_lll d2_g11_lll "
    "d0_g12_lll d1_g12_lll d2_g12_lll d0_g22_lll d1_g22_lll d2_g22_lll "
    "d0_g00_luu d1_g00_luu d2_g00_luu d0_g01_luu d1_g01_luu d2_g01_luu "
    "d0_g02_luu d1_g02_luu d2_g02_luu d0_g11_luu d1_g11_luu d2_g11_luu "
    "d0_g12_luu d1_g12_luu d2_g12_luu d0_g22_luu d1_g22_luu d2_g22_luu "
    "alpha beta1_u beta1_l beta2_u beta2_l gamma11_ll gamma11_uu gamma12_ll gamma12_uu "
    "gamma22_ll gamma22_uu d1_alpha_l d2_alpha_l "
    "d1_beta1_lu d1_beta2_lu d2_beta1_lu d2_beta2_lu d1_beta1_ll d1_beta2_ll d2_beta1_ll d2_beta2_ll "
    "d1_gamma11_lll d2_gamma11_lll d1_gamma12_lll d2_gamma12_lll d1_gamma22_lll d2_gamma22_lll "
    "d1_gamma11_luu d2_gamma11_luu d1_gamma12_luu d2_gamma12_luu d1_gamma22_luu d2_gamma22_luu "
    "K11_ll K12_ll K22_ll "
    "tetrad00_ul tetrad01_ul tetrad02_ul tetrad10_ul tetrad11_ul tetrad12_ul "
    "tetrad20_ul tetrad21_ul tetrad22_ul "
    "tetrad00_lu tetrad01_lu tetrad02_lu tetrad10_lu tetrad11_lu tetrad12_lu "
    "tetrad20_lu tetrad21_lu tetrad22_lu"
).split()
assert len(METRIC_NAMES) == N_METRIC_ARRAYS

_P = C.POINTER(C.c_double)


class Params(C.Structure):
    _fields_ = [
        ("nx_", C.c_int64), ("ny_", C.c_int64),
        ("startx", C.c_double), ("starty", C.c_double),
        ("endx", C.c_double), ("endy", C.c_double), ("cfl", C.c_double),
        ("metric_kind", C.c_int32), ("m", C.c_double), ("a", C.c_double),
        ("excision", C.c_double),
        ("n_dir", C.c_int32), ("n_fourier", C.c_int32),
        ("streaming_type", C.c_int32), ("initial_data_type", C.c_int32),
        ("keep_source_nodes_active", C.c_int32), ("n_steps", C.c_int32),
        ("rk_tol", C.c_double), ("use_run_simulation", C.c_int32),
        ("n_threads", C.c_int32), ("update_tables_each_step", C.c_int32),
    ]


class Inputs(C.Structure):
    _fields_ = [(n, _P) for n in ("kappa0", "kappa1", "kappaA", "eta", "ux", "uy")] + [
        ("is_initial", C.POINTER(C.c_uint8)),
        ("initial_I", _P),
    ] + [(n, _P) for n in ("initial_E_LF", "initial_Fx_LF", "initial_Fy_LF",
                           "initial_Pxx_LF", "initial_Pxy_LF", "initial_Pyy_LF",
                           "metric_override")]


_OUT_NODE = ("E", "Fx", "Fy", "Pxx", "Pxy", "Pyy",
             "E_LF", "Fx_LF", "Fy_LF", "Pxx_LF", "Pxy_LF", "Pyy_LF", "F_LF")
_OUT_COEF = ("coefS", "coefX", "coefY", "coefCx", "coefCy")


class Outputs(C.Structure):
    _fields_ = [(n, _P) for n in _OUT_NODE] + [("I", _P)] + [(n, _P) for n in _OUT_COEF] + [
        ("metric_arrays", _P),
        ("st_w", _P), ("st_phi", _P), ("st_cx", _P), ("st_cy", _P),
        ("ig_index", C.POINTER(C.c_int64)), ("ig_weight", _P),
        ("ss_phi", _P), ("ss_w", _P),
        ("max_iterations", C.c_int32), ("average_iterations", C.c_double),
        ("computation_time_s", C.c_double), ("table_time_s", C.c_double),
        ("step_times", _P),
    ]


def _ptr(a: np.ndarray, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct))


_libs: dict[str, C.CDLL] = {}


def library(kind: str = "oracle") -> C.CDLL:
    """kind: 'oracle' (C restatement), 'ref_fast' or 'ref_strict' (reference)."""
    if kind in _libs:
        return _libs[kind]
    if kind == "oracle":
        path, sym = HERE / "liboracle.so", "oracle_run"
    else:
        path, sym = HERE / "_ref" / f"lib{kind}.so", "ref_run"
    if not path.exists():
        raise FileNotFoundError(f"{path} is not built (run __graft_entry__.build())")
    lib = C.CDLL(str(path))
    fn = getattr(lib, sym)
    fn.argtypes = [C.POINTER(Params), C.POINTER(Inputs), C.POINTER(Outputs)]
    fn.restype = C.c_int
    lib.run_fn = fn
    _libs[kind] = lib
    return lib


def set_frames(kind: str, write_period: float | None, workdir: str | None):
    """Frame output of the reference's RunSimulation (run(..., use_run_simulation=True)):
    every write_period, written under <workdir>/../output/ref_run/Moments/;
    workdir None turns it off.  Reference libraries only."""
    lib = library(kind)
    lib.ref_set_frames.argtypes = [C.c_double, C.c_char_p]
    lib.ref_set_frames.restype = None
    lib.ref_set_frames(float(write_period or 1e300), workdir.encode() if workdir else None)


def write_frame(kind: str, case: dict, time: float, r, g, b, a, directory: str, name: str = ""):
    """The reference's Grid::WriteFrametoCsv for host arrays (reference libraries only)."""
    lib = library(kind)
    lib.ref_write_frame.argtypes = [C.POINTER(Params), C.c_float] + [C.POINTER(C.c_double)] * 4 + \
        [C.c_char_p, C.c_char_p]
    lib.ref_write_frame.restype = C.c_int
    p = Params(nx_=int(case["nx_"]), ny_=int(case["ny_"]), startx=case["start"][0], starty=case["start"][1],
               endx=case["end"][0], endy=case["end"][1], cfl=case["cfl"])
    arrs = [np.ascontiguousarray(x, dtype=np.float64) for x in (r, g, b, a)]
    return lib.ref_write_frame(C.byref(p), float(time), *[_ptr(x) for x in arrs], directory.encode(), name.encode())


def available(kind: str) -> bool:
    try:
        library(kind)
        return True
    except (FileNotFoundError, OSError):
        return False


def run(case: dict, kind: str = "oracle", metric_override: np.ndarray | None = None,
        want_metric: bool = False, use_run_simulation: bool = False, n_threads: int = 0,
        update_tables_each_step: bool = False) -> dict:
    """Run one case (a dict as built by the package's ``workloads`` module).

    Returns every output of oracle/ref_api.h as numpy arrays (node arrays of
    shape (ny, nx) flattened as ij = i + j*nx, intensities cell-major)."""
    nx = int(case["nx_"]) + 2
    ny = int(case["ny_"]) + 2
    nxy = nx * ny
    nd = int(case["n_dir"])
    nf = int(case["n_fourier"])
    p = Params(
        nx_=int(case["nx_"]), ny_=int(case["ny_"]),
        startx=case["start"][0], starty=case["start"][1],
        endx=case["end"][0], endy=case["end"][1], cfl=case["cfl"],
        metric_kind=int(case["metric_kind"]), m=case["m"], a=case["a"],
        excision=case["excision"], n_dir=nd, n_fourier=nf,
        streaming_type=int(case["streaming_type"]),
        initial_data_type=int(case["initial_data_type"]),
        keep_source_nodes_active=int(case["keep_source_nodes_active"]),
        n_steps=int(case["n_steps"]), rk_tol=case["rk_tol"],
        use_run_simulation=int(use_run_simulation), n_threads=n_threads,
        update_tables_each_step=int(update_tables_each_step),
    )
    f = case["fields"]
    keep = []

    def arr(name, n):
        a = np.ascontiguousarray(f[name], dtype=np.float64).reshape(-1)
        assert a.size == n, (name, a.size, n)
        keep.append(a)
        return _ptr(a)

    mask = np.ascontiguousarray(f["is_initial"], dtype=np.uint8).reshape(-1)
    keep.append(mask)
    mo = None
    if metric_override is not None:
        mo = np.ascontiguousarray(metric_override, dtype=np.float64).reshape(-1)
        assert mo.size == N_METRIC_ARRAYS * nxy
        keep.append(mo)
    inp = Inputs(
        kappa0=arr("kappa0", nxy), kappa1=arr("kappa1", nxy), kappaA=arr("kappaA", nxy),
        eta=arr("eta", nxy), ux=arr("ux", nxy), uy=arr("uy", nxy),
        is_initial=_ptr(mask, C.c_uint8), initial_I=arr("initial_I", nxy * nd),
        initial_E_LF=arr("initial_E_LF", nxy), initial_Fx_LF=arr("initial_Fx_LF", nxy),
        initial_Fy_LF=arr("initial_Fy_LF", nxy), initial_Pxx_LF=arr("initial_Pxx_LF", nxy),
        initial_Pxy_LF=arr("initial_Pxy_LF", nxy), initial_Pyy_LF=arr("initial_Pyy_LF", nxy),
        metric_override=_ptr(mo) if mo is not None else None,
    )
    res: dict = {n: np.zeros(nxy) for n in _OUT_NODE}
    res["I"] = np.zeros(nxy * nd)
    for n in _OUT_COEF:
        res[n] = np.zeros(nxy * nf)
    res["metric_arrays"] = np.zeros(N_METRIC_ARRAYS * nxy) if want_metric else None
    for n in ("st_w", "st_phi", "st_cx", "st_cy"):
        res[n] = np.zeros(nd)
    res["ig_index"] = np.zeros(4 * 10 * nd, dtype=np.int64)
    res["ig_weight"] = np.zeros(4 * 10 * nd)
    res["ss_phi"] = np.zeros(nf)
    res["ss_w"] = np.zeros(nf)
    res["step_times"] = np.zeros(max(int(case["n_steps"]), 1))
    out = Outputs(**{k: (_ptr(v, C.c_int64) if v.dtype == np.int64 else _ptr(v))
                     for k, v in res.items() if v is not None})
    lib = library(kind)
    rc = lib.run_fn(C.byref(p), C.byref(inp), C.byref(out))
    if rc != 0:
        raise RuntimeError(f"{kind} run failed with status {rc}")
    res["max_iterations"] = int(out.max_iterations)
    res["average_iterations"] = float(out.average_iterations)
    res["computation_time_s"] = float(out.computation_time_s)
    res["table_time_s"] = float(out.table_time_s)
    res["nx"], res["ny"] = nx, ny
    if want_metric:
        res["metric_arrays"] = res["metric_arrays"].reshape(N_METRIC_ARRAYS, nxy)
    return res


def reference_root() -> str:
    """Where the reference tree is read from: $GRLBM_REFERENCE, else the
    default of the build recipe (oracle/Makefile, REF ?= ...)."""
    env = os.environ.get("GRLBM_REFERENCE")
    if env:
        return env
    for line in (HERE / "Makefile").read_text().splitlines():
        if line.startswith("REF ?="):
            return line.split("=", 1)[1].strip()
    return ""


def build(with_reference: bool | None = None, ref_root: str | None = None) -> None:
    """Build liboracle.so, and the reference libraries when the reference tree
    is present (or when with_reference is True).  With the reference, also the
    beam demo of the C++ class (target `facade`) when libgrlbm.so exists."""
    import subprocess
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    ref_root = ref_root or reference_root()
    if with_reference is None:
        with_reference = bool(ref_root) and os.path.isdir(os.path.join(ref_root, "src"))
    if with_reference:
        subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REF={ref_root}"], check=True)
        if (HERE.parent / "2dradiation_b200" / "libgrlbm.so").exists():
            subprocess.run(["make", "-s", "-C", str(HERE), "facade", f"REF={ref_root}"], check=True)
