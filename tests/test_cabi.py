"""The C-ABI library loads without a GPU, exports every entry point that
include/*.h declares, and rejects bad arguments with status codes (it never
exits the process)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(grlbm_\w+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "grlbm_create" in syms and "grlbm_step" in syms and len(syms) >= 20


def test_library_exports_every_declared_symbol(grlbm):
    lib = grlbm.lib()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_python_signatures_cover_header(grlbm):
    assert set(declared_symbols()) <= set(grlbm.SIGNATURES)


def _create(grlbm, case, **over):
    g, m = grlbm.grid_desc(case), grlbm.metric_desc(case)
    r = grlbm.RunDesc(int(case["n_dir"]), int(case["n_fourier"]), int(case["streaming_type"]), 0,
                      int(case["keep_source_nodes_active"]), int(case["initial_data_type"]))
    for k, v in over.items():
        for s in (g, m, r):
            if hasattr(s, k):
                setattr(s, k, v)
    h = C.c_void_p()
    rc = grlbm.lib().grlbm_create(C.byref(g), C.byref(m), C.byref(r), -1, C.byref(h))
    msg = grlbm.lib().grlbm_last_error(None).decode()
    if h:
        grlbm.lib().grlbm_destroy(h)
    return rc, msg


@pytest.mark.parametrize("over,code", [
    (dict(nx_=1), 1), (dict(endx=-7.0), 1), (dict(cfl=0.0), 1), (dict(kind=7), 1),
    (dict(streaming_type=4), 4),
    (dict(streaming_type=9), 1), (dict(n_dir=2), 1), (dict(n_fourier=0), 1), (dict(n_fourier=65), 1),
    (dict(precision=3), 1), (dict(initial_data_type=5), 1),
])
def test_create_rejects_bad_arguments(grlbm, W, over, code):
    rc, msg = _create(grlbm, W.curved_shell(nx_=8, ny_=8, n_dir=8, steps=1), **over)
    assert rc == code, msg
    assert msg


def test_fast_fp64_form_takes_fixed_streaming_only(grlbm, W):
    """GRLBM_FAST_FP64 is refused (unsupported, before any device call) for
    the adaptive streaming types, and for states of 2^31 values or more."""
    case = W.curved_shell(nx_=8, ny_=8, n_dir=8, steps=1)
    for st in (1, 3):
        rc, msg = _create(grlbm, case, precision=2, streaming_type=st)
        assert rc == 4 and "fixed streaming" in msg, msg
    rc, msg = _create(grlbm, case, precision=2, nx_=6000, ny_=6000, n_dir=64)
    assert rc == 1 and "2^31" in msg, msg


@pytest.mark.parametrize("precision", [0, 1, 2])
def test_direction_limit(grlbm, W, precision):
    rc, msg = _create(grlbm, W.curved_shell(nx_=8, ny_=8, n_dir=257, steps=1), precision=precision)
    assert rc == 1 and "n_dir" in msg


def test_host_helpers_reject_bad_arguments(grlbm):
    out = np.zeros(4)
    assert grlbm.lib().grlbm_host_stencil(0, 1, None, None, None, None, None, None) == 1
    assert grlbm.lib().grlbm_host_metric_arrays(None, None, out.ctypes.data_as(C.POINTER(C.c_double))) == 1
    assert grlbm.lib().grlbm_metric_array_count() == 102


def test_null_context_calls_return_argument_error(grlbm):
    L = grlbm.lib()
    assert L.grlbm_step(None, 1) == 1
    assert L.grlbm_update_fourier_coefficients(None, 1e-4, 0) == 1
    assert L.grlbm_get_moments_if(None, None, None, None, None, None, None) == 1
    L.grlbm_destroy(None)  # no-op
