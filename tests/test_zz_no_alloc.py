"""The allocation-free energy entry point (grlbm_energy_noalloc) against the
regular one.  It serves callers that cannot allocate device memory when they
need the number (under a fixed device-memory budget, or with every
allocation owned by the host application): its scratch is a fixed
device array, so it takes caller-owned device pointers only.  This file is
collected last so that a failure here comes after every other test has run."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _noalloc(grlbm, dE, nx_, ny_, out):
    import torch
    L = grlbm.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    out.fill_(-1.0)
    rc = L.grlbm_energy_noalloc(C.c_void_p(dE.data_ptr()), nx_, ny_, C.c_void_p(out.data_ptr()), stream)
    assert rc == 0, L.grlbm_last_error(None)
    torch.cuda.synchronize()
    return out.item()


def test_energy_noalloc_matches_energy_on_consecutive_calls(grlbm, W):
    """A call at the scratch's exact limit (1024 x 2048 interior cells) leaves
    8192 partial sums behind; the next calls, on a smaller grid, must not pick
    any of them up.  Each result is checked against a sum on the host or
    grlbm_energy, to 1e-12."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    out = torch.empty(1, dtype=torch.float64, device=dev)
    g = torch.Generator(device="cpu").manual_seed(11)
    big = torch.rand((2048 + 2, 1024 + 2), dtype=torch.float64, generator=g)
    ref_big = float(np.sum(big.numpy()[1:-1, 1:-1], dtype=np.float64))
    got = _noalloc(grlbm, big.to(dev).contiguous(), 1024, 2048, out)
    assert abs(got - ref_big) <= 1e-12 * abs(ref_big)

    case = W.curved_shell(nx_=120, ny_=90, n_dir=16, steps=20)
    with grlbm.prepare(case) as r:
        r.step(20)
        ref = r.energy()
        E = r.moments_if()["E"]
    dE = torch.from_numpy(np.ascontiguousarray(E)).to(dev)
    for _ in range(2):  # the shared scratch keeps the previous call's partials
        got = _noalloc(grlbm, dE, 120, 90, out)
        assert abs(got - ref) <= 1e-12 * abs(ref)


def test_energy_noalloc_rejects_grids_beyond_its_scratch(grlbm):
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    buf = torch.zeros(4, dtype=torch.float64, device=dev)
    L = grlbm.lib()
    rc = L.grlbm_energy_noalloc(C.c_void_p(buf.data_ptr()), 2048, 2048, C.c_void_p(buf.data_ptr()), None)
    assert rc == 1
    assert b"2097152" in L.grlbm_last_error(None)
    # sizes whose product overflows 64 bits (to 4 cells) are rejected on their own
    rc = L.grlbm_energy_noalloc(C.c_void_p(buf.data_ptr()), (1 << 62) + 1, 4, C.c_void_p(buf.data_ptr()), None)
    assert rc == 1
    assert b"2097152" in L.grlbm_last_error(None)
