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


def test_energy_noalloc_matches_energy_on_consecutive_calls(grlbm, W):
    import torch
    case = W.curved_shell(nx_=120, ny_=90, n_dir=16, steps=20)
    with grlbm.prepare(case) as r:
        r.step(20)
        ref = r.energy()
        E = r.moments_if()["E"]
    dev = torch.device("cuda", torch.cuda.current_device())
    dE = torch.from_numpy(np.ascontiguousarray(E)).to(dev)
    out = torch.empty(1, dtype=torch.float64, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    L = grlbm.lib()
    for _ in range(2):  # the shared scratch keeps the previous call's partials
        out.fill_(-1.0)
        rc = L.grlbm_energy_noalloc(C.c_void_p(dE.data_ptr()), 120, 90, C.c_void_p(out.data_ptr()), stream)
        assert rc == 0, L.grlbm_last_error(None)
        torch.cuda.synchronize()
        assert abs(out.item() - ref) <= 1e-12 * abs(ref)


def test_energy_noalloc_rejects_grids_beyond_its_scratch(grlbm):
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    buf = torch.zeros(4, dtype=torch.float64, device=dev)
    L = grlbm.lib()
    rc = L.grlbm_energy_noalloc(C.c_void_p(buf.data_ptr()), 2048, 2048, C.c_void_p(buf.data_ptr()), None)
    assert rc == 1
    assert b"2097152" in L.grlbm_last_error(None)
