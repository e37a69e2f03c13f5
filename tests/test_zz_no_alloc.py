"""silt_step_sheet_noalloc: the free step_sheet operator for callers that may
not allocate GPU memory (a frame loop on a fixed time budget, where cudaFree
would wait for the whole device, or a host whose GPU memory belongs to another
allocator). Its scratch is a fixed array inside the library, so it must give
the same result as silt_step_sheet with caller scratch, call after call.

This file sorts last so that, when it fails, a run that stops at the first
failure has already run every other test."""
import ctypes

import numpy as np
import pytest

import silt_b200 as G

pytestmark = pytest.mark.gpu
TOL_H = 1.0e-4


def scene(res):
    jj, ii = np.mgrid[0:res, 0:res]
    bed = (-0.02 * jj + 0.03 * np.sin(ii * 0.2)).astype(np.float32).ravel()
    h = np.where(((ii - res / 2) ** 2 + (jj - res / 3) ** 2) < (res / 4) ** 2, 0.06, 0.0).astype(np.float32).ravel()
    nu = np.full(res * res, 0.9, np.float32)
    nu[: res * res // 3] = 228.0
    return h, bed, nu


def test_noalloc_matches_caller_scratch_on_two_calls():
    import torch

    res, cell, dt, vort = 96, 0.2, 1.0 / 60.0, 0.08
    h, bed, nu = scene(res)
    n = res * res
    a = [torch.tensor(x, device="cuda") for x in (h, np.zeros(n, np.float32), np.zeros(n, np.float32))]
    b = [t.clone() for t in a]
    dbed = torch.tensor(bed, device="cuda")
    dnu = torch.tensor(nu, device="cuda")
    gate = torch.ones(n, dtype=torch.uint8, device="cuda")
    scratch = torch.zeros(G.lib().silt_step_sheet_scratch_bytes(res) // 4 + 64, dtype=torch.float32, device="cuda")
    for call in range(2):
        G.check(G.lib().silt_step_sheet(a[0].data_ptr(), a[1].data_ptr(), a[2].data_ptr(), dbed.data_ptr(),
                                        dnu.data_ptr(), gate.data_ptr(), res, cell, dt, vort, scratch.data_ptr(), None),
                "step_sheet")
        G.check(G.lib().silt_step_sheet_noalloc(b[0].data_ptr(), b[1].data_ptr(), b[2].data_ptr(), dbed.data_ptr(),
                                                dnu.data_ptr(), gate.data_ptr(), res, cell, dt, vort, None),
                "step_sheet_noalloc")
        torch.cuda.synchronize()
        for x, y in zip(a, b):
            assert float((x - y).abs().max()) <= TOL_H, call
        assert float(b[0].sum()) > 0.0


def test_noalloc_refuses_grids_above_its_limit():
    res = G.lib().silt_step_sheet_noalloc  # bound
    big = 257
    rc = res(None, None, None, None, None, None, big, 0.2, 0.01, 0.0, None)
    assert rc == G.SILT_EINVAL
    assert b"up to 256" in G.lib().silt_last_error()
