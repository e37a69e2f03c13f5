"""Host-side pieces of the learned closure that need no GPU: the training
targets (face transfers from a depth difference), parameter layout and
initialisation, and the C ABI symbols."""
import ctypes
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import silt_closure as C
import silt_closure_train as T

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_divergence_moves_depth_between_neighbours_only():
    g = torch.Generator().manual_seed(3)
    gx = torch.randn((3, C.CROP, C.CROP), generator=g, dtype=torch.float64)
    gz = torch.randn((3, C.CROP, C.CROP), generator=g, dtype=torch.float64)
    gx[..., :, -1] = 0.0
    gz[..., -1, :] = 0.0
    d = T.divergence(gx, gz)
    assert float(d.sum(dim=(-2, -1)).abs().max()) < 1e-9  # volume neutral
    # One transfer to +x from (row 4, col 7): 7 loses it, 8 gains it.
    gx = torch.zeros((C.CROP, C.CROP), dtype=torch.float64)
    gz = torch.zeros_like(gx)
    gx[4, 7] = 0.5
    d = T.divergence(gx, gz)
    assert float(d[4, 7]) == -0.5 and float(d[4, 8]) == 0.5 and float(d.abs().sum()) == 1.0


def test_parameter_layout_and_init():
    assert C.NPARAM == 18512
    p = C.init_params(seed=1)
    assert p.size == C.NPARAM and p.dtype == np.float32
    P = C.split_params(torch.tensor(p))
    assert tuple(P["W1"].shape) == (9, 16, 32) and tuple(P["W3"].shape) == (9, 32, 16)
    assert float(P["W1"][:, C.IN_USED:, :].abs().max()) == 0.0
    assert float(P["W3"][:, :, C.OUT_USED:].abs().max()) == 0.0


def test_crop_clips_at_the_window_edge():
    plane = torch.arange(50 * 50, dtype=torch.float32).view(50, 50)
    c = T.crop(plane, -4, 30)
    assert float(c[0, 0]) == 0.0 and float(c[0, 4]) == float(plane[30, 0])
    assert float(c[19, 4]) == float(plane[49, 0]) and float(c[20, 4]) == 0.0


def test_closure_header_symbols_exported():
    import re

    text = open(os.path.join(ROOT, "include", "silt_closure.h")).read()
    names = sorted(set(re.findall(r"^\s*int\s+(silt_\w+)\s*\(", text, re.M)))
    assert len(names) >= 10
    lib = ctypes.CDLL(os.path.join(ROOT, "dirty-gen_b200", "libsilt_b200.so"))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(C._SIGS), sorted(set(names) - set(C._SIGS))
