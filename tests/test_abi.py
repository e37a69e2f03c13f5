"""The C ABI library builds for sm_100a, loads without a GPU, and exports
every function include/silt_sheet.h declares."""
import ctypes
import os

import silt_b200


def test_library_exports_every_declared_symbol():
    names = silt_b200.header_functions()
    assert len(names) >= 30
    lib = ctypes.CDLL(silt_b200.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_built_for_sm100a_only():
    """The build recipe compiles every kernel for sm_100a and nothing else."""
    mk = open(os.path.join(os.path.dirname(silt_b200.LIB_PATH), "Makefile")).read()
    arch = [ln for ln in mk.splitlines() if ln.startswith("ARCH")]
    assert arch and "arch=compute_100a,code=sm_100a" in arch[0], arch
    assert "sm_90" not in mk and "compute_90" not in mk


def test_binding_declares_every_header_function():
    lib = silt_b200.lib()
    for n in silt_b200.header_functions():
        assert getattr(lib, n).restype is not None or n in ("silt_cfg_default",)


def test_window_origin_matches_the_oracle_snap():
    """silt_window_origin is host code (FluidCore::window_origin,
    src/fluid_core.rs:6987-6990): the same snap as the oracle's window."""
    import oracle

    for c in ((0.0, 0.0), (3.3, -7.1), (-125.07, 40.93), (0.1, 0.1), (19.9999, -0.0001)):
        assert silt_b200.window_origin(c) == oracle.Core(center=c).origin(), c


def test_known_exact_divisors_need_no_device():
    """The table of divisors taken as checked is host data: 2 cell, cell^2,
    231 and cell of the 0.2 m and 0.02 m sheets, each once."""
    import numpy as np

    got = silt_b200.known_exact_divisors()
    f = np.float32
    assert len(got) == len(set(got)) == 7
    assert float(f(0.2) * f(0.2)) in got and float(f(0.02) * f(0.02)) in got and 231.0 in got
