"""The FP64 restatement of the oracle (the same source built with
-DORACLE_F64): the nested-sheet oracle that the learned closure's errors are
stated against. It must be the f32 step's model in double precision: close to
the f32 oracle on the reference's window, with the volume books of a step
closing to double rounding."""
import numpy as np

import oracle as O
import silt_scenes as S

DT = 1.0 / 120.0


def test_fp64_oracle_tracks_the_f32_oracle_on_window200():
    sc = S.window200()
    a, b = O.Core(), O.Core64()
    for c in (a, b):
        S.seed_core(c, sc)
    for _ in range(50):
        a.step(DT)
        b.step(DT)
    wb = b.get("water")
    assert wb.dtype == np.float64
    d = float(np.abs(a.get("water").astype(np.float64) - wb).max())
    assert 0.0 < d < 1e-5, d
    assert float(np.abs(a.get("slurry").astype(np.float64) - b.get("slurry")).max()) < 1e-5


def test_fp64_oracle_conserves_to_double_rounding():
    """A window covered everywhere (a 5 cm sheet with a 5 cm mound, so no cell
    dries and the dry cut removes nothing): the FP64 books close per step to
    double rounding, far below the f32 step's own rounding."""
    sc = S.window200()
    x = np.arange(200, dtype=np.float32) * np.float32(0.2) - np.float32(19.9)
    X, Z = np.meshgrid(x, x)
    water = (np.float32(0.05) + np.float32(0.05) * np.exp(-(X * X + Z * Z) / np.float32(8.0))).astype(np.float32)
    worst = {}
    for cls in (O.Core, O.Core64):
        c = cls()
        c.map_water_bed(sc["bed"], water.ravel())
        prev, w = None, 0.0
        for _ in range(40):
            c.step(DT)
            v = c.ledger()["water64"]
            if prev is not None:
                w = max(w, abs(v - prev) / v)
            prev = v
        worst[cls.__name__] = w
    assert worst["Core64"] < 1e-12, worst
    assert worst["Core"] > 10 * worst["Core64"], worst
