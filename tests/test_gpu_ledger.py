"""The FP64 books over long runs, and the rounding book.

The state is the reference's f32 arithmetic, so a step's cell updates do not
conserve volume exactly: each transport update rounds. The books close the
rest exactly in FP64 (the dry cut, spray, inflow and parking have their own
books), and the transport's rounding is booked too (round_m3: each updated
cell's f32 change less the exact sum of its face fluxes). Per step the gap is
|(total + cut - opened) now - before| / total; with the rounding book taken
off, a sheet whose only depth updates are transport and the dry cut closes to
FP64 summation rounding."""
import numpy as np
import pytest

import silt_b200 as G
import silt_scenes as S

pytestmark = pytest.mark.gpu
DT = 1.0 / 120.0


def kept(led, with_round):
    v = led["total_m3"] + led["cut_m3"] - led["opened_m3"]
    return v - led["round_m3"] if with_round else v


@pytest.mark.parametrize("engine", [G.ENGINE_WINDOW, G.ENGINE_GRID])
def test_rounding_book_closes_transport_to_fp64(engine):
    dev = G.Sheet(engine=engine)
    S.seed_core(dev, S.window200())
    prev = dev.ledger()
    raw = booked = 0.0
    for _ in range(60):
        dev.step(DT, want_spray=False)
        led = dev.ledger()
        raw = max(raw, abs(kept(led, False) - kept(prev, False)) / led["total_m3"])
        booked = max(booked, abs(kept(led, True) - kept(prev, True)) / led["total_m3"])
        prev = led
    print(f"engine {engine}: gap per step {raw:.3e}, after the rounding book {booked:.3e}, "
          f"round_m3 {prev['round_m3']:.3e}")
    assert prev["round_m3"] != 0.0
    assert booked < 1e-13, (raw, booked)
    assert raw > 10 * booked


def test_grid2048_ledger_over_1000_steps():
    """The benchmark scene (2048^2, eight puddles, inflow, four tire patches)
    for 1000 steps: the per-step gap of the books, raw and after the rounding
    book, every step."""
    dev = G.Sheet(res=2048, fine_res=64, layout=G.FINE_PER_TIRE)
    S.seed_core(dev, S.grid(res=2048))
    dev.set_inflow(0, -2.0, 2.0, 0.5)
    prev = dev.ledger()
    raw, booked = [], []
    for k in range(1000):
        for t in S.tires_at(k * DT, speed=5.0):
            dev.push_tire(**t)
        dev.step(DT, want_spray=False)
        led = dev.ledger()
        raw.append(abs(kept(led, False) - kept(prev, False)) / led["total_m3"])
        booked.append(abs(kept(led, True) - kept(prev, True)) / led["total_m3"])
        prev = led
    print(f"1000 steps: gap max {max(raw):.3e} median {np.median(raw):.3e}; after the rounding book "
          f"max {max(booked):.3e} median {np.median(booked):.3e}; round_m3 {prev['round_m3']:.3e}")
    # The transport's rounding is only part of this scene's gap: the nested
    # patches' coupling and the near-field tiles round too, so the booked
    # figure is reported beside the raw one, not required to be smaller.
    assert max(raw) < 1e-8
    assert max(booked) < 1e-8
