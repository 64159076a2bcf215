"""CPU checks of the measurement helpers of bench.py: the cells a step
updates, the algorithmic bytes of a stage launch, and the error measures of
the report (normwise max and RMS relative error over the prognostic cells)."""
import importlib.util
import os

import numpy as np

from conftest import small_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_prognostic_cells_and_mask_agree():
    b = bench()
    g, _ = small_case(nxp=4, nlev=8, ntr=1)
    mask = b.prognostic_mask(g)
    assert not mask[0].any()                       # the dummy point
    assert int(mask.sum()) == b.prognostic_cells(g)
    assert b.cell_updates(g, 7) == 7 * b.prognostic_cells(g)


def test_stage_bytes():
    b = bench()
    g, _ = small_case(nxp=4, nlev=8, ntr=1)
    c = b.prognostic_cells(g)
    assert b.bytes_per_launch(g, 128, 1) == c * (128 * 12 + 32)
    assert b.bytes_per_launch(g, 128, 2) == c * (128 * 16 + 32)


def test_field_errors():
    b = bench()
    rng = np.random.default_rng(3)
    ref = rng.random((5, 6)) + 1.0
    mask = np.ones_like(ref, bool)
    mask[0] = False
    assert b.field_errors(ref, ref, mask) == (0.0, 0.0)
    out = ref.copy()
    out[2, 3] += 1e-3                              # one cell off
    mx, rms = b.field_errors(out, ref, mask)
    assert abs(mx - 1e-3 / ref[mask].max()) < 1e-15
    assert abs(rms - 1e-3 / np.sqrt((ref[mask] ** 2).sum())) < 1e-15
    out[0, 0] += 5.0                               # outside the mask: ignored
    assert b.field_errors(out, ref, mask)[0] == mx


def test_recomputed_steps():
    b = bench()
    # whole segments: every step once
    assert b.recomputed_steps(24, 6, 0) == 24
    assert b.recomputed_steps(24, 6, 6) == 24
    assert b.recomputed_steps(5, 2, 0) == 5
    # a checkpoint every 12 steps, parts of 4: 12 + 8 + 4 per segment
    assert b.recomputed_steps(24, 12, 4) == 2 * (12 + 8 + 4)
    # a ragged last segment and part: segments [0, 3), [3, 5); parts of 1
    assert b.recomputed_steps(5, 3, 1) == (3 + 2 + 1) + (2 + 1)


def test_clock_samples_of_the_timed_region():
    """Only samples that arrive after begin() count; throttle reasons are
    read from the active columns."""
    b = bench()

    class FakeProc:
        def terminate(self):
            pass

        def wait(self, timeout=None):
            return 0

        def poll(self):
            return 0

    c = b.Clocks(0)
    c.proc = FakeProc()
    c.t0 = 10.0
    row = "0, {sm}, 1965, 700.0, 0x0, Not Active, Not Active, Not Active, {cap}"
    c.lines = [(9.0, row.format(sm=900, cap="Not Active")),      # warm-up: left out
               (10.1, row.format(sm=1900, cap="Not Active")),
               (10.2, row.format(sm=1800, cap="Active")),
               (10.3, "garbled")]
    r = c.stop()
    assert r["samples"] == 2
    assert r["sm_mhz"] == 1850.0 and r["sm_max_mhz"] == 1965.0
    assert r["reasons"] == ["sw_power_cap"]
