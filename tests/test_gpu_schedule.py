"""The reference's update schedule on one device: frozen block-face links after a
cumulative random shift (qcb_heatbath_frozen), the periodic translation of the field
(qcb_translate), and the driver's `schedule = reference` mode built from the two.

References: frozen links src/geometry/GeometryCB.cpp:33-56, random shift
src/mpi/Shift.cpp:109-186, per-shift sweeps src/bin/gauge_hb_ncb.cpp:116-127.
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as orc
import qcb

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
DRIVER = ROOT / "ecmc-qncb_b200" / "bin" / "gauge_hb_ncb"


def test_frozen_heatbath_matches_oracle_and_reference_count(ctx):
    dims, lcore, shift = (8, 8, 8, 8), 4, (1, 2, 3, 0)
    u = orc.hot_philox(dims, 12)
    f = qcb.GaugeField(ctx, dims)
    f.set_links(u)
    f.heatbath_frozen(6.0, 1, 1, 99, 0, lcore, shift)
    got = f.get_links()
    ref, fails = orc.heatbath_cb_frozen(u, dims, 6.0, 1, 1, 99, 0, lcore, shift)
    assert fails == 0
    assert np.abs(got - ref).max() < 1e-11
    changed = np.any(np.abs(got - u) > 0, axis=(-2, -1))
    # per direction: 8 free values along mu x 3 of 4 values in each of the 3 other directions
    assert int(changed.sum()) == 4 * 8 * 6 ** 3 == 16 * 4 * 4 * 27
    # a frozen link: x = (3, 0, 0, 0) has (x_y + 2) % 4 != 0, (x_z + 3) % 4 != 0 but
    # (x_t + 0) % 4 == 0, so its mu = 0 link stays
    assert np.array_equal(got[0, 0, 0, 3, 0], u[0, 0, 0, 3, 0])


def test_frozen_heatbath_fp32_12_tracks_fp64(ctx):
    dims, lcore, shift = (8, 8, 8, 8), 2, (1, 0, 1, 1)
    u = orc.hot_philox(dims, 3)
    f = qcb.GaugeField(ctx, dims, "fp32", 12)
    f.set_links(u)
    f.heatbath_frozen(6.0, 1, 1, 5, 0, lcore, shift)
    ref, _ = orc.heatbath_cb_frozen(u, dims, 6.0, 1, 1, 5, 0, lcore, shift)
    got = f.get_links()
    assert np.abs(got - ref).max() < 1e-4
    frozen = ~np.any(np.abs(ref - u) > 0, axis=(-2, -1))
    assert np.abs(got - u)[frozen].max() < 1e-6  # frozen links keep their (FP32-rounded) value


def test_translate_matches_roll(ctx):
    dims = (4, 6, 8, 10)
    u = orc.hot_philox(dims, 8)
    for prec, nr, tol in (("fp64", 18, 0.0), ("fp32", 12, 1e-6)):
        f = qcb.GaugeField(ctx, dims, prec, nr)
        f.set_links(u)
        base = f.get_links()
        f.translate((1, -2, 3, 5))
        want = np.roll(base, (5, 3, -2, 1), axis=(0, 1, 2, 3))
        assert np.abs(f.get_links() - want).max() <= tol
        f.close()


def test_frozen_heatbath_rejects_bad_core(ctx):
    f = qcb.GaugeField(ctx, (8, 8, 8, 6))
    with pytest.raises(qcb.QcbError):
        f.heatbath_frozen(6.0, 1, 1, 1, 0, 4, (0, 0, 0, 0))  # 4 does not divide 6
    with pytest.raises(qcb.QcbError):
        f.heatbath_frozen(6.0, 1, 1, 1, 0, 0, (0, 0, 0, 0))


INPUT = """L_core=4
n_core_dims=2
cold_start=false
seed=1234
N_shift_therm = 0
N_shift=6
beta = 6.0
N_sweeps = 1
N_hits = 1
N_shift_plaquette = 1
topo = false
run_name = refsched
run_dir = {run_dir}
save_each_shifts = 100
schedule = reference
"""


def test_driver_reference_schedule(ctx, tmp_path):
    inp = tmp_path / "in.txt"
    inp.write_text(INPUT.format(run_dir=tmp_path / "data"))
    r = subprocess.run([str(DRIVER), str(inp)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    printed = [tuple(int(v) for v in line[len("Shift ("):-1].split(", "))
               for line in r.stdout.splitlines() if line.startswith("Shift (")]
    want = orc.shift_sequence(1234, 4, 6)
    assert np.array_equal(np.array(printed), want)

    # replay: hot start, per shift the cumulative shift and frozen sweeps, one translation
    dims = (8, 8, 8, 8)
    g = qcb.GaugeField(ctx, dims)
    g.hot_start(1234)
    cum = np.zeros(4, np.int64)
    for k, s in enumerate(want):
        cum = (cum + s) % 8
        g.heatbath_frozen(6.0, 1, 1, 1234, k, 4, tuple(int(v) for v in cum))
    g.translate(tuple(int(v) for v in cum))
    h = qcb.GaugeField(ctx, dims)
    h.load_ildg(tmp_path / "data" / "refsched" / "refsched")
    assert np.array_equal(g.get_links(), h.get_links())
    plaq = (tmp_path / "data" / "refsched" / "refsched_plaquette.txt").read_text().split()
    assert len(plaq) == 6 and abs(float(plaq[-1]) - qcb.observables.mean_plaquette_global(h)) < 1e-10
