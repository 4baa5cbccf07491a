"""End-to-end run of the drop-in driver gauge_hb_ncb on the plain-method workload.

Workload: one 8^4 lattice (L_core=8, n_core_dims=1), beta=6.0, cold start, seed=1234,
N_sweeps=1, N_hits=1, N_shift_therm=0, N_shift=200 with the plaquette every shift; then the
Wilson flow on the saved final configuration (eps=0.02, N_steps_gf=50, N_rk_steps=1), FP64,
compared with the oracle on that same configuration to 1e-12.  The output files follow the
reference's formats (src/io/io.cpp:20-105, 233-287, 725-772), and a second invocation
resumes the chain exactly.
"""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

import oracle as orc
import qcb

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
DRIVER = ROOT / "ecmc-qncb_b200" / "bin" / "gauge_hb_ncb"

INPUT = """#Lattice params
L_core=8
n_core_dims=1
cold_start=true

#Run params
seed=1234
N_shift_therm = 0
N_shift={n_shift}
N_switch_eo=1

#Heatbath params
beta = 6.0
N_sweeps = 1
N_hits = 1

#Plaquette params
N_shift_plaquette = 1

#Topo params
topo = {topo}
N_shift_topo = 100
N_steps_gf = 5
N_rk_steps = 2

#Save params
run_name = plain8
run_dir = {run_dir}
save_each_shifts = 100
"""


def run_driver(tmp_path, n_shift, topo="false"):
    inp = tmp_path / f"in_{n_shift}.txt"
    inp.write_text(INPUT.format(n_shift=n_shift, topo=topo, run_dir=tmp_path / "data"))
    r = subprocess.run([str(DRIVER), str(inp)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def test_driver_plain_method_and_resume(ctx, tmp_path):
    out = run_driver(tmp_path, 200)
    run = tmp_path / "data" / "plain8"
    plaq = (run / "plain8_plaquette.txt").read_text().splitlines()
    assert len(plaq) == 200
    assert all(re.fullmatch(r"\d\.\d{10}", line) for line in plaq)
    params = (run / "plain8_params.txt").read_text()
    assert "L_core=8" in params and "cold_start=true" in params and "N_shift_therm = 0" in params
    assert params.count("Saved shift 100") == 1 and params.count("Saved shift 200") == 1
    assert params.rstrip().endswith("Saved final state !")
    assert "Elapsed time : " in out
    seed_text = (run / "plain8_seed" / "plain8_seed0.txt").read_text().split()
    assert seed_text[0] == "qcb-philox4x32-10" and seed_text[2] == "200"

    # the saved configuration is the chain of 200 checkerboard sweeps from a cold start
    dims = (8, 8, 8, 8)
    f = qcb.GaugeField(ctx, dims)
    f.load_ildg(run / "plain8")
    assert abs(qcb.observables.mean_plaquette_global(f) - float(plaq[-1])) < 1e-10
    g = qcb.GaugeField(ctx, dims)
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(g.h, 6.0, 200, 1, 1234, 0))
    assert np.array_equal(g.get_links(), f.get_links())

    # flow on the final configuration: FP64 parity with the oracle (N_steps_gf=50, N_rk=1)
    u = f.get_links()
    got = qcb.observables.topo_charge_flowed(f, qcb.GradientFlow(0.02), 50, 1).reshape(-1, 3)
    ref = orc.flow_measure(u, dims, 0.02, 50, 1).reshape(-1, 3)
    assert np.abs(got[:, 1] - ref[:, 1]).max() < 1e-12 * max(1.0, np.abs(ref[:, 1]).max())
    assert np.abs(got[:, 2] - ref[:, 2]).max() < 1e-12 * ref[:, 2].max()
    assert abs(orc.plaquette(u, dims) - float(plaq[-1])) < 1e-10

    # resume: 10 more shifts continue the same Philox stream (sweeps 200..209)
    out2 = run_driver(tmp_path, 10, topo="true")
    assert "Resuming" in out2
    plaq2 = (run / "plain8_plaquette.txt").read_text().splitlines()
    assert len(plaq2) == 210
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(g.h, 6.0, 10, 1, 1234, 200))
    h = qcb.GaugeField(ctx, dims)
    h.load_ildg(run / "plain8")
    assert np.array_equal(g.get_links(), h.get_links())
    topo = (run / "plain8_topo.txt").read_text().splitlines()
    assert len(topo) == 5  # one measurement (shift 0) of N_steps_gf = 5 records
    t, q, e = (float(v) for v in topo[1].split())
    assert abs(t - 0.04) < 1e-12 and e > 0

