"""End-to-end runs of the drop-in event-chain driver gauge_ecmc_ncb
(src/bin/gauge_ecmc_ncb.cpp:20-317) on the reference's own example input inputs/ecold6.txt
(8^4 as 16 blocks of 4^4, beta 6.0, cold start, theta_sample 1000): the output files follow
the reference's formats (src/io/io.cpp:20-105, 49-75, 140-192, 577-627), the saved
configuration equals the same schedule replayed through the Python mirror, and a run split
in two invocations (resume) ends on the same configuration as one run.
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
DRIVER = ROOT / "ecmc-qncb_b200" / "bin" / "gauge_ecmc_ncb"

INPUT = """#Lattice params
L_core=4
n_core_dims=2
cold_start=true

#Run params
seed=12345
N_shift_therm = {n_therm}
N_shift={n_shift}

#ECMC params
beta=6.0
param_theta_sample=1000
param_theta_refresh_site=500
param_theta_refresh_R=3.3
poisson=false
epsilon_set=0.15

#Plaquette params
N_shift_plaquette = 2

#Topo params
topo = {topo}
N_shift_topo = 4
N_steps_gf = 3
N_rk_steps = 2

#Save params
run_name = ecold
run_dir = {run_dir}
save_each_shifts = 2000
"""


def run_driver(run_dir, n_shift, n_therm=0, topo="true"):
    run_dir.mkdir(parents=True, exist_ok=True)
    inp = run_dir / f"in_{n_shift}.txt"
    inp.write_text(INPUT.format(n_shift=n_shift, n_therm=n_therm, topo=topo, run_dir=run_dir))
    r = subprocess.run([str(DRIVER), str(inp)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return r.stdout


def test_outputs_and_replay(ctx, tmp_path):
    out = run_driver(tmp_path / "a", 8, n_therm=2)
    run = tmp_path / "a" / "ecold"
    plaq = [float(x) for x in (run / "ecold_plaquette.txt").read_text().split()]
    assert len(plaq) == 4
    assert all(re.fullmatch(r"\d\.\d{10}", s) for s in (run / "ecold_plaquette.txt").read_text().split())
    ev = [line.split() for line in (run / "ecold_nbevent.txt").read_text().splitlines()]
    assert len(ev) == 4 and all(len(e) == 4 for e in ev)
    events, lifts, revs, lam = (int(ev[0][0]), int(ev[0][1]), int(ev[0][2]), float(ev[0][3]))
    assert events >= lifts > revs >= 0 and lam > 0
    # lambda = N_shift_plaquette * theta_sample * ranks / total lifts; ev holds per-rank averages
    assert abs(lam * lifts / (2 * 1000.0) - 1.0) < 0.05
    topo = np.loadtxt(run / "ecold_topo.txt")
    assert topo.shape == (2 * 3, 3)
    params = (run / "ecold_params.txt").read_text()
    assert "theta_sample = 1000" in params and "poisson = false" in params and "N_shift_therm = 2" in params
    assert params.rstrip().endswith("Saved final state !")
    assert "Average λ" in out and "Shift (" in out
    states = sorted((run / "ecold_state").glob("ecold_state*.txt"))
    seeds = sorted((run / "ecold_seed").glob("ecold_seed*.txt"))
    assert len(states) == 16 and len(seeds) == 16
    first = (run / "ecold_state" / "ecold_state0.txt").read_text().splitlines()
    assert len(first) == 4 and len(first[0].split()) == 12 and all(len(r.split()) == 6 for r in first[1:])
    site = int(first[0].split()[0])
    c = [(site // 6 ** k) % 6 for k in range(4)]  # padded (L_core + 2)^4 block index
    assert all(1 <= v <= 4 for v in c)

    # replay: the same translations (std::mt19937_64(seed), uniform in [0, L_core)) and the
    # same chains through the Python mirror give the saved configuration bit for bit
    dims = (8, 8, 8, 8)
    shifts = orc.shift_sequence(12345, 4, 10).reshape(10, 4)
    f = qcb.GaugeField(ctx, dims)
    f.cold_start()
    ch = qcb.EventChains(f, qcb.ecmc.params(theta_sample=1000.0, theta_refresh_site=500.0, theta_refresh_R=3.3,
                                            l_core=4), 12345)
    cum = np.zeros(4, int)
    got_plaq = []
    for i, s in enumerate(shifts):
        cum = (cum + s) % 8
        ch.sample(cum)
        if i >= 2 and (i - 2) % 2 == 0:
            got_plaq.append(qcb.observables.mean_plaquette_global(f))
    f.translate(cum)
    saved = orc.read_ildg(run / "ecold", dims)
    assert np.array_equal(f.get_links(), saved)
    assert np.allclose(got_plaq, plaq, atol=1e-10)
    ch.close()
    f.close()


def test_resume_continues_the_chains(ctx, tmp_path):
    run_driver(tmp_path / "one", 4, topo="false")
    run_driver(tmp_path / "two", 2, topo="false")
    out = run_driver(tmp_path / "two", 2, topo="false")
    assert "Resuming" in out
    dims = (8, 8, 8, 8)
    a = orc.read_ildg(tmp_path / "one" / "ecold" / "ecold", dims)
    b = orc.read_ildg(tmp_path / "two" / "ecold" / "ecold", dims)
    assert np.array_equal(a, b)
