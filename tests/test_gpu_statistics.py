"""Statistical parity of the GPU heatbath chains with the reference's chain, at 2 sigma.

The reference updates links in lexicographic order with frozen block-face links and a
random translation before every sweep, drawing from std::mt19937_64
(src/heatbath/heatbath_mpi.cpp:37-69, src/mpi/Shift.cpp:163-186).  The oracle restates that
schedule exactly for one rank, and tests/golden/ref_schedule_plaquette.json holds its chains'
statistics (8 independent chains per case; make_ref_schedule_plaquette.py beside it).  The
library updates every link by checkerboard passes with Philox draws.  Both are Gibbs
samplers of the same Wilson action on the same periodic lattice, so after thermalisation
their mean plaquettes must agree.

For each lattice size (4^4, 8^4), beta (5.7, 6.0, 6.2) and storage (FP64 18-real, and the
FP32 12-real form that the benchmark measures), 16 independent GPU chains run in one batch
from cold starts, as the reference chains do (on these small boxes beta 6.0 and 6.2 lie above
the finite-volume deconfinement transition, where a hot start can leave a chain in a
metastable twisted state for longer than the run).  Each chain's integrated autocorrelation
time tau_int is measured; the bin length is at least 10 times the largest tau_int of the
chains, so bin means are independent.  The error of a mean is the larger of the pooled-bin
error and the scatter of the chain means.  z = |mean_gpu - mean_ref| / sqrt(err_gpu^2 +
err_ref^2) must be below 2.  Seeds are fixed, so every run computes the same z.  With
QCB_STATS_TABLE set to a path, the table of means, errors, tau_int and z is written there as
markdown.
"""
import json
import os
from pathlib import Path

import numpy as np
import pytest

import qcb
from stats import chains_estimate, chains_summary

pytestmark = pytest.mark.gpu

GOLD = json.loads((Path(__file__).resolve().parent / "golden" / "ref_schedule_plaquette.json").read_text())
CASES = {(c["L"], c["beta"]): c for c in GOLD["cases"]}
N_CHAINS = 16
SWEEPS = {4: 20000, 8: 6000}
THERM = {4: 2000, 8: 1000}
STORAGES = [("fp64", 18), ("fp32", 12)]
ROWS = []


def gpu_chains(ctx, L, beta, prec, nr):
    """Plaquette after every sweep of N_CHAINS independent lattices, shape (chains, sweeps)."""
    fields = [qcb.GaugeField(ctx, (L, L, L, L), prec, nr) for _ in range(N_CHAINS)]
    seeds = [7000 + 100 * L + int(round(beta * 10)) * 1000 + k for k in range(N_CHAINS)]
    for f in fields:
        f.cold_start()
    batch = qcb.Batch(ctx, fields)
    betas = [beta] * N_CHAINS
    batch.heatbath(betas, THERM[L], 1, seeds, [0] * N_CHAINS)
    n = SWEEPS[L]
    out = np.empty((n, N_CHAINS))
    for s in range(n):
        batch.heatbath(betas, 1, 1, seeds, [THERM[L] + s] * N_CHAINS)
        out[s] = batch.plaquette()
    batch.close()
    for f in fields:
        f.close()
    return out.T


@pytest.mark.parametrize("prec,nr", STORAGES)
@pytest.mark.parametrize("L,beta", sorted(CASES))
def test_mean_plaquette_agrees_with_reference_chain(ctx, L, beta, prec, nr):
    ref = CASES[(L, beta)]
    mr, er, nbr = chains_estimate(ref["bins"])
    g = chains_summary(gpu_chains(ctx, L, beta, prec, nr))
    mg, eg, _ = chains_estimate(g["bins"])
    z = abs(mg - mr) / np.hypot(eg, er)
    row = (f"| {L}^4 | {beta} | {prec}-{nr} | {mg:.6f} ± {eg:.6f} | {max(g['tau_int']):.2f} | "
           f"{g['bin_length']} | {g['n_bins']} | {mr:.6f} ± {er:.6f} | {max(ref['tau_int']):.2f} | "
           f"{ref['bin_length']} | {nbr} | {z:.2f} |")
    ROWS.append(row)
    print(row)
    path = os.environ.get("QCB_STATS_TABLE")
    if path:
        head = ("| lattice | beta | GPU storage | GPU mean ± err | GPU tau_int (max) | GPU bin | GPU bins | "
                "reference-schedule mean ± err | ref tau_int (max) | ref bin | ref bins | z |\n"
                "|---|---|---|---|---|---|---|---|---|---|---|---|\n")
        Path(path).write_text(head + "\n".join(ROWS) + "\n")
    # bins of at least 10 tau_int and enough of them for the error estimate
    assert g["bin_length"] >= 10 * max(g["tau_int"]) and g["n_bins"] >= 100
    assert ref["bin_length"] >= 10 * max(ref["tau_int"]) and nbr >= 100
    assert z < 2.0, row
    assert 0.45 < mg < 0.7
