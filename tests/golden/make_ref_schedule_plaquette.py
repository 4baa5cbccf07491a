"""Generates ref_schedule_plaquette.json: mean-plaquette statistics of the reference's
heatbath chain, as the oracle restates it.

The chain is the reference's single-rank schedule (src/bin/gauge_hb_ncb.cpp:18-179): the
links of local coordinate 0 frozen in every direction d != mu (src/geometry/GeometryCB.cpp:33-56),
a random translation of the field before every sweep (src/mpi/Shift.cpp:163-186), a
lexicographic Cabibbo-Marinari sweep with N_hits = 1 (src/heatbath/heatbath_mpi.cpp:11-69,
src/heatbath/heatbath.cpp:8-44), every draw from one std::mt19937_64 seeded per chain, and
a cold start (every link the identity).  For each lattice size and beta, several independent
chains run; after n_therm discarded sweeps the plaquette of every sweep is recorded.  The
file keeps, per chain, tau_int and the means of bins of at least 10 tau_int sweeps, so a test
recomputes the mean and its error from the file alone.

Cold starts: on these small lattices beta 6.0 and 6.2 (and 5.7 on 4^4) lie at or above the
finite-box deconfinement transition, where a hot start can leave a chain in a metastable state
with twisted Polyakov-loop sectors (a lower plaquette) for far longer than one chain; an
ordered start samples one sector, and all sectors have the same plaquette distribution.

Run from the repository root (about 30 minutes on 8 cores):
    python tests/golden/make_ref_schedule_plaquette.py
or, to regenerate some lattice sizes only and keep the other cases of the existing file:
    python tests/golden/make_ref_schedule_plaquette.py 4
"""
import json
import multiprocessing as mp
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
OUT = HERE / "ref_schedule_plaquette.json"

# (L, n_chains, n_therm, n_sweeps) per lattice size; betas of the statistical oracle.
SIZES = [(4, 32, 2000, 40000), (8, 16, 1000, 5000)]
BETAS = [5.7, 6.0, 6.2]
# Bins are lengthened by a whole factor until a case has at most this many (longer bins are
# still at least 10 tau_int), which keeps the file small.
MAX_BINS = 1000


def seed_of(L: int, beta: float, chain: int) -> int:
    return 100000 * L + 1000 * int(round(beta * 10)) + chain


def run_chain(args):
    L, beta, chain, n_therm, n_sweeps = args
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    c = oracle.RefChain(L, seed_of(L, beta, chain), True)
    c.run(beta, n_therm, 1, 1)
    return (L, beta, chain), c.run(beta, n_sweeps, 1, 1)


def main():
    sys.path.insert(0, str(ROOT / "oracle"))
    sys.path.insert(0, str(ROOT / "tests"))
    import oracle
    from stats import between_chain_err, chains_summary

    oracle.build()
    only = {int(a) for a in sys.argv[1:]}
    sizes = [z for z in SIZES if not only or z[0] in only]
    kept = []
    if only:
        kept = [c for c in json.loads(OUT.read_text())["cases"] if c["L"] not in only]
    jobs = [(L, b, k, th, n) for (L, nc, th, n) in sizes for b in BETAS for k in range(nc)]
    series = {}
    with mp.get_context("spawn").Pool() as pool:
        for key, x in pool.imap_unordered(run_chain, jobs):
            series[key] = x
            print("done", key, flush=True)
    out = {"generator": "tests/golden/make_ref_schedule_plaquette.py", "schedule": "reference (frozen links, "
           "random shift per sweep, lexicographic sweep, mt19937_64, cold start)", "cases": []}
    for (L, nc, th, n) in sizes:
        for b in BETAS:
            chains = [series[(L, b, k)] for k in range(nc)]
            s = chains_summary(chains)
            m = -(-s["n_bins"] // MAX_BINS)
            if m > 1:
                s = chains_summary(chains, factor=10.0, length=s["bin_length"] * m)
            out["cases"].append({
                "L": L, "beta": b, "n_chains": nc, "n_therm": th, "n_sweeps": n,
                "seeds": [seed_of(L, b, k) for k in range(nc)],
                "updates_per_sweep": 4 * L * (L - 1) ** 3,
                "tau_int": [round(t, 3) for t in s["tau_int"]],
                "bin_length": s["bin_length"],
                "bins": [[round(float(v), 10) for v in c] for c in s["bins"]],
                "mean": s["mean"], "err": s["err"], "err_between_chains": between_chain_err(s["bins"]),
            })
            print(f"L={L} beta={b}: {s['mean']:.6f} +- {s['err']:.6f}, tau_int max "
                  f"{max(s['tau_int']):.2f}, bin {s['bin_length']}, {s['n_bins']} bins")
    out["cases"] = sorted(out["cases"] + kept, key=lambda c: (c["L"], c["beta"]))
    text = json.dumps(out, separators=(",", ":")).replace('{"L"', '\n{"L"')
    OUT.write_text(text + "\n")


if __name__ == "__main__":
    main()
