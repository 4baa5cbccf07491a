"""The oracle's restatement of the reference's update schedule, on CPU: the frozen-link
mask of the L_core block faces (src/geometry/GeometryCB.cpp:33-56) after a cumulative
shift, and the shift draws of mpi::shift::random_shift (src/mpi/Shift.cpp:163-172)."""
import numpy as np

import oracle as orc


def test_frozen_mask_count_and_unshifted_faces():
    dims, lcore = (4, 4, 4, 4), 2
    u = orc.hot_philox(dims, 1)
    for shift in ((0, 0, 0, 0), (1, 0, 1, 0)):
        out, fails = orc.heatbath_cb_frozen(u, dims, 6.0, 1, 1, 7, 0, lcore, shift)
        assert fails == 0
        changed = np.any(np.abs(out - u) > 0, axis=(-2, -1))  # (t, z, y, x, mu)
        # per direction: 4 values along mu x 2 of 4 values in each of the 3 other directions
        assert int(changed.sum()) == 4 * 4 * 2 ** 3
        for mu in range(4):
            c = changed[..., mu]
            coords = np.argwhere(c)[:, ::-1]  # (x, y, z, t)
            others = [d for d in range(4) if d != mu]
            assert np.all((coords[:, others] + np.array(shift)[others]) % lcore != 0)


def test_frozen_with_core_equal_to_lattice_is_reference_one_rank():
    # one block of edge L: only the links on the c_d = 0 faces (d != mu) are frozen
    dims = (4, 4, 4, 4)
    u = orc.hot_philox(dims, 2)
    out, _ = orc.heatbath_cb_frozen(u, dims, 6.0, 1, 1, 3, 0, 4, (0, 0, 0, 0))
    changed = np.any(np.abs(out - u) > 0, axis=(-2, -1))
    assert int(changed.sum()) == 4 * 4 * 3 ** 3


def test_shift_sequence_range_and_determinism():
    a = orc.shift_sequence(1234, 4, 50)
    b = orc.shift_sequence(1234, 4, 50)
    assert a.shape == (50, 4) and np.array_equal(a, b)
    assert a.min() >= 0 and a.max() <= 3 and len(np.unique(a)) == 4
    assert not np.array_equal(a, orc.shift_sequence(1235, 4, 50))


def test_fixture_chain_reproduced_by_the_oracle():
    """The first recorded sweeps of one fixture chain come out of the oracle again: the
    fixture's bins of the 4^4, beta = 6.0 case start with the mean of the first bin of
    chain 0 (cold start) after n_therm discarded sweeps."""
    import json
    from pathlib import Path

    gold = json.loads((Path(__file__).resolve().parent / "golden" / "ref_schedule_plaquette.json").read_text())
    case = next(c for c in gold["cases"] if c["L"] == 4 and c["beta"] == 6.0)
    chain = orc.RefChain(4, case["seeds"][0], True)
    chain.run(6.0, case["n_therm"], 1, 1)
    x = chain.run(6.0, case["bin_length"], 1, 1)
    assert abs(x.mean() - case["bins"][0][0]) < 1e-9


def test_fixture_statistics_are_consistent():
    """Pooled mean and error recomputed from the stored bins equal the stored ones; the bins
    are at least 10 tau_int long and the cases cover 4^4 and 8^4 at beta 5.7, 6.0, 6.2."""
    import json
    from pathlib import Path

    from stats import pooled_mean_err

    gold = json.loads((Path(__file__).resolve().parent / "golden" / "ref_schedule_plaquette.json").read_text())
    assert sorted((c["L"], c["beta"]) for c in gold["cases"]) == [(L, b) for L in (4, 8) for b in (5.7, 6.0, 6.2)]
    for c in gold["cases"]:
        m, e, n = pooled_mean_err(c["bins"])
        assert abs(m - c["mean"]) < 1e-9 and abs(e - c["err"]) < 1e-9 * max(1.0, c["err"])
        assert c["bin_length"] >= 10 * max(c["tau_int"]) and n >= 100
        assert len(c["bins"]) == c["n_chains"] == len(c["seeds"])


def _fast_build_chain(_):
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).resolve().parent.parent / "oracle"))
    import oracle

    oracle.select_build("fast")
    c = oracle.RefChain(4, 77, False)
    return c.run(6.0, 3, 1, 1)


def test_timing_build_runs_the_same_chain():
    """The timing build (-O3 -march=native -fcx-limited-range) differs from the checker only in
    rounding: three reference-schedule sweeps give the same plaquettes to 1e-9."""
    import multiprocessing as mp

    orc.build_fast()
    with mp.get_context("spawn").Pool(1) as p:
        fast = p.map(_fast_build_chain, [0])[0]
    ref = orc.RefChain(4, 77, False).run(6.0, 3, 1, 1)
    assert np.abs(fast - ref).max() < 1e-9
