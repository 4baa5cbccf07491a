"""Batches of lattices (one persistent launch per phase) against single-lattice runs.

Every batched result must be bit-identical to running the lattice alone with the same
seed and sweep counter, whatever the mix of sizes and the tiles the autotuner picks.
"""
import numpy as np
import pytest

import oracle as orc
import qcb

pytestmark = pytest.mark.gpu

DIMS = [(4, 4, 4, 4), (4, 6, 4, 8), (8, 8, 8, 8), (6, 6, 6, 6), (4, 4, 4, 4)]
BETAS = [5.7, 5.85, 6.0, 6.2, 6.0]
SEEDS = [11, 22, 33, 44, 55]
OFFS = [0, 5, 100, 7, 0]


def make_fields(ctx, prec, nr, starts):
    fields = []
    for k, d in enumerate(DIMS):
        f = qcb.GaugeField(ctx, d, prec, nr)
        if starts[k] == "hot":
            f.hot_start(1000 + k)
        fields.append(f)
    return fields


@pytest.mark.parametrize("prec,nr", [("fp64", 18), ("fp32", 12)])
def test_batched_heatbath_and_flow_bit_identical(ctx, prec, nr):
    starts = ["hot", "cold", "hot", "cold", "hot"]
    single = make_fields(ctx, prec, nr, starts)
    batched = make_fields(ctx, prec, nr, starts)
    lib = qcb._lib.lib()
    for f, b, s, o in zip(single, BETAS, SEEDS, OFFS):
        qcb._lib.check(lib.qcb_heatbath(f.h, b, 3, 2, s, o))
        qcb._lib.check(lib.qcb_flow_steps(f.h, 0.02, 3))
    batch = qcb.Batch(ctx, batched)
    batch.heatbath(BETAS, 3, 2, SEEDS, OFFS)
    batch.flow_steps(0.02, 3)
    ctx.sync()
    for f, g in zip(single, batched):
        assert np.array_equal(f.get_links(), g.get_links())
    p = batch.plaquette()
    q, e = batch.topo_qe()
    for k, f in enumerate(single):
        assert abs(p[k] - qcb.observables.mean_plaquette_global(f)) < 1e-13
        qs, es = qcb.observables.topo_q_e_clover_global(f)
        assert abs(q[k] - qs) < 1e-12 * max(1, abs(qs)) and abs(e[k] - es) < 1e-12 * max(1, es)
    batch.close()


def test_batched_heatbath_matches_oracle_fp64(ctx):
    fields = [qcb.GaugeField(ctx, d) for d in DIMS[:3]]
    us = [orc.hot_philox(d, 7 + k) for k, d in enumerate(DIMS[:3])]
    for f, u in zip(fields, us):
        f.set_links(u)
    batch = qcb.Batch(ctx, fields)
    batch.heatbath(BETAS[:3], 2, 1, SEEDS[:3], OFFS[:3])
    ctx.sync()
    for k, (f, u) in enumerate(zip(fields, us)):
        ref, fails = orc.heatbath_cb(u, DIMS[k], BETAS[k], 2, 1, SEEDS[k], OFFS[k])
        assert fails == 0
        assert np.abs(f.get_links() - ref).max() < 1e-11


def test_tiles_and_autotune_do_not_change_results(ctx, tmp_path):
    starts = ["hot"] * 5
    a = make_fields(ctx, "fp32", 12, starts)
    b = make_fields(ctx, "fp32", 12, starts)
    ba, bb = qcb.Batch(ctx, a), qcb.Batch(ctx, b)
    ba.set_tiles(hb=[32, 64, 96, 128, 4096], flow=[64, 32, 256, 512, 128])
    cache = tmp_path / "tune.json"
    bb.autotune(cache)
    assert cache.exists() and "hb|8x8x8x8" in cache.read_text()
    hb_tiles, fl_tiles = bb.tiles()
    assert all(t % 32 == 0 for t in hb_tiles + fl_tiles)
    for bt in (ba, bb):
        bt.heatbath(BETAS, 2, 1, SEEDS, OFFS)
        bt.flow_steps(0.02, 2)
    ctx.sync()
    for f, g in zip(a, b):
        assert np.array_equal(f.get_links(), g.get_links())
    # a second autotune reads the cache
    bb.autotune(cache)
    assert bb.tiles() == (hb_tiles, fl_tiles)


def test_graph_captured_workload(ctx):
    starts = ["hot", "cold", "hot", "cold", "hot"]
    fields = make_fields(ctx, "fp32", 12, starts)
    ref = make_fields(ctx, "fp32", 12, starts)
    batch = qcb.Batch(ctx, fields)
    plaq, rec, used = batch.run(BETAS, SEEDS, OFFS, n_sweeps=4, n_hits=1, eps=0.02, n_groups=3, rk_per_group=2)
    assert used, "the plan should run as a CUDA graph"
    lib = qcb._lib.lib()
    for k, f in enumerate(ref):
        qcb._lib.check(lib.qcb_heatbath(f.h, BETAS[k], 4, 1, SEEDS[k], OFFS[k]))
        assert plaq[k] == pytest.approx(qcb.observables.mean_plaquette_global(f), abs=1e-12)
        tqe = qcb.observables.topo_charge_flowed(f, qcb.GradientFlow(0.02), 4, 2).reshape(-1, 3)
        assert np.allclose(rec[k], tqe, rtol=0, atol=1e-10)
        # the batch's links advanced exactly like the single run
        assert np.array_equal(fields[k].get_links(), f.get_links())
    # replay: the next sweeps continue the chain (sweep offsets advanced by the caller)
    offs2 = [o + 4 for o in OFFS]
    plaq2, rec2, used2 = batch.run(BETAS, SEEDS, offs2, n_sweeps=4, n_hits=1, eps=0.02, n_groups=3, rk_per_group=2)
    assert used2
    for k, f in enumerate(ref):
        qcb._lib.check(lib.qcb_heatbath(f.h, BETAS[k], 4, 1, SEEDS[k], offs2[k]))
        assert plaq2[k] == pytest.approx(qcb.observables.mean_plaquette_global(f), abs=1e-12)


def test_batch_rejects_mixed_storage(ctx):
    a = qcb.GaugeField(ctx, (4, 4, 4, 4), "fp32", 12)
    b = qcb.GaugeField(ctx, (4, 4, 4, 4), "fp64", 18)
    with pytest.raises(qcb.QcbError) as e:
        qcb.Batch(ctx, [a, b])
    assert e.value.code == 1
