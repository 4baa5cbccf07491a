"""The request server: continuous batching, admission by HBM budget, cancellation.

A job's result must be the same alone and in the mix (bit-identical: counter-based random
numbers and per-lattice arithmetic), and equal to the direct library calls.
"""
import numpy as np
import pytest

import qcb

pytestmark = pytest.mark.gpu

SIZES = [(4, 4, 4, 4), (6, 6, 6, 6), (8, 8, 8, 8), (4, 6, 4, 8), (8, 8, 8, 8), (6, 6, 6, 6)]


def prepared(ctx, k, dims):
    f = qcb.GaugeField(ctx, dims, "fp32", 12)
    f.hot_start(500 + k)
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(f.h, 6.0, 5, 1, 500 + k, 0))
    return f


def jobs_spec():
    # alternating sweeps / flow jobs of different lengths
    return [("sweeps", 6.0, 7), ("flow", 0.02, 9), ("sweeps", 5.8, 3), ("flow", 0.02, 4),
            ("flow", 0.02, 13), ("sweeps", 6.2, 10)]


def run_jobs(srv, fields, which):
    ids = {}
    for k in which:
        kind, a, n = jobs_spec()[k]
        if kind == "sweeps":
            ids[srv.submit_sweeps(fields[k], a, n, seed=900 + k, sweep_offset=5)] = k
        else:
            ids[srv.submit_flow(fields[k], a, n)] = k
    srv.drain(300)
    out = {}
    for r in srv.poll(1000):
        assert r.status == 0
        out[ids[r.id]] = (r.plaquette, r.t, r.q, r.e)
    return out


def test_same_result_alone_and_in_mix(ctx):
    srv = qcb.Server(ctx, "fp32", 12, hbm_budget=1 << 30, quantum_sweeps=2, quantum_steps=3)
    alone_f = [prepared(ctx, k, d) for k, d in enumerate(SIZES)]
    mix_f = [prepared(ctx, k, d) for k, d in enumerate(SIZES)]
    alone = {}
    for k in range(len(SIZES)):
        alone.update(run_jobs(srv, alone_f, [k]))
    mixed = run_jobs(srv, mix_f, list(range(len(SIZES))))
    for k in range(len(SIZES)):
        assert alone[k] == mixed[k], (k, alone[k], mixed[k])
        assert np.array_equal(alone_f[k].get_links(), mix_f[k].get_links())
    # and equal to the direct library calls
    ref = [prepared(ctx, k, d) for k, d in enumerate(SIZES)]
    lib = qcb._lib.lib()
    for k, (kind, a, n) in enumerate(jobs_spec()):
        if kind == "sweeps":
            qcb._lib.check(lib.qcb_heatbath(ref[k].h, a, n, 1, 900 + k, 5))
            assert np.array_equal(ref[k].get_links(), mix_f[k].get_links())
            assert mixed[k][0] == pytest.approx(qcb.observables.mean_plaquette_global(ref[k]), abs=1e-12)
        else:
            tqe = qcb.observables.topo_charge_flowed(ref[k], qcb.GradientFlow(a), 2, n).reshape(-1, 3)
            assert mixed[k][1] == pytest.approx(tqe[1, 0], abs=1e-12)
            assert mixed[k][2] == pytest.approx(tqe[1, 1], abs=1e-9)
            assert mixed[k][3] == pytest.approx(tqe[1, 2], rel=1e-9)
    st = srv.stats()
    assert st["completed"] == st["submitted"] == 2 * len(SIZES) and st["max_active"] >= 2
    srv.close()


def test_admission_in_arrival_order_under_small_budget(ctx):
    # budget for exactly one 8^4 flow job's work space: flow jobs run one at a time, FIFO
    f = [prepared(ctx, k, (8, 8, 8, 8)) for k in range(3)]
    one = 2 * 48 * 8 * 2048 + 32 * 8 * 2048 + 1024
    srv = qcb.Server(ctx, "fp32", 12, hbm_budget=one + 512, quantum_steps=2)
    ids = [srv.submit_flow(x, 0.02, 6) for x in f]
    srv.drain(300)
    res = {r.id: r for r in srv.poll()}
    admits = [res[i].admit_s for i in ids]
    finishes = [res[i].finish_s for i in ids]
    assert admits == sorted(admits) and finishes == sorted(finishes)
    assert admits[1] >= finishes[0] - 1e-6 and admits[2] >= finishes[1] - 1e-6
    assert srv.stats()["max_active"] == 1
    # a job larger than the whole budget is refused at submission
    big = qcb.GaugeField(ctx, (16, 16, 16, 16), "fp32", 12)
    with pytest.raises(qcb.QcbError) as e:
        srv.submit_flow(big, 0.02, 1)
    assert e.value.code == 5
    srv.close()


def test_cancel(ctx):
    srv = qcb.Server(ctx, "fp32", 12, hbm_budget=1 << 28, quantum_sweeps=1)
    f = prepared(ctx, 0, (8, 8, 8, 8))
    jid = srv.submit_sweeps(f, 6.0, 100000, seed=1)
    srv.cancel(jid)
    srv.drain(120)
    (r,) = srv.poll()
    assert r.id == jid and r.status == 8
    srv.close()
