"""Size-independent properties checked at the benchmark's lattice size, 32^4, where the oracle
would take too long: the plaquette, Q and E are invariant under a random gauge transformation
and under a translation of the field, and E(t) decreases along the Wilson flow.  FP64 18-real
to FP64 rounding; FP32 12-real with the FP32 bounds written in each test."""
import numpy as np
import pytest

import qcb

pytestmark = pytest.mark.gpu

DIMS = (32, 32, 32, 32)


def thermalised(ctx, prec, nr, sweeps=20):
    f = qcb.GaugeField(ctx, DIMS, prec, nr)
    f.hot_start(31)
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(f.h, 6.0, sweeps, 1, 31, 0))
    return f


def observables(f):
    p = qcb.observables.mean_plaquette_global(f)
    q, e = qcb.observables.topo_q_e_clover_global(f)
    return p, q, e


@pytest.mark.parametrize("prec,nr,tp,tq,te", [("fp64", 18, 1e-13, 1e-9, 1e-12), ("fp32", 12, 1e-6, 1e-3, 1e-5)])
def test_observables_gauge_invariant_at_32x4(ctx, prec, nr, tp, tq, te):
    """A random gauge transformation (computed in FP64, stored in the lattice's precision)
    leaves P, Q and E unchanged up to the storage's rounding."""
    f = thermalised(ctx, prec, nr)
    p0, q0, e0 = observables(f)
    f.gauge_transform(77)
    p1, q1, e1 = observables(f)
    assert 0.5 < p0 < 0.7
    assert abs(p1 - p0) < tp
    assert abs(q1 - q0) < tq
    assert abs(e1 - e0) < te * e0
    f.close()


@pytest.mark.parametrize("prec,nr", [("fp64", 18), ("fp32", 12)])
def test_observables_translation_invariant_at_32x4(ctx, prec, nr):
    """A translation moves links without arithmetic: every site's plaquette and clover values
    are the same numbers summed in another order (FP64 block sums), so P, Q and E agree to
    FP64 rounding in both storages."""
    f = thermalised(ctx, prec, nr)
    p0, q0, e0 = observables(f)
    f.translate((3, 1, 7, 5))
    p1, q1, e1 = observables(f)
    assert abs(p1 - p0) < 1e-12
    assert abs(q1 - q0) < 1e-9
    assert abs(e1 - e0) < 1e-12 * e0
    f.close()


def test_flow_energy_decreases_at_32x4_fp32(ctx):
    """E(t) along the FP32-12 flow (records every 10 RK3 steps to t = 2) decreases strictly,
    and the flow leaves the lattice's own links untouched."""
    f = thermalised(ctx, "fp32", 12)
    before = f.get_links()
    rec = qcb.observables.topo_charge_flowed(f, qcb.GradientFlow(0.02), 10, 10).reshape(-1, 3)
    assert np.all(np.isfinite(rec))
    assert np.allclose(rec[:, 0], 0.2 * np.arange(10))
    assert np.all(np.diff(rec[:, 2]) < 0)
    assert np.array_equal(f.get_links(), before)
    f.close()


def test_heatbath_and_flow_deterministic_at_32x4_fp32(ctx):
    """The same seed gives the same links, bit for bit, whatever the block size of the passes
    (the Philox draws are keyed by link, sweep, hit and subgroup, not by thread)."""
    lib = qcb._lib.lib()
    outs = []
    for block in (128, 64, 128):
        ctx.set_block(block)
        f = qcb.GaugeField(ctx, DIMS, "fp32", 12)
        f.hot_start(5)
        qcb._lib.check(lib.qcb_heatbath(f.h, 6.0, 5, 1, 5, 0))
        qcb._lib.check(lib.qcb_flow_steps(f.h, 0.02, 4))
        outs.append(f.get_links())
        f.close()
    ctx.set_block(0)
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])
