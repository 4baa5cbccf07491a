"""Parity with the FP64 oracle on lattice shapes away from powers of two: Lx/2 odd or 1, extents
6 and 10 (the coordinate division runs on multiply-high reciprocals, exact for these divisors),
Lt not a multiple of 4, and 8^4.  FP64 18-real to the bounds of test_gpu_parity; FP32 with the
tolerances written in each test (FP32 rounding, with the same Philox stream as the oracle)."""
import numpy as np
import pytest

import oracle as orc
import qcb

pytestmark = pytest.mark.gpu

SHAPES = [(10, 6, 6, 4), (6, 10, 4, 6), (2, 6, 10, 4), (8, 8, 8, 8)]


def lattice(ctx, u, dims, prec="fp64", nr=18):
    f = qcb.GaugeField(ctx, dims, prec, nr)
    f.set_links(u)
    return f


def heated(dims, seed, sweeps=2, beta=6.0):
    u, fails = orc.heatbath_cb(orc.hot_philox(dims, seed), dims, beta, sweeps, 1, seed + 1)
    assert fails == 0
    return u


@pytest.mark.parametrize("dims", SHAPES)
def test_heatbath_fp64_matches_oracle_on_shapes(ctx, dims):
    u = orc.hot_philox(dims, 51)
    f = lattice(ctx, u, dims)
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(f.h, 5.8, 2, 1, 99, 0))
    ref, fails = orc.heatbath_cb(u, dims, 5.8, 2, 1, 99, 0)
    assert fails == 0
    assert np.abs(f.get_links() - ref).max() < 1e-11


@pytest.mark.parametrize("dims", SHAPES)
def test_plaquette_qe_and_flow_fp64_match_oracle_on_shapes(ctx, dims):
    u = heated(dims, 52)
    f = lattice(ctx, u, dims)
    assert abs(qcb.observables.mean_plaquette_global(f) - orc.plaquette(u, dims)) < 1e-12
    q, e = qcb.observables.topo_q_e_clover_global(f)
    rq, re_ = orc.topo_qe(u, dims)
    assert abs(q - rq) < 1e-12 * max(1.0, abs(rq))
    assert abs(e - re_) < 1e-12 * max(1.0, abs(re_))
    qcb._lib.check(qcb._lib.lib().qcb_flow_steps(f.h, 0.02, 2))
    assert np.abs(f.get_links() - orc.flow_steps(u, dims, 0.02, 2)).max() < 1e-12


@pytest.mark.parametrize("dims", SHAPES)
@pytest.mark.parametrize("nr", [12, 18])
def test_fp32_flow_tracks_oracle_on_shapes(ctx, dims, nr):
    """Three RK3 steps in FP32 (the per-site kernel, FP64 Horner coefficients and stage-3
    re-orthonormalisation) against the FP64 oracle from the same FP64 input: every link
    element within 2e-5, the mean deviation within 2e-6."""
    u = heated(dims, 53)
    f = lattice(ctx, u, dims, "fp32", nr)
    qcb._lib.check(qcb._lib.lib().qcb_flow_steps(f.h, 0.02, 3))
    d = np.abs(f.get_links() - orc.flow_steps(u, dims, 0.02, 3))
    assert d.max() < 2e-5, d.max()
    assert d.mean() < 2e-6, d.mean()


@pytest.mark.parametrize("dims", SHAPES)
def test_fp32_flow_records_track_oracle_on_shapes(ctx, dims):
    """Flow records of FP32-12 (clover summed inside stage 1 of each record's step) against the
    oracle's FP64 records: |dQ| < 1e-4 and |dE| / E < 1e-5."""
    u = heated(dims, 54)
    f = lattice(ctx, u, dims, "fp32", 12)
    got = qcb.observables.topo_charge_flowed(f, qcb.GradientFlow(0.02), 5, 3).reshape(-1, 3)
    ref = orc.flow_measure(u, dims, 0.02, 5, 3).reshape(-1, 3)
    assert np.allclose(got[:, 0], ref[:, 0])
    assert np.abs(got[:, 1] - ref[:, 1]).max() < 1e-4
    assert (np.abs(got[:, 2] - ref[:, 2]) / ref[:, 2]).max() < 1e-5


@pytest.mark.parametrize("dims", SHAPES)
def test_fp32_heatbath_tracks_oracle_on_shapes(ctx, dims):
    """One FP32-12 sweep on the oracle's Philox stream: all but rare accept/reject flips agree
    with the FP64 oracle to FP32 rounding."""
    u = orc.hot_philox(dims, 55)
    f = lattice(ctx, u, dims, "fp32", 12)
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(f.h, 6.0, 1, 1, 17, 0))
    ref, _ = orc.heatbath_cb(u, dims, 6.0, 1, 1, 17, 0)
    d = np.abs(f.get_links() - ref).reshape(-1, 9).max(axis=1)
    assert np.mean(d < 1e-4) > 0.99
