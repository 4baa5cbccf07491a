"""Parity of the CUDA library (through the C ABI) with the FP64 oracle.

FP64 18-real storage is checked against the oracle to 1e-12 relative (plaquette, clover
Q/E, flow records, heatbath links); FP32 storage is checked with the tolerances written in
each test.  All inputs are seeded.
"""
import numpy as np
import pytest

import oracle as orc
import qcb

pytestmark = pytest.mark.gpu

STORAGES = [("fp64", 18), ("fp64", 12), ("fp32", 18), ("fp32", 12)]


def lattice(ctx, u, dims, prec="fp64", nr=18):
    f = qcb.GaugeField(ctx, dims, prec, nr)
    f.set_links(u)
    return f


def heated(dims, seed, sweeps=3, beta=6.0):
    u, fails = orc.heatbath_cb(orc.hot_philox(dims, seed), dims, beta, sweeps, 1, seed + 1)
    assert fails == 0
    return u


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


@pytest.mark.parametrize("prec,nr", STORAGES)
def test_set_get_roundtrip(ctx, prec, nr):
    dims = (4, 6, 4, 8)
    u = orc.hot_philox(dims, 1)
    f = lattice(ctx, u, dims, prec, nr)
    back = f.get_links()
    tol = 1e-15 if prec == "fp64" else 2e-7
    assert np.abs(back - u).max() < tol * (1 if nr == 18 else 8)


@pytest.mark.parametrize("prec,nr", STORAGES)
def test_cold_start_exact(ctx, prec, nr):
    f = qcb.GaugeField(ctx, (4, 4, 4, 4), prec, nr)
    assert qcb.observables.mean_plaquette_global(f) == 1.0
    assert qcb.observables.topo_q_e_clover_global(f) == (0.0, 0.0)


def test_hot_start_matches_oracle(ctx):
    dims = (6, 4, 4, 4)
    f = qcb.GaugeField(ctx, dims)
    f.hot_start(7)
    assert np.abs(f.get_links() - orc.hot_philox(dims, 7)).max() < 1e-14


def test_gauge_transform_matches_oracle(ctx):
    dims = (4, 4, 4, 4)
    u = heated(dims, 3)
    f = lattice(ctx, u, dims)
    f.gauge_transform(99)
    assert np.abs(f.get_links() - orc.gauge_transform_philox(u, dims, 99)).max() < 1e-13


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (6, 4, 8, 4)])
def test_plaquette_and_qe_fp64(ctx, dims):
    u = heated(dims, 11)
    f = lattice(ctx, u, dims)
    p = qcb.observables.mean_plaquette_global(f)
    assert rel(p, orc.plaquette(u, dims)) < 1e-12
    q, e = qcb.observables.topo_q_e_clover_global(f)
    qo, eo = orc.topo_qe(u, dims)
    assert abs(q - qo) < 1e-12 * max(1.0, abs(qo))
    assert rel(e, eo) < 1e-12


def test_smallest_extents(ctx):
    """Extents of 2 (Lx/2 = 1: the coordinate division by one) and mixed sizes."""
    dims = (2, 2, 4, 6)
    u = orc.hot_philox(dims, 17)
    f = lattice(ctx, u, dims)
    assert rel(qcb.observables.mean_plaquette_global(f), orc.plaquette(u, dims)) < 1e-12
    q, e = qcb.observables.topo_q_e_clover_global(f)
    qo, eo = orc.topo_qe(u, dims)
    assert abs(q - qo) < 1e-12 * max(1.0, abs(qo)) and rel(e, eo) < 1e-12
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(f.h, 6.0, 2, 1, 8, 0))
    ref, fails = orc.heatbath_cb(u, dims, 6.0, 2, 1, 8, 0)
    assert fails == 0
    assert np.abs(f.get_links() - ref).max() < 1e-11


@pytest.mark.parametrize("prec,nr,tol", [("fp64", 12, 1e-12), ("fp32", 18, 1e-6), ("fp32", 12, 1e-6)])
def test_plaquette_and_qe_other_storage(ctx, prec, nr, tol):
    dims = (8, 8, 8, 8)
    u = heated(dims, 12, sweeps=2)
    f = lattice(ctx, u, dims, prec, nr)
    assert abs(qcb.observables.mean_plaquette_global(f) - orc.plaquette(u, dims)) < tol
    q, e = qcb.observables.topo_q_e_clover_global(f)
    qo, eo = orc.topo_qe(u, dims)
    assert abs(q - qo) < 1e-4 if prec == "fp32" else abs(q - qo) < 1e-11
    assert abs(e - eo) < 10 * tol


def test_flow_measure_fp64(ctx):
    dims = (4, 4, 4, 4)
    u = heated(dims, 21, sweeps=4)
    f = lattice(ctx, u, dims)
    got = qcb.observables.topo_charge_flowed(f, qcb.GradientFlow(0.02), 6, 2).reshape(-1, 3)
    ref = orc.flow_measure(u, dims, 0.02, 6, 2).reshape(-1, 3)
    assert np.array_equal(got[:, 0], ref[:, 0])
    assert np.abs(got[:, 1] - ref[:, 1]).max() < 1e-12
    assert np.abs(got[:, 2] - ref[:, 2]).max() < 1e-12 * ref[:, 2].max()
    # the lattice itself is untouched (the flow runs on a copy)
    assert np.array_equal(f.get_links(), u)


def test_flow_measure_many_records(ctx):
    # more records than one device staging chunk (32)
    dims = (4, 4, 4, 4)
    u = heated(dims, 22, sweeps=2)
    f = lattice(ctx, u, dims)
    got = qcb.observables.topo_charge_flowed(f, qcb.GradientFlow(0.02), 40, 1).reshape(-1, 3)
    ref = orc.flow_measure(u, dims, 0.02, 40, 1).reshape(-1, 3)
    assert np.abs(got - ref).max() < 1e-12 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("n", [1, 2, 3])
def test_flow_steps_in_place(ctx, n):
    dims = (4, 6, 4, 4)
    u = heated(dims, 23)
    f = lattice(ctx, u, dims)
    qcb._lib.check(qcb._lib.lib().qcb_flow_steps(f.h, 0.02, n))
    assert np.abs(f.get_links() - orc.flow_steps(u, dims, 0.02, n)).max() < 1e-13


def test_heatbath_fp64_matches_oracle(ctx):
    dims = (4, 4, 6, 4)
    u = orc.hot_philox(dims, 31)
    f = lattice(ctx, u, dims)
    rng = qcb.PhiloxStream(seed=777)
    hp = qcb.io.default_params()
    hp.beta, hp.N_sweeps, hp.N_hits, hp.N_samples = 5.7, 2, 2, 1
    qcb.heatbathcb.samples(f, hp, rng)      # sweeps 0, 1
    qcb.heatbathcb.sweep(f, 5.7, 2, rng)    # sweep 2
    ctx.sync()
    ref, fails = orc.heatbath_cb(u, dims, 5.7, 3, 2, 777, 0)
    assert fails == 0
    got = f.get_links()
    assert np.abs(got - ref).max() < 1e-11
    assert rng.sweep == 3


def test_heatbath_cold_start_fp64(ctx):
    dims = (4, 4, 4, 4)
    f = qcb.GaugeField(ctx, dims)
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(f.h, 6.0, 2, 1, 1234, 0))
    ref, _ = orc.heatbath_cb(orc.cold(dims), dims, 6.0, 2, 1, 1234, 0)
    assert np.abs(f.get_links() - ref).max() < 1e-12


def test_heatbath_independent_of_block_size(ctx):
    dims = (8, 4, 4, 6)
    u = orc.hot_philox(dims, 5)
    outs = []
    for block in (32, 64, 128):
        ctx.set_block(block)
        f = lattice(ctx, u, dims, "fp32", 12)
        qcb._lib.check(qcb._lib.lib().qcb_heatbath(f.h, 6.0, 2, 1, 42, 0))
        outs.append(f.get_links())
    ctx.set_block(0)
    assert np.array_equal(outs[0], outs[1]) and np.array_equal(outs[0], outs[2])


@pytest.mark.parametrize("prec,nr", [("fp32", 18), ("fp32", 12)])
def test_heatbath_fp32_tracks_fp64(ctx, prec, nr):
    dims = (6, 6, 6, 6)
    u = orc.hot_philox(dims, 41)
    f = lattice(ctx, u, dims, prec, nr)
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(f.h, 6.0, 1, 1, 9, 0))
    ref, _ = orc.heatbath_cb(u, dims, 6.0, 1, 1, 9, 0)
    d = np.abs(f.get_links() - ref).reshape(-1, 9).max(axis=1)
    # same Philox stream: all but (rare) accept/reject flips agree to FP32 rounding
    assert np.mean(d < 1e-4) > 0.995
    assert abs(qcb.observables.mean_plaquette_global(f) - orc.plaquette(ref, dims)) < 1e-3


def test_heatbath_fp64_12_matches_oracle(ctx):
    """12-real FP64 storage: rows 0 and 1 stored, row 2 rebuilt, links re-orthonormalised in
    FP64 after each update; the chain stays on the oracle's to 1e-10."""
    dims = (4, 4, 6, 4)
    u = orc.hot_philox(dims, 33)
    f = lattice(ctx, u, dims, "fp64", 12)
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(f.h, 5.9, 2, 1, 4242, 0))
    ref, fails = orc.heatbath_cb(u, dims, 5.9, 2, 1, 4242, 0)
    assert fails == 0
    assert np.abs(f.get_links() - ref).max() < 1e-10


def test_flow_fp64_12_matches_oracle(ctx):
    dims = (4, 4, 4, 6)
    u = heated(dims, 24)
    f = lattice(ctx, u, dims, "fp64", 12)
    qcb._lib.check(qcb._lib.lib().qcb_flow_steps(f.h, 0.02, 3))
    assert np.abs(f.get_links() - orc.flow_steps(u, dims, 0.02, 3)).max() < 1e-12


def test_fp32_flow_links_stay_unitary(ctx):
    """FP32 links are re-orthonormalised in FP64 once per RK3 step, so 60 steps leave them
    unitary to FP32 rounding."""
    dims = (6, 6, 6, 6)
    base = qcb.GaugeField(ctx, dims)
    base.hot_start(5)
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(base.h, 6.0, 5, 1, 5, 0))
    for nr in (12, 18):
        f = qcb.GaugeField(ctx, dims, "fp32", nr)
        f.copy_from(base)
        qcb._lib.check(qcb._lib.lib().qcb_flow_steps(f.h, 0.02, 60))
        m = f.get_links().reshape(-1, 3, 3)
        dev = np.abs(m @ np.conj(np.transpose(m, (0, 2, 1))) - np.eye(3)).max()
        assert dev < 2e-6, (nr, dev)
        assert np.abs(np.linalg.det(m) - 1).max() < 2e-6
        f.close()


def test_kp_cap_reports_error(ctx):
    # beta -> 0 makes alpha tiny, so KP acceptance (~2 alpha) is far below 1/4096
    f = qcb.GaugeField(ctx, (4, 4, 4, 4))
    f.hot_start(3)
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(f.h, 1e-9, 1, 1, 1, 0))
    with pytest.raises(qcb.QcbError) as e:
        ctx.sync()
    assert e.value.code == 6
    ctx.sync()  # status was cleared


def test_ildg_roundtrip_and_bytes(ctx, tmp_path):
    dims = (4, 4, 4, 6)
    u = heated(dims, 51, sweeps=1)
    f = lattice(ctx, u, dims)
    p_gpu, p_orc = tmp_path / "gpu", tmp_path / "orc"
    f.save_ildg(p_gpu)
    orc.write_ildg(p_orc, u, dims)
    assert p_gpu.read_bytes() == p_orc.read_bytes()
    g = qcb.GaugeField(ctx, dims)
    g.load_ildg(p_orc)
    assert np.array_equal(g.get_links(), u)
    # wrong lattice size and truncated data are reported, not read
    h = qcb.GaugeField(ctx, (4, 4, 4, 4))
    with pytest.raises(qcb.QcbError) as e:
        h.load_ildg(p_gpu)
    assert e.value.code == 4
    (tmp_path / "trunc").write_bytes(p_gpu.read_bytes()[:-1000])
    with pytest.raises(qcb.QcbError) as e:
        g.load_ildg(tmp_path / "trunc")
    assert e.value.code == 4


def test_ildg_run_dir_layout(ctx, tmp_path):
    dims = (4, 4, 4, 4)
    f = qcb.GaugeField(ctx, dims)
    f.hot_start(1)
    path = qcb.save_ildg_clime("run1", str(tmp_path), f)
    assert path.endswith("run1/run1")
    g = qcb.GaugeField(ctx, dims)
    qcb.read_ildg_clime("run1", str(tmp_path), g)
    assert np.array_equal(g.get_links(), f.get_links())


def test_reunitarize_fp32(ctx):
    dims = (4, 4, 4, 4)
    u = orc.hot_philox(dims, 61)
    noisy = u * (1 + 1e-4)
    f = lattice(ctx, noisy, dims, "fp64", 18)
    f.reunitarize()
    m = f.get_links().reshape(-1, 3, 3)
    assert np.abs(np.einsum("nij,nkj->nik", m, m.conj()) - np.eye(3)).max() < 1e-14
    assert np.abs(m - u.reshape(-1, 3, 3)).max() < 1e-12


def test_precision_fp32_flow_vs_fp64(ctx):
    """Same FP64 configuration flowed in FP32-12 and FP64-18: |dQ| < 1e-4, |dP| < 1e-6."""
    dims = (8, 8, 8, 8)
    base = qcb.GaugeField(ctx, dims)
    base.hot_start(7)
    qcb._lib.check(qcb._lib.lib().qcb_heatbath(base.h, 6.0, 20, 1, 7, 0))
    f32 = qcb.GaugeField(ctx, dims, "fp32", 12)
    f32.copy_from(base)
    assert abs(qcb.observables.mean_plaquette_global(f32) - qcb.observables.mean_plaquette_global(base)) < 1e-6
    gf = qcb.GradientFlow(0.02)
    r64 = qcb.observables.topo_charge_flowed(base, gf, 6, 10).reshape(-1, 3)
    r32 = qcb.observables.topo_charge_flowed(f32, gf, 6, 10).reshape(-1, 3)
    assert np.abs(r64[:, 1] - r32[:, 1]).max() < 1e-4
    assert np.abs(r64[:, 2] - r32[:, 2]).max() < 1e-4 * r64[:, 2].max()
    # with the per-step FP64 re-orthonormalisation E tracks FP64 to about 1e-7 relative
    assert (np.abs(r64[:, 2] - r32[:, 2]) / r64[:, 2]).max() < 1e-6


def test_context_destroyed_before_its_lattices():
    """Destroying a context with live lattices defers the free until the last one goes."""
    L = qcb._lib.lib()
    c = qcb.Context(0)
    f = qcb.GaugeField(c, (4, 4, 4, 4))
    g = qcb.GaugeField(c, (4, 4, 4, 4))
    raw_ctx, raw_f = c.h, f.h
    c.h = None  # destroy through the C ABI directly, children still alive
    assert L.qcb_ctx_destroy(raw_ctx) == 0
    assert qcb.observables.mean_plaquette_global(f) == 1.0
    f.h = None
    assert L.qcb_lattice_destroy(raw_f) == 0
    g.close()  # the last child frees the context
