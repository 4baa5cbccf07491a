"""Measurements fused into the update kernels, against the separate kernels and the oracle.

qcb_heatbath_plaquette sums the plaquette inside the last sweep's mu = 3 passes (the
reference measures with mean_plaquette_global after the sweeps, observables_mpi.cpp:8-43):
the links must be bit-identical to qcb_heatbath's and the plaquette equal to qcb_plaquette's
to rounding (1e-12 relative in FP64, 1e-7 absolute in FP32, where every site's sum is formed in
FP32), and to the oracle's plaquette of the oracle's links to 1e-12 in FP64.
"""
import numpy as np
import pytest

import oracle as orc
import qcb
from qcb import _lib

pytestmark = pytest.mark.gpu


def fused(f, beta, n, hits, seed, off):
    import ctypes as C

    out = C.c_double()
    _lib.check(_lib.lib().qcb_heatbath_plaquette(f.h, beta, n, hits, seed, off, C.byref(out)))
    return out.value


@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (4, 6, 4, 8), (2, 2, 4, 6), (6, 4, 4, 4)])
@pytest.mark.parametrize("prec,nr", [("fp64", 18), ("fp64", 12), ("fp32", 18), ("fp32", 12)])
def test_heatbath_plaquette_matches_separate_kernels(ctx, dims, prec, nr):
    a = qcb.GaugeField(ctx, dims, prec, nr)
    b = qcb.GaugeField(ctx, dims, prec, nr)
    a.hot_start(5)
    b.hot_start(5)
    lib = _lib.lib()
    for n, off in ((1, 0), (3, 1), (2, 4)):
        _lib.check(lib.qcb_heatbath(a.h, 6.0, n, 1, 21, off))
        pa = qcb.observables.mean_plaquette_global(a)
        pb = fused(b, 6.0, n, 1, 21, off)
        assert np.array_equal(a.get_links(), b.get_links())
        tol = 1e-12 * abs(pa) if prec == "fp64" else 1e-7
        assert abs(pa - pb) <= tol, (n, pa, pb)
    # n_sweeps = 0 only measures
    assert abs(fused(b, 6.0, 0, 1, 21, 0) - qcb.observables.mean_plaquette_global(a)) <= 1e-12
    a.close()
    b.close()


def test_heatbath_plaquette_matches_oracle_fp64(ctx):
    dims = (4, 6, 4, 8)
    u = orc.hot_philox(dims, 8)
    f = qcb.GaugeField(ctx, dims)
    f.set_links(u)
    p = fused(f, 5.9, 2, 2, 13, 3)
    ref, fails = orc.heatbath_cb(u, dims, 5.9, 2, 2, 13, 3)
    assert fails == 0
    assert np.abs(f.get_links() - ref).max() < 1e-11
    assert abs(p - orc.plaquette(ref, dims)) < 1e-12
    f.close()


def test_heatbath_plaquette_rejects_slabs_and_bad_arguments(ctx):
    import ctypes as C

    lib = _lib.lib()
    f = qcb.GaugeField(ctx, (4, 4, 4, 4))
    out = C.c_double()
    assert lib.qcb_heatbath_plaquette(f.h, 6.0, 1, 1, 1, 0, None) == 1
    assert lib.qcb_heatbath_plaquette(f.h, -1.0, 1, 1, 1, 0, C.byref(out)) == 1
    assert lib.qcb_heatbath_plaquette(f.h, 6.0, -1, 1, 1, 0, C.byref(out)) == 1
    f.close()
    s = C.c_void_p()
    _lib.check(lib.qcb_lattice_create_slab(ctx.h, (C.c_int * 4)(4, 4, 4, 8), 0, 4, 0, 18, C.byref(s)))
    assert lib.qcb_heatbath_plaquette(s, 6.0, 1, 1, 1, 0, C.byref(out)) == 7
    lib.qcb_lattice_destroy(s)


@pytest.mark.parametrize("dims", [(8, 8, 8, 8), (4, 6, 4, 8), (2, 2, 4, 6)])
@pytest.mark.parametrize("nr", [12, 18])
def test_flow_measure_fused_qe_matches_clover_kernel_fp32(ctx, dims, nr):
    """FP32 topo_charge_flowed sums each record's clover inside stage 1 of the next RK3 step
    (observables_mpi.cpp:153-178 measures before each group of N_rk_steps): every site's
    (q, e) is the clover kernel's, so the records agree with a replay through qcb_topo_qe and
    qcb_flow_steps to the rounding of the FP64 sums (1e-10)."""
    f = qcb.GaugeField(ctx, dims, "fp32", nr)
    f.hot_start(17)
    _lib.check(_lib.lib().qcb_heatbath(f.h, 6.0, 5, 1, 17, 0))
    n_gf, n_rk = 6, 2
    got = qcb.observables.topo_charge_flowed(f, qcb.GradientFlow(0.02), n_gf, n_rk).reshape(-1, 3)
    g = qcb.GaugeField(ctx, dims, "fp32", nr)
    g.copy_from(f)
    for s in range(n_gf):
        q, e = qcb.observables.topo_q_e_clover_global(g)
        assert got[s, 0] == pytest.approx(s * n_rk * 0.02, abs=1e-12)
        assert abs(got[s, 1] - q) <= 1e-10 * max(1.0, abs(q)), (s, got[s, 1], q)
        assert abs(got[s, 2] - e) <= 1e-10 * e, (s, got[s, 2], e)
        _lib.check(_lib.lib().qcb_flow_steps(g.h, 0.02, n_rk))
    f.close()
    g.close()
