"""Argument edges of the C ABI on the device: extents, volume limit, empty work, errors."""
import ctypes as C

import numpy as np
import pytest

import oracle as orc
import qcb
from qcb import _lib

pytestmark = pytest.mark.gpu


def _create(ctx, dims, prec=qcb.FP64, storage=qcb.R18):
    h = C.c_void_p()
    rc = _lib.lib().qcb_lattice_create(ctx.h, (C.c_int * 4)(*dims), prec, storage, C.byref(h))
    return rc, h


@pytest.mark.parametrize("dims", [(8, 8, 8, 7), (0, 8, 8, 8), (8, -2, 8, 8), (1024, 1024, 1024, 2)])
def test_lattice_create_rejects_bad_extents(ctx, dims):
    rc, h = _create(ctx, dims)
    assert rc == 1 and not h.value
    assert b"extents" in _lib.lib().qcb_last_error()


def test_lattice_create_rejects_bad_kind(ctx):
    assert _create(ctx, (4, 4, 4, 4), prec=7)[0] == 1
    assert _create(ctx, (4, 4, 4, 4), storage=16)[0] == 1


def test_zero_work_leaves_links_unchanged(ctx):
    dims = (4, 4, 4, 6)
    u = orc.hot_philox(dims, 3)
    f = qcb.GaugeField(ctx, dims)
    f.set_links(u)
    lib = _lib.lib()
    _lib.check(lib.qcb_heatbath(f.h, 6.0, 0, 1, 1, 0))      # no sweeps
    _lib.check(lib.qcb_heatbath(f.h, 6.0, 1, 0, 1, 0))      # no hits
    _lib.check(lib.qcb_flow_steps(f.h, 0.02, 0))            # no flow steps
    assert qcb.observables.topo_charge_flowed(f, qcb.GradientFlow(0.02), 0, 1).size == 0
    assert np.array_equal(f.get_links(), u)
    # N_rk_steps = 0: every record measures the unflowed configuration at t = 0
    rec = qcb.observables.topo_charge_flowed(f, qcb.GradientFlow(0.02), 3, 0).reshape(-1, 3)
    q, e = qcb.observables.topo_q_e_clover_global(f)
    assert np.all(rec[:, 0] == 0.0) and np.allclose(rec[:, 1], q, atol=1e-12) and np.allclose(rec[:, 2], e)


def test_heatbath_rejects_bad_arguments(ctx):
    f = qcb.GaugeField(ctx, (4, 4, 4, 4))
    lib = _lib.lib()
    assert lib.qcb_heatbath(f.h, 0.0, 1, 1, 1, 0) == 1
    assert lib.qcb_heatbath(f.h, -1.0, 1, 1, 1, 0) == 1
    assert lib.qcb_heatbath(f.h, 6.0, -1, 1, 1, 0) == 1
    assert lib.qcb_heatbath(None, 6.0, 1, 1, 1, 0) == 1
    assert lib.qcb_flow_measure(f.h, 0.02, -1, 1, None) == 1
    assert lib.qcb_flow_measure(f.h, 0.02, 2, 1, None) == 1
    # the lattice is still a cold start
    assert qcb.observables.mean_plaquette_global(f) == 1.0
