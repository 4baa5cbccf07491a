"""The allocation-free plaquette entry point (qcb_plaquette_noalloc) through the C ABI.

It exists for callers that cannot allocate device memory themselves, such as a host whose
pool allocator owns the device memory, or a loop that cannot afford cudaMalloc's implicit
device synchronisation.  The test owns the output buffer (allocated here, not by the entry
point) and compares two calls in a row, on two lattices of different sizes and storages,
with the allocating entry point qcb_plaquette, within the library's FP64 tolerance (1e-12
relative).  This file sorts last so that a run stopping at the first failure has run
every other test before it.
"""
import ctypes as C

import pytest

import qcb
from qcb import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-12


def noalloc_plaquette(field: qcb.GaugeField, out_ptr: int, stream: int) -> None:
    ptr, stride, _nchunk, _cbytes = field.device_links()
    rc = _lib.lib().qcb_plaquette_noalloc(C.c_void_p(ptr), (C.c_int * 4)(*field.dims), field.precision,
                                          field.storage, stride, C.c_void_p(out_ptr), C.c_void_p(stream))
    _lib.check(rc)


def test_plaquette_noalloc_matches_allocating_entry_point():
    import torch

    ctx = qcb.Context(0)
    out = torch.full((4,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    cases = [((8, 8, 8, 8), "fp64", 18, 5), ((4, 6, 4, 8), "fp32", 12, 6), ((16, 16, 16, 16), "fp64", 18, 7)]
    for dims, prec, nr, seed in cases:
        f = qcb.GaugeField(ctx, dims, prec, nr)
        f.hot_start(seed)
        _lib.check(_lib.lib().qcb_heatbath(f.h, 6.0, 2, 1, seed, 0))
        ref = qcb.observables.mean_plaquette_global(f)
        for _call in range(2):  # two calls in a row share the static scratch
            out.fill_(float("nan"))
            torch.cuda.synchronize()
            noalloc_plaquette(f, out.data_ptr(), ctx.stream)
            ctx.sync()
            got = float(out[0].item())
            assert abs(got - ref) <= TOL * abs(ref), (dims, prec, nr, got, ref)
        f.close()
    ctx.close()


def test_plaquette_noalloc_allocates_nothing_and_runs_on_any_stream():
    """After a warm-up call, further calls leave the device's free memory unchanged, and a
    call on a stream other than the context's gives the same value."""
    import torch

    ctx = qcb.Context(0)
    f = qcb.GaugeField(ctx, (8, 8, 8, 8), "fp32", 12)
    f.hot_start(3)
    ref = qcb.observables.mean_plaquette_global(f)
    out = torch.full((2,), float("nan"), dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    noalloc_plaquette(f, out.data_ptr(), ctx.stream)  # warm-up: loads the module's device code
    ctx.sync()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        noalloc_plaquette(f, out.data_ptr(), ctx.stream)
    ctx.sync()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)
    out.fill_(float("nan"))
    torch.cuda.synchronize()
    noalloc_plaquette(f, out.data_ptr() + 8, side.cuda_stream)
    side.synchronize()
    got = float(out[1].item())
    assert abs(got - ref) <= TOL * abs(ref), (got, ref)
    f.close()
    ctx.close()


def test_plaquette_noalloc_rejects_bad_arguments():
    L = _lib.lib()
    dims = (C.c_int * 4)(8, 8, 8, 8)
    # null links / output
    assert L.qcb_plaquette_noalloc(None, dims, 0, 18, 2048, C.c_void_p(16), None) == 1
    # odd extent
    bad = (C.c_int * 4)(8, 7, 8, 8)
    assert L.qcb_plaquette_noalloc(C.c_void_p(16), bad, 0, 18, 2048, C.c_void_p(16), None) == 1
    assert b"even" in L.qcb_last_error()
    # stride below half the volume
    assert L.qcb_plaquette_noalloc(C.c_void_p(16), dims, 0, 18, 100, C.c_void_p(16), None) == 1
    assert b"stride" in L.qcb_last_error()
    # links off the 16-byte chunk boundary (FP64, FP32 12-real) or the 8-byte one (FP32 18-real)
    assert L.qcb_plaquette_noalloc(C.c_void_p(24), dims, 0, 18, 2048, C.c_void_p(16), None) == 1
    assert b"aligned" in L.qcb_last_error()
    assert L.qcb_plaquette_noalloc(C.c_void_p(24), dims, 1, 12, 2048, C.c_void_p(16), None) == 1
    assert L.qcb_plaquette_noalloc(C.c_void_p(20), dims, 1, 18, 2048, C.c_void_p(16), None) == 1
    # output not 8-byte aligned
    assert L.qcb_plaquette_noalloc(C.c_void_p(16), dims, 0, 18, 2048, C.c_void_p(12), None) == 1
    assert b"out must be 8-byte aligned" in L.qcb_last_error()
