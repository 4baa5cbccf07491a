"""One lattice split along t into slabs with halo exchanges (qcb/slabs.py): the slabs must
reproduce the whole-lattice heatbath and flow bit for bit, and their observables must sum to
the whole lattice's.  The two-process test runs one slab per process on the same GPU with the
faces exchanged through gloo on the host (the processes' kernels never wait on each other)."""
import ctypes as C
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

import oracle as orc
import qcb
from qcb import _lib
from qcb import slabs as qs

pytestmark = pytest.mark.gpu

CASES = [((4, 4, 6, 8), 2, "fp64", 18), ((4, 6, 4, 8), 4, "fp64", 12), ((6, 4, 4, 8), 2, "fp32", 12),
         ((4, 4, 4, 12), 3, "fp32", 18)]


@pytest.mark.parametrize("dims,n,prec,nr", CASES)
def test_slab_heatbath_and_flow_bit_identical(ctx, dims, n, prec, nr):
    u = orc.hot_philox(dims, 91)
    whole = qcb.GaugeField(ctx, dims, prec, nr)
    whole.set_links(u)
    sl = qs.SlabLattice(ctx, dims, n, prec, nr)
    sl.set_links(u)
    assert np.array_equal(sl.get_links(), whole.get_links())
    _lib.check(_lib.lib().qcb_heatbath(whole.h, 6.0, 2, 1, 17, 3))
    sl.heatbath(6.0, 2, 1, 17, 3)
    assert np.array_equal(sl.get_links(), whole.get_links())
    _lib.check(_lib.lib().qcb_flow_steps(whole.h, 0.02, 3))
    sl.flow_steps(0.02, 3)
    assert np.array_equal(sl.get_links(), whole.get_links())
    tol = 1e-12 if prec == "fp64" else 1e-6
    assert abs(sl.plaquette() - qcb.observables.mean_plaquette_global(whole)) < tol
    q, e = sl.topo_qe()
    qw, ew = qcb.observables.topo_q_e_clover_global(whole)
    assert abs(q - qw) < tol * max(1.0, abs(qw)) and abs(e - ew) < tol * max(1.0, ew)
    sl.close()
    whole.close()


def test_slab_hot_start_matches_whole_lattice(ctx):
    dims = (4, 4, 4, 8)
    whole = qcb.GaugeField(ctx, dims)
    whole.hot_start(5)
    sl = qs.SlabLattice(ctx, dims, 2)
    sl.hot_start(5)
    assert np.array_equal(sl.get_links(), whole.get_links())
    # the halos hold the neighbours' links
    for s in sl.slabs:
        assert np.array_equal(s.get_links(), s.local_from_global(whole.get_links()))


def test_packed_faces_match_single_face_copies(ctx):
    """qcb_slab_faces_copy_async packs the faces of every (mu, parity) of one side back to back,
    in the order of qcb_slab_face_copy, and unpacks them the same way: a packed buffer equals the
    per-face copies concatenated, and unpacking it into a halo gives that halo the same links."""
    import torch

    dims = (4, 6, 4, 8)
    u = orc.hot_philox(dims, 13)
    for prec, nr in (("fp64", 18), ("fp32", 12)):
        sl = qs.SlabLattice(ctx, dims, 2, prec, nr)
        sl.set_links(u)
        s = sl.slabs[0]
        ns, nb = s.face_shape()
        face = ns * nb
        for mu, par, nf in ((-1, -1, 8), (2, -1, 2), (1, 0, 1)):
            packed = torch.zeros(nf * face, dtype=torch.uint8, device="cuda")
            _lib.check(_lib.lib().qcb_slab_faces_copy_async(s.h, qs.LINKS, 1, mu, par, C.c_void_p(packed.data_ptr()), 0))
            ctx.sync()
            ref = np.zeros(nf * face, np.uint8)
            k = 0
            for m in (range(4) if mu < 0 else [mu]):
                for p_ in (range(2) if par < 0 else [par]):
                    s.face_copy(qs.LINKS, 1, m, p_, ref[k * face:].ctypes.data, False)
                    k += 1
            assert np.array_equal(packed.cpu().numpy(), ref), (prec, mu, par)
        # an exchange by hand: the lower slab's last own slice, packed, unpacked into the upper
        # slab's low halo (first cleared), gives that halo the lower slab's last own slice
        lo, up = sl.slabs[0], sl.slabs[1]
        zeros = torch.zeros(8 * face, dtype=torch.uint8, device="cuda")
        _lib.check(_lib.lib().qcb_slab_faces_copy_async(up.h, qs.LINKS, 0, -1, -1, C.c_void_p(zeros.data_ptr()), 1))
        ctx.sync()
        assert not np.array_equal(up.get_links()[0], lo.get_links()[lo.t_local])
        packed = torch.zeros(8 * face, dtype=torch.uint8, device="cuda")
        _lib.check(_lib.lib().qcb_slab_faces_copy_async(lo.h, qs.LINKS, 2, -1, -1, C.c_void_p(packed.data_ptr()), 0))
        _lib.check(_lib.lib().qcb_slab_faces_copy_async(up.h, qs.LINKS, 0, -1, -1, C.c_void_p(packed.data_ptr()), 1))
        ctx.sync()
        assert np.array_equal(up.get_links()[0], lo.get_links()[lo.t_local])
        sl.close()


def test_slab_rejects_whole_lattice_calls(ctx):
    s = qs.Slab(ctx, (4, 4, 4, 8), 0, 4)
    lib = _lib.lib()
    assert lib.qcb_heatbath(s.h, 6.0, 1, 1, 1, 0) == 7
    assert lib.qcb_flow_steps(s.h, 0.02, 1) == 7
    b = C.c_void_p()
    arr = (C.c_void_p * 1)(s.h.value)
    assert lib.qcb_batch_create(ctx.h, 1, arr, C.byref(b)) == 1
    h = C.c_void_p()
    assert lib.qcb_lattice_create_slab(ctx.h, (C.c_int * 4)(4, 4, 4, 8), 1, 4, 0, 18, C.byref(h)) == 1  # odd t0
    assert lib.qcb_lattice_create_slab(ctx.h, (C.c_int * 4)(4, 4, 4, 8), 6, 4, 0, 18, C.byref(h)) == 1  # past Lt
    s.close()


def _free_port():
    with socket.socket() as k:
        k.bind(("127.0.0.1", 0))
        return k.getsockname()[1]


def _rank_main(rank, world, port, dims, u, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": "0",
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    from qcb import replicas

    dist = replicas.init("gloo", timeout_s=120)
    try:
        ctx = qcb.Context(0)
        ds = qs.DistSlab(ctx, dims, dist, "fp64", 18, transport="host")
        ds.slab.set_links(ds.slab.local_from_global(u))
        ds.heatbath(6.0, 1, 1, 23, 0)
        ds.flow_steps(0.02, 2)
        p = ds.plaquette()
        q.put((rank, ds.slab.own(ds.slab.get_links()), p))
        ds.slab.close()
        ctx.close()
    finally:
        dist.destroy_process_group()


def test_two_process_slabs_match_whole_lattice(ctx):
    dims = (4, 4, 4, 8)
    u = orc.hot_philox(dims, 5)
    whole = qcb.GaugeField(ctx, dims)
    whole.set_links(u)
    _lib.check(_lib.lib().qcb_heatbath(whole.h, 6.0, 1, 1, 23, 0))
    _lib.check(_lib.lib().qcb_flow_steps(whole.h, 0.02, 2))
    want, pw = whole.get_links(), qcb.observables.mean_plaquette_global(whole)
    world, port = 2, _free_port()
    mpc = mp.get_context("spawn")
    q = mpc.Queue()
    procs = [mpc.Process(target=_rank_main, args=(r, world, port, dims, u, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=300) for _ in range(world)), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = np.concatenate([o[1] for o in out], axis=0)
    assert np.array_equal(got, want)
    assert all(abs(o[2] - pw) < 1e-12 for o in out)
