"""One lattice split along t into slabs: the multi-device decomposition of a single lattice.

The reference splits one lattice over n_core_dims^4 MPI ranks with halo exchanges and frozen
block faces (src/mpi/MpiTopology.cpp:7-24, src/mpi/HalosExchange.cpp, src/geometry/
GeometryCB.cpp:33-56).  Here the lattice is cut along t into slabs of t_local time slices,
each with one halo slice on either side (qcb_lattice_create_slab).  Every checkerboard
heatbath pass and every RK3 stage is followed by one face exchange between neighbouring
slabs, so the slabs reproduce the whole-lattice run bit for bit (the random numbers are
keyed by the global link).

SlabLattice keeps all slabs in this process (on one device or several; the exchange is a
device or peer copy).  DistSlab is one slab per process (one process per GPU) and exchanges
faces through torch.distributed: "host" transport stages the faces through CPU tensors
(gloo), "device" through CUDA tensors (NCCL).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import Context, GaugeField, _precision
from ._lib import check, lib

LINKS, WORK = 0, 1  # face buffers: the links, the flow work buffer


class Slab(GaugeField):
    """One slab: global times t0 .. t0 + t_local - 1 of a lattice of extents global_dims, as
    local times 1 .. t_local, with halo slices 0 and t_local + 1."""

    def __init__(self, ctx: Context, global_dims, t0: int, t_local: int, precision="fp64", storage: int = 18):
        gd = tuple(int(d) for d in global_dims)
        self.ctx = ctx
        self.global_dims = gd
        self.t0, self.t_local = int(t0), int(t_local)
        self.dims = (gd[0], gd[1], gd[2], self.t_local + 2)
        self.precision = _precision(precision)
        self.storage = int(storage)
        h = C.c_void_p()
        check(lib().qcb_lattice_create_slab(ctx.h, (C.c_int * 4)(*gd), self.t0, self.t_local, self.precision,
                                            self.storage, C.byref(h)))
        self.h = h
        ctx._adopt(self)

    def local_from_global(self, u: np.ndarray) -> np.ndarray:
        """This slab's local array (halos included) cut from a global (Lt, Lz, Ly, Lx, 4, 3, 3) array."""
        ts = [(self.t0 - 1 + k) % self.global_dims[3] for k in range(self.t_local + 2)]
        return np.ascontiguousarray(u[ts])

    def own(self, local: np.ndarray) -> np.ndarray:
        return local[1:self.t_local + 1]

    def heatbath_pass(self, mu, parity, beta, n_hits, seed, sweep) -> None:
        check(lib().qcb_heatbath_pass(self.h, int(mu), int(parity), float(beta), int(n_hits), C.c_uint64(seed),
                                      C.c_uint64(sweep)))

    def flow_stage(self, stage, eps, step) -> None:
        check(lib().qcb_flow_stage(self.h, int(stage), float(eps), int(step)))

    def flow_finish(self, n_steps) -> None:
        check(lib().qcb_flow_finish(self.h, int(n_steps)))

    def face_shape(self, which=LINKS, side=1, mu=0, parity=0):
        seg = (C.c_void_p * 9)()
        nb, ns = C.c_size_t(), C.c_int()
        check(lib().qcb_slab_face(self.h, which, side, mu, parity, seg, C.byref(nb), C.byref(ns)))
        return ns.value, nb.value

    def face_copy(self, which, side, mu, parity, ptr: int, to_face: bool) -> None:
        check(lib().qcb_slab_face_copy(self.h, which, side, mu, parity, C.c_void_p(ptr), 1 if to_face else 0))

    def partial_plaquette(self) -> float:
        out = C.c_double()
        check(lib().qcb_plaquette(self.h, C.byref(out)))
        return out.value

    def partial_qe(self):
        q, e = C.c_double(), C.c_double()
        check(lib().qcb_topo_qe(self.h, C.byref(q), C.byref(e)))
        return q.value, e.value


def flow_dst(stage: int, step: int) -> int:
    """Buffer written by `stage` of RK3 step `step` (qcb_flow_stage): stages 1 and 3 write the
    work buffer on even steps, stage 2 the links; swapped on odd steps."""
    return WORK if ((stage != 2) != bool(step & 1)) else LINKS


def _split(dims, n_slabs):
    lt = int(dims[3])
    if n_slabs < 1 or lt % n_slabs or (lt // n_slabs) % 2:
        raise ValueError("Lt must split into slabs of an even number of time slices")
    tl = lt // n_slabs
    return [(k * tl, tl) for k in range(n_slabs)]


class SlabLattice:
    """A lattice as n slabs held by this process (contexts used round-robin)."""

    def __init__(self, ctxs, dims, n_slabs, precision="fp64", storage: int = 18):
        ctxs = ctxs if isinstance(ctxs, (list, tuple)) else [ctxs]
        self.dims = tuple(int(d) for d in dims)
        self.slabs = [Slab(ctxs[k % len(ctxs)], self.dims, t0, tl, precision, storage)
                      for k, (t0, tl) in enumerate(_split(self.dims, n_slabs))]

    def set_links(self, u: np.ndarray) -> None:
        for s in self.slabs:
            s.set_links(s.local_from_global(u))

    def get_links(self) -> np.ndarray:
        return np.concatenate([s.own(s.get_links()) for s in self.slabs], axis=0)

    def hot_start(self, seed: int) -> None:
        for s in self.slabs:  # global link ids: the halos hold the neighbours' links
            s.hot_start(seed)

    def exchange(self, which: int, mu: int = -1, parity: int = -1) -> None:
        n = len(self.slabs)
        for k in range(n):
            check(lib().qcb_slab_exchange(self.slabs[k].h, self.slabs[(k + 1) % n].h, which, mu, parity))

    def heatbath(self, beta, n_sweeps, n_hits, seed, sweep_offset=0) -> None:
        for sw in range(n_sweeps):
            for mu in range(4):
                for par in range(2):
                    for s in self.slabs:
                        s.heatbath_pass(mu, par, beta, n_hits, seed, sweep_offset + sw)
                    self.exchange(LINKS, mu, par)

    def flow_steps(self, eps, n) -> None:
        for step in range(n):
            for stage in (1, 2, 3):
                for s in self.slabs:
                    s.flow_stage(stage, eps, step)
                self.exchange(flow_dst(stage, step))
        for s in self.slabs:
            s.flow_finish(n)

    def plaquette(self) -> float:
        return float(sum(s.partial_plaquette() for s in self.slabs))

    def topo_qe(self):
        parts = [s.partial_qe() for s in self.slabs]
        return float(sum(p[0] for p in parts)), float(sum(p[1] for p in parts))

    def close(self) -> None:
        for s in self.slabs:
            s.close()


class DistSlab:
    """One slab per process of a torch.distributed group: rank r holds slab r of
    `world` equal slabs, and the faces move to the ranks r - 1 and r + 1 (periodically).

    One exchange moves every face of a pass or stage at once, ordered on the library's
    stream: the faces of each side are packed back to back into one buffer
    (qcb_slab_faces_copy_async), the four messages go as one batch (batch_isend_irecv), and
    the received faces are unpacked the same way.  With the "device" transport (NCCL) the
    host never waits: the library's stream is the current torch stream while the batch is
    issued, so the sends start after the packs and the unpacks after the receives.  With the
    "host" transport (gloo, pinned CPU buffers) the host waits once per exchange, for the packs,
    before handing the buffers to gloo."""

    def __init__(self, ctx: Context, dims, dist, precision="fp64", storage: int = 18, transport: str = "host"):
        import torch

        self.dist = dist
        self.ctx = ctx
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.dims = tuple(int(d) for d in dims)
        t0, tl = _split(self.dims, self.world)[self.rank]
        self.slab = Slab(ctx, self.dims, t0, tl, precision, storage)
        ns, nb = self.slab.face_shape()
        self.face_bytes = ns * nb
        self.device = transport != "host"
        nbytes = 8 * self.face_bytes  # all four directions and both parities
        mk = (lambda: torch.empty(nbytes, dtype=torch.uint8, device="cuda")) if self.device else \
            (lambda: torch.empty(nbytes, dtype=torch.uint8, pin_memory=True))
        self.buf = {k: mk() for k in ("send_lo", "send_hi", "recv_lo", "recv_hi")}
        self.stream = torch.cuda.ExternalStream(ctx.stream) if self.device else None

    def _copy(self, which, side, mu, parity, key, to_face) -> None:
        check(lib().qcb_slab_faces_copy_async(self.slab.h, which, side, mu, parity,
                                              C.c_void_p(self.buf[key].data_ptr()), 1 if to_face else 0))

    def exchange(self, which: int, mu: int = -1, parity: int = -1) -> None:
        import torch

        if self.world == 1:  # the slab is its own neighbour
            check(lib().qcb_slab_exchange(self.slab.h, self.slab.h, which, mu, parity))
            return
        n = (4 if mu < 0 else 1) * (2 if parity < 0 else 1) * self.face_bytes
        lo, hi = (self.rank - 1) % self.world, (self.rank + 1) % self.world
        b = self.buf
        # my first own slice goes to the rank below (its high halo), my last to the rank above
        # (its low halo); the message order below is the matching order on every rank
        self._copy(which, 1, mu, parity, "send_lo", False)
        self._copy(which, 2, mu, parity, "send_hi", False)
        ops = [self.dist.P2POp(self.dist.isend, b["send_lo"][:n], lo),
               self.dist.P2POp(self.dist.isend, b["send_hi"][:n], hi),
               self.dist.P2POp(self.dist.irecv, b["recv_hi"][:n], hi),
               self.dist.P2POp(self.dist.irecv, b["recv_lo"][:n], lo)]
        if self.device:
            with torch.cuda.stream(self.stream):
                for r in self.dist.batch_isend_irecv(ops):
                    r.wait()  # orders the library stream after the receives; the host goes on
        else:
            self.ctx.sync()  # the packed faces are in the pinned buffers
            for r in self.dist.batch_isend_irecv(ops):
                r.wait()
        self._copy(which, 0, mu, parity, "recv_lo", True)
        self._copy(which, 3, mu, parity, "recv_hi", True)

    def heatbath(self, beta, n_sweeps, n_hits, seed, sweep_offset=0) -> None:
        for sw in range(n_sweeps):
            for mu in range(4):
                for par in range(2):
                    self.slab.heatbath_pass(mu, par, beta, n_hits, seed, sweep_offset + sw)
                    self.exchange(LINKS, mu, par)

    def flow_steps(self, eps, n) -> None:
        for step in range(n):
            for stage in (1, 2, 3):
                self.slab.flow_stage(stage, eps, step)
                self.exchange(flow_dst(stage, step))
        self.slab.flow_finish(n)

    def _sum(self, values):
        import torch

        t = torch.tensor(values, dtype=torch.float64, device=self.buf["send_lo"].device)
        self.dist.all_reduce(t)
        return [float(v) for v in t.cpu()]

    def plaquette(self) -> float:
        return self._sum([self.slab.partial_plaquette()])[0]

    def topo_qe(self):
        q, e = self._sum(list(self.slab.partial_qe()))
        return q, e
