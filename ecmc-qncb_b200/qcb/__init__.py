"""qcb — Python mirror of the ECMC-QNCB heatbath / plaquette / Wilson-flow interface on the
B200 library (libqcb.so, C ABI in include/qcb.h).

The names follow the reference's function boundary:

    reference (C++, MPI)                                   here
    ---------------------------------------------------------------------------------------
    GaugeField(geo), hot_start, cold_start                 GaugeField(ctx, L or dims, ...)
      (src/gauge/GaugeField.h:18-62)
    mpi::heatbathcb::samples(field, geo, topo, hp, rng)    heatbathcb.samples(field, hp, rng)
      (src/heatbath/heatbath_mpi.h:17)
    mpi::observables::mean_plaquette_global(field, ...)    observables.mean_plaquette_global(field)
    mpi::observables::topo_q_e_clover_global(field, ...)   observables.topo_q_e_clover_global(field)
    mpi::observables::topo_charge_flowed(field, geo, gf,   observables.topo_charge_flowed(field, gf,
        topo, N_steps_gf, N_rk_steps)                          N_steps_gf, N_rk_steps)
      (src/observables/observables_mpi.h:9-18)
    GradientFlow(eps, field, geo)                          GradientFlow(eps)
    save_ildg_clime / read_ildg_clime(run_name, run_dir,   save_ildg_clime / read_ildg_clime(run_name,
        field, geo, topo) (src/io/ildg.h:17-20)                run_dir, field)
    io::load_params(file, RunParamsHbCB&) (io.cpp:353)     io.load_params(file) -> HbParams

The reference's std::mt19937_64 is replaced by a counter-based stream: `rng` here is a
PhiloxStream (seed + sweep counter), so a chain is reproducible from (seed, sweep).
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from dataclasses import dataclass

import numpy as np

from ._lib import (FP32, FP64, R12, R18, BatchPlan, HbParams, Job, JobResult, QcbError, ServerConfig, ServerStats,
                   check, lib)

__all__ = ["Context", "GaugeField", "Batch", "BatchPlan", "Server", "PhiloxStream", "GradientFlow", "HbParams", "QcbError", "heatbathcb",
           "EventChains", "EcmcParams", "ecmccb",
           "observables", "io", "save_ildg_clime", "read_ildg_clime", "FP32", "FP64", "R12", "R18",
           "device_count"]


def device_count() -> int:
    n = C.c_int()
    check(lib().qcb_device_count(C.byref(n)))
    return n.value


class Context:
    """One CUDA device + stream (qcb_ctx)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(lib().qcb_ctx_create(device, 0, C.byref(h)))
        self.h = h
        self.device = device
        self._children = []  # weak references, in creation order

    def _adopt(self, obj) -> None:
        self._children.append(weakref.ref(obj))

    def sync(self) -> None:
        check(lib().qcb_ctx_sync(self.h))

    def launches(self) -> int:
        n = C.c_uint64()
        check(lib().qcb_ctx_launch_count(self.h, C.byref(n)))
        return n.value

    def set_block(self, threads: int) -> None:
        check(lib().qcb_ctx_set_block(self.h, threads))

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        check(lib().qcb_ctx_stream(self.h, C.byref(s)))
        return s.value or 0

    def close(self) -> None:
        """Closes the objects created on this context (newest first), then the context."""
        if getattr(self, "h", None):
            for ref in reversed(self._children):
                obj = ref()
                if obj is not None:
                    obj.close()
            self._children = []
            lib().qcb_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _precision(p) -> int:
    if p in (FP64, "fp64", "f64", "double"):
        return FP64
    if p in (FP32, "fp32", "f32", "float"):
        return FP32
    raise ValueError(f"bad precision {p!r}")


class GaugeField:
    """Periodic SU(3) gauge field on the device (qcb_lattice); starts cold."""

    def __init__(self, ctx: Context, L, precision="fp64", storage: int = R18):
        dims = (L, L, L, L) if isinstance(L, int) else tuple(int(d) for d in L)
        if len(dims) != 4:
            raise ValueError("dims must have 4 entries (Lx, Ly, Lz, Lt)")
        self.ctx = ctx
        self.dims = dims
        self.precision = _precision(precision)
        self.storage = int(storage)
        h = C.c_void_p()
        check(lib().qcb_lattice_create(ctx.h, (C.c_int * 4)(*dims), self.precision, self.storage, C.byref(h)))
        self.h = h
        ctx._adopt(self)

    @property
    def volume(self) -> int:
        lx, ly, lz, lt = self.dims
        return lx * ly * lz * lt

    @property
    def shape(self):
        lx, ly, lz, lt = self.dims
        return (lt, lz, ly, lx, 4, 3, 3)

    def device_bytes(self) -> int:
        b = C.c_size_t()
        check(lib().qcb_lattice_info(self.h, None, None, None, C.byref(b)))
        return b.value

    def device_links(self):
        p, st, nc, cb = C.c_void_p(), C.c_size_t(), C.c_int(), C.c_int()
        check(lib().qcb_lattice_device_links(self.h, C.byref(p), C.byref(st), C.byref(nc), C.byref(cb)))
        return p.value, st.value, nc.value, cb.value

    def cold_start(self) -> None:
        check(lib().qcb_cold_start(self.h))

    def hot_start(self, seed: int) -> None:
        check(lib().qcb_hot_start(self.h, C.c_uint64(seed)))

    def set_links(self, u: np.ndarray) -> None:
        """Links from a host complex128 array in ILDG order, shape (Lt, Lz, Ly, Lx, 4, 3, 3)."""
        u = np.ascontiguousarray(u, dtype=np.complex128)
        if u.size != self.volume * 36:
            raise ValueError("link array size does not match the lattice")
        check(lib().qcb_set_links(self.h, u.ctypes.data_as(C.POINTER(C.c_double))))

    def set_links_ptr(self, ptr: int) -> None:
        """Links from a host address holding 72*V doubles (e.g. a pinned tensor)."""
        check(lib().qcb_set_links(self.h, C.cast(C.c_void_p(ptr), C.POINTER(C.c_double))))

    def get_links(self) -> np.ndarray:
        u = np.empty(self.shape, np.complex128)
        check(lib().qcb_get_links(self.h, u.ctypes.data_as(C.POINTER(C.c_double))))
        return u

    def copy_from(self, other: "GaugeField") -> None:
        check(lib().qcb_copy_links(self.h, other.h))

    def reunitarize(self) -> None:
        check(lib().qcb_reunitarize(self.h))

    def gauge_transform(self, seed: int) -> None:
        check(lib().qcb_gauge_transform(self.h, C.c_uint64(seed)))

    def heatbath_frozen(self, beta, n_sweeps, n_hits, seed, sweep_offset, l_core, shift) -> None:
        """Heatbath sweeps with the reference's frozen links of l_core blocks after the
        cumulative translation `shift` (qcb_heatbath_frozen)."""
        check(lib().qcb_heatbath_frozen(self.h, float(beta), int(n_sweeps), int(n_hits), C.c_uint64(seed),
                                        C.c_uint64(sweep_offset), int(l_core), (C.c_int * 4)(*shift)))

    def translate(self, shift) -> None:
        """U'(x) = U(x - shift), periodic (mpi::shift::shift_field on one device)."""
        check(lib().qcb_translate(self.h, (C.c_int * 4)(*shift)))

    def save_ildg(self, path) -> None:
        check(lib().qcb_save_ildg(self.h, os.fsencode(path)))

    def load_ildg(self, path) -> None:
        check(lib().qcb_load_ildg(self.h, os.fsencode(path)))

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().qcb_lattice_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many lattices advanced by one persistent launch per phase (qcb_batch).  Borrows the
    fields, which must outlive it."""

    def __init__(self, ctx: Context, fields):
        self.ctx = ctx
        self.fields = list(fields)
        arr = (C.c_void_p * len(self.fields))(*[f.h.value for f in self.fields])
        h = C.c_void_p()
        check(lib().qcb_batch_create(ctx.h, len(self.fields), arr, C.byref(h)))
        self.h = h
        ctx._adopt(self)

    @property
    def n(self) -> int:
        return len(self.fields)

    @staticmethod
    def _u64(v):
        return (C.c_uint64 * len(v))(*[int(x) for x in v])

    @staticmethod
    def _f64(v):
        return (C.c_double * len(v))(*[float(x) for x in v])

    def set_tiles(self, hb=None, flow=None) -> None:
        mk = lambda v: None if v is None else (C.c_int * self.n)(*v)  # noqa: E731
        check(lib().qcb_batch_set_tiles(self.h, mk(hb), mk(flow)))

    def tiles(self):
        hb, fl = (C.c_int * self.n)(), (C.c_int * self.n)()
        check(lib().qcb_batch_get_tiles(self.h, hb, fl))
        return list(hb), list(fl)

    def heatbath(self, betas, n_sweeps, n_hits, seeds, sweep_offsets) -> None:
        check(lib().qcb_batch_heatbath(self.h, self._f64(betas), int(n_sweeps), int(n_hits), self._u64(seeds),
                                       self._u64(sweep_offsets)))

    def flow_steps(self, eps, n) -> None:
        check(lib().qcb_batch_flow_steps(self.h, float(eps), int(n)))

    def plaquette(self) -> np.ndarray:
        out = np.zeros(self.n)
        check(lib().qcb_batch_plaquette(self.h, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def topo_qe(self):
        q, e = np.zeros(self.n), np.zeros(self.n)
        check(lib().qcb_batch_topo_qe(self.h, q.ctypes.data_as(C.POINTER(C.c_double)),
                                      e.ctypes.data_as(C.POINTER(C.c_double))))
        return q, e

    def run(self, betas, seeds, sweep_offsets, n_sweeps, n_hits=1, eps=0.02, n_groups=0, rk_per_group=0):
        """Graph-captured workload; returns (plaquette[n], records[n, n_groups+1, 3], used_graph)."""
        plan = BatchPlan(int(n_sweeps), int(n_hits), float(eps), int(n_groups), int(rk_per_group))
        per = 1 + 3 * (n_groups + 1)
        out = np.zeros(self.n * per)
        used = C.c_int()
        check(lib().qcb_batch_run(self.h, C.byref(plan), self._f64(betas), self._u64(seeds),
                                  self._u64(sweep_offsets), out.ctypes.data_as(C.POINTER(C.c_double)),
                                  C.byref(used)))
        out = out.reshape(self.n, per)
        return out[:, 0].copy(), out[:, 1:].reshape(self.n, n_groups + 1, 3), bool(used.value)

    def autotune(self, cache_path=None) -> None:
        check(lib().qcb_batch_autotune(self.h, None if cache_path is None else os.fsencode(cache_path)))

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().qcb_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


JOB_FLOW, JOB_SWEEPS = 1, 2


class Server:
    """Request server with continuous batching (qcb_server)."""

    def __init__(self, ctx: Context, precision="fp32", storage: int = R12, hbm_budget: int = 0, max_jobs: int = 0,
                 quantum_sweeps: int = 0, quantum_steps: int = 0, tile: int = 0):
        cfg = ServerConfig(_precision(precision), int(storage), int(hbm_budget), int(max_jobs), int(quantum_sweeps),
                           int(quantum_steps), int(tile))
        h = C.c_void_p()
        check(lib().qcb_server_create(ctx.h, C.byref(cfg), C.byref(h)))
        self.h = h
        self.ctx = ctx
        ctx._adopt(self)

    def submit_sweeps(self, field: GaugeField, beta, n_sweeps, seed, sweep_offset=0, n_hits=1) -> int:
        job = Job(JOB_SWEEPS, field.h.value, float(beta), int(seed), int(sweep_offset), int(n_sweeps), int(n_hits),
                  0.0, 0)
        jid = C.c_uint64()
        check(lib().qcb_server_submit(self.h, C.byref(job), C.byref(jid)))
        return jid.value

    def submit_flow(self, field: GaugeField, eps, n_steps) -> int:
        job = Job(JOB_FLOW, field.h.value, 0.0, 0, 0, 0, 1, float(eps), int(n_steps))
        jid = C.c_uint64()
        check(lib().qcb_server_submit(self.h, C.byref(job), C.byref(jid)))
        return jid.value

    def poll(self, max_results: int = 256):
        buf = (JobResult * max_results)()
        n = C.c_int()
        check(lib().qcb_server_poll(self.h, buf, max_results, C.byref(n)))
        return [buf[k] for k in range(n.value)]

    def drain(self, timeout_s: float = 600.0) -> None:
        check(lib().qcb_server_drain(self.h, float(timeout_s)))

    def cancel(self, job_id: int) -> None:
        check(lib().qcb_server_cancel(self.h, C.c_uint64(job_id)))

    def clock(self) -> float:
        return lib().qcb_server_clock(self.h)

    def stats(self) -> dict:
        st = ServerStats()
        check(lib().qcb_server_stats_get(self.h, C.byref(st)))
        return {name: getattr(st, name) for name, _ in st._fields_}

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().qcb_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class PhiloxStream:
    """Counter-based replacement of the reference's per-rank std::mt19937_64: the key is the
    seed, and `sweep` counts the heatbath sweeps drawn so far."""
    seed: int
    sweep: int = 0


@dataclass
class GradientFlow:
    """GradientFlow(epsilon) (src/flow/gradient_flow.h:11-27); work buffers live with the field."""
    epsilon: float = 0.02


class heatbathcb:
    """mpi::heatbathcb (src/heatbath/heatbath_mpi.h:14-18)."""

    @staticmethod
    def samples(field: GaugeField, hp, rng: PhiloxStream) -> None:
        """hp.N_samples x hp.N_sweeps checkerboard sweeps of hp.N_hits Cabibbo-Marinari hits."""
        n = int(getattr(hp, "N_samples", 1)) * int(hp.N_sweeps)
        check(lib().qcb_heatbath(field.h, float(hp.beta), n, int(hp.N_hits), C.c_uint64(rng.seed),
                                 C.c_uint64(rng.sweep)))
        rng.sweep += n

    @staticmethod
    def sweep(field: GaugeField, beta: float, N_hits: int, rng: PhiloxStream) -> None:
        check(lib().qcb_heatbath(field.h, float(beta), 1, int(N_hits), C.c_uint64(rng.seed), C.c_uint64(rng.sweep)))
        rng.sweep += 1

    @staticmethod
    def samples_plaquette(field: GaugeField, hp, rng: PhiloxStream) -> float:
        """samples() followed by mean_plaquette_global(), with the plaquette summed inside the
        last sweep (one call, no separate plaquette launch)."""
        n = int(getattr(hp, "N_samples", 1)) * int(hp.N_sweeps)
        out = C.c_double()
        check(lib().qcb_heatbath_plaquette(field.h, float(hp.beta), n, int(hp.N_hits), C.c_uint64(rng.seed),
                                           C.c_uint64(rng.sweep), C.byref(out)))
        rng.sweep += n
        return out.value


class observables:
    """mpi::observables (src/observables/observables_mpi.h:9-18)."""

    @staticmethod
    def mean_plaquette_global(field: GaugeField) -> float:
        out = C.c_double()
        check(lib().qcb_plaquette(field.h, C.byref(out)))
        return out.value

    @staticmethod
    def topo_q_e_clover_global(field: GaugeField):
        q, e = C.c_double(), C.c_double()
        check(lib().qcb_topo_qe(field.h, C.byref(q), C.byref(e)))
        return q.value, e.value

    @staticmethod
    def topo_charge_flowed(field: GaugeField, gf: GradientFlow, N_steps_gf: int, N_rk_steps: int) -> np.ndarray:
        out = np.zeros(3 * int(N_steps_gf))
        check(lib().qcb_flow_measure(field.h, float(gf.epsilon), int(N_steps_gf), int(N_rk_steps),
                                     out.ctypes.data_as(C.POINTER(C.c_double))))
        return out


def save_ildg_clime(run_name: str, run_dir: str, field: GaugeField) -> str:
    """save_ildg_clime (src/io/ildg.cpp:34-136): writes run_dir/run_name/run_name."""
    d = os.path.join(run_dir, run_name)
    os.makedirs(d, exist_ok=True)
    path = os.path.join(d, run_name)
    field.save_ildg(path)
    return path


def read_ildg_clime(run_name: str, run_dir: str, field: GaugeField) -> None:
    """read_ildg_clime (src/io/ildg.cpp:138-237): reads run_dir/run_name/run_name."""
    field.load_ildg(os.path.join(run_dir, run_name, run_name))


class io:
    """io::load_params (src/io/io.cpp:353-399) with the defaults of src/io/params.h."""

    @staticmethod
    def default_params() -> HbParams:
        p = HbParams()
        check(lib().qcb_params_default(C.byref(p)))
        return p

    @staticmethod
    def load_params(path) -> HbParams:
        p = io.default_params()
        check(lib().qcb_params_load(os.fsencode(path), C.byref(p)))
        return p

    @staticmethod
    def load_ecmc_params(path):
        """io::load_params(file, RunParamsECB&) (src/io/io.cpp:298-341) -> EcmcRunParams."""
        from ._lib import EcmcRunParams
        p = EcmcRunParams()
        check(lib().qcb_ecmc_run_params_default(C.byref(p)))
        check(lib().qcb_ecmc_run_params_load(os.fsencode(path), C.byref(p)))
        return p

    @staticmethod
    def ildg_probe(path):
        off, n = C.c_uint64(), C.c_uint64()
        check(lib().qcb_ildg_probe(os.fsencode(path), C.byref(off), C.byref(n)))
        return off.value, n.value


from ._lib import EcmcParams  # noqa: E402
from .ecmc import CHAIN_DTYPE, EventChains, ecmccb  # noqa: E402
