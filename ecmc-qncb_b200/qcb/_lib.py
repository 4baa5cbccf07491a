"""ctypes binding of libqcb.so (the C ABI declared in include/qcb.h).

The library is the in-tree build ecmc-qncb_b200/lib/libqcb.so.  There is no fallback:
if it is missing, every entry point raises QcbError, and on a host without a CUDA device
context creation fails with the library's own error.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent.parent
LIB_PATH = Path(os.environ.get("QCB_LIB", PKG_DIR / "lib" / "libqcb.so"))

QCB_OK = 0
ERRORS = {1: "INVALID", 2: "CUDA", 3: "IO", 4: "FORMAT", 5: "NOMEM", 6: "KP_CAP", 7: "STATE", 8: "CANCELLED"}
FP64, FP32 = 0, 1
R18, R12 = 18, 12


class QcbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"qcb error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class BatchPlan(C.Structure):
    """qcb_batch_plan."""
    _fields_ = [("n_sweeps", C.c_int), ("n_hits", C.c_int), ("eps", C.c_double), ("n_groups", C.c_int),
                ("rk_per_group", C.c_int)]


class Job(C.Structure):
    """qcb_job."""
    _fields_ = [("kind", C.c_int), ("lat", C.c_void_p), ("beta", C.c_double), ("seed", C.c_uint64),
                ("sweep_offset", C.c_uint64), ("n_sweeps", C.c_int), ("n_hits", C.c_int), ("eps", C.c_double),
                ("n_steps", C.c_int)]


class JobResult(C.Structure):
    """qcb_job_result."""
    _fields_ = [("id", C.c_uint64), ("status", C.c_int), ("kind", C.c_int), ("plaquette", C.c_double),
                ("t", C.c_double), ("q", C.c_double), ("e", C.c_double), ("submit_s", C.c_double),
                ("admit_s", C.c_double), ("finish_s", C.c_double)]


class ServerConfig(C.Structure):
    """qcb_server_config."""
    _fields_ = [("precision", C.c_int), ("storage", C.c_int), ("hbm_budget", C.c_size_t), ("max_jobs", C.c_int),
                ("quantum_sweeps", C.c_int), ("quantum_steps", C.c_int), ("tile", C.c_int)]


class ServerStats(C.Structure):
    """qcb_server_stats."""
    _fields_ = [("submitted", C.c_uint64), ("admitted", C.c_uint64), ("completed", C.c_uint64),
                ("ticks", C.c_uint64), ("max_active", C.c_int), ("arena_bytes", C.c_size_t),
                ("arena_peak", C.c_size_t)]


class HbParams(C.Structure):
    """qcb_hb_params: RunParamsHbCB of the reference (src/io/params.h:46-63)."""
    _fields_ = [("L_core", C.c_int), ("n_core_dims", C.c_int), ("cold_start", C.c_int),
                ("N_switch_eo", C.c_int), ("N_shift", C.c_int), ("seed", C.c_int),
                ("beta", C.c_double),
                ("N_samples", C.c_int), ("N_hits", C.c_int), ("N_sweeps", C.c_int), ("N_therm", C.c_int),
                ("topo", C.c_int), ("N_shift_plaquette", C.c_int), ("N_shift_topo", C.c_int),
                ("N_steps_gf", C.c_int), ("N_rk_steps", C.c_int), ("save_each_shifts", C.c_int),
                ("run_name", C.c_char * 256), ("run_dir", C.c_char * 1024)]

    def as_dict(self) -> dict:
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = v.decode() if isinstance(v, bytes) else v
        return d


class EcmcParams(C.Structure):
    """qcb_ecmc_params: ECMCParams of the reference (src/io/params.h:9-17) plus the block edge."""
    _fields_ = [("beta", C.c_double), ("theta_sample", C.c_double), ("theta_refresh_site", C.c_double),
                ("theta_refresh_R", C.c_double), ("epsilon_set", C.c_double), ("poisson", C.c_int),
                ("l_core", C.c_int)]


class EcmcRunParams(C.Structure):
    """qcb_ecmc_run_params: RunParamsECB of the reference (src/io/params.h:27-44)."""
    _fields_ = [("L_core", C.c_int), ("n_core_dims", C.c_int), ("cold_start", C.c_int), ("seed", C.c_int),
                ("N_shift", C.c_int), ("ecmc", EcmcParams),
                ("N_therm", C.c_int), ("topo", C.c_int), ("N_shift_plaquette", C.c_int), ("N_shift_topo", C.c_int),
                ("N_steps_gf", C.c_int), ("N_rk_steps", C.c_int), ("save_each_shifts", C.c_int),
                ("run_name", C.c_char * 256), ("run_dir", C.c_char * 1024)]

    def as_dict(self) -> dict:
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            if name == "ecmc":
                d.update({k: getattr(v, k) for k, _ in v._fields_})
            else:
                d[name] = v.decode() if isinstance(v, bytes) else v
        return d


_lib = None

# name -> (restype, argtypes)
_vp, _ip, _dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
SIGNATURES = {
    "qcb_abi_version": (C.c_int, []),
    "qcb_last_error": (C.c_char_p, []),
    "qcb_device_count": (C.c_int, [_ip]),
    "qcb_ctx_create": (C.c_int, [C.c_int, C.c_uint, C.POINTER(C.c_void_p)]),
    "qcb_ctx_destroy": (C.c_int, [_vp]),
    "qcb_ctx_sync": (C.c_int, [_vp]),
    "qcb_ctx_launch_count": (C.c_int, [_vp, C.POINTER(C.c_uint64)]),
    "qcb_ctx_set_block": (C.c_int, [_vp, C.c_int]),
    "qcb_ctx_stream": (C.c_int, [_vp, C.POINTER(C.c_void_p)]),
    "qcb_lattice_create": (C.c_int, [_vp, _ip, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "qcb_lattice_destroy": (C.c_int, [_vp]),
    "qcb_lattice_info": (C.c_int, [_vp, _ip, _ip, _ip, C.POINTER(C.c_size_t)]),
    "qcb_lattice_device_links": (C.c_int, [_vp, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t), _ip, _ip]),
    "qcb_cold_start": (C.c_int, [_vp]),
    "qcb_hot_start": (C.c_int, [_vp, C.c_uint64]),
    "qcb_set_links": (C.c_int, [_vp, _dp]),
    "qcb_get_links": (C.c_int, [_vp, _dp]),
    "qcb_copy_links": (C.c_int, [_vp, _vp]),
    "qcb_reunitarize": (C.c_int, [_vp]),
    "qcb_gauge_transform": (C.c_int, [_vp, C.c_uint64]),
    "qcb_save_ildg": (C.c_int, [_vp, C.c_char_p]),
    "qcb_load_ildg": (C.c_int, [_vp, C.c_char_p]),
    "qcb_ildg_probe": (C.c_int, [C.c_char_p, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "qcb_heatbath": (C.c_int, [_vp, C.c_double, C.c_int, C.c_int, C.c_uint64, C.c_uint64]),
    "qcb_heatbath_plaquette": (C.c_int, [_vp, C.c_double, C.c_int, C.c_int, C.c_uint64, C.c_uint64,
                                         C.POINTER(C.c_double)]),
    "qcb_heatbath_frozen": (C.c_int, [_vp, C.c_double, C.c_int, C.c_int, C.c_uint64, C.c_uint64, C.c_int, _ip]),
    "qcb_translate": (C.c_int, [_vp, _ip]),
    "qcb_plaquette": (C.c_int, [_vp, _dp]),
    "qcb_topo_qe": (C.c_int, [_vp, _dp, _dp]),
    "qcb_flow_measure": (C.c_int, [_vp, C.c_double, C.c_int, C.c_int, _dp]),
    "qcb_flow_steps": (C.c_int, [_vp, C.c_double, C.c_int]),
    "qcb_plaquette_noalloc": (C.c_int, [_vp, _ip, C.c_int, C.c_int, C.c_size_t, _vp, _vp]),
    "qcb_batch_create": (C.c_int, [_vp, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "qcb_batch_destroy": (C.c_int, [_vp]),
    "qcb_batch_set_tiles": (C.c_int, [_vp, _ip, _ip]),
    "qcb_batch_get_tiles": (C.c_int, [_vp, _ip, _ip]),
    "qcb_batch_heatbath": (C.c_int, [_vp, _dp, C.c_int, C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "qcb_batch_flow_steps": (C.c_int, [_vp, C.c_double, C.c_int]),
    "qcb_batch_plaquette": (C.c_int, [_vp, _dp]),
    "qcb_batch_topo_qe": (C.c_int, [_vp, _dp, _dp]),
    "qcb_batch_run": (C.c_int, [_vp, C.POINTER(BatchPlan), _dp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), _dp,
                                _ip]),
    "qcb_batch_autotune": (C.c_int, [_vp, C.c_char_p]),
    "qcb_server_create": (C.c_int, [_vp, C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]),
    "qcb_server_submit": (C.c_int, [_vp, C.POINTER(Job), C.POINTER(C.c_uint64)]),
    "qcb_server_poll": (C.c_int, [_vp, C.POINTER(JobResult), C.c_int, _ip]),
    "qcb_server_drain": (C.c_int, [_vp, C.c_double]),
    "qcb_server_cancel": (C.c_int, [_vp, C.c_uint64]),
    "qcb_server_stats_get": (C.c_int, [_vp, C.POINTER(ServerStats)]),
    "qcb_server_clock": (C.c_double, [_vp]),
    "qcb_server_destroy": (C.c_int, [_vp]),
    "qcb_wait_selftest": (C.c_int, [_vp, C.c_double, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "qcb_lattice_create_slab": (C.c_int, [_vp, _ip, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "qcb_slab_info": (C.c_int, [_vp, _ip, _ip, _ip]),
    "qcb_heatbath_pass": (C.c_int, [_vp, C.c_int, C.c_int, C.c_double, C.c_int, C.c_uint64, C.c_uint64]),
    "qcb_flow_stage": (C.c_int, [_vp, C.c_int, C.c_double, C.c_int]),
    "qcb_flow_finish": (C.c_int, [_vp, C.c_int]),
    "qcb_slab_exchange": (C.c_int, [_vp, _vp, C.c_int, C.c_int, C.c_int]),
    "qcb_slab_face": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p),
                                C.POINTER(C.c_size_t), _ip]),
    "qcb_slab_face_copy": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, C.c_int]),
    "qcb_slab_faces_copy_async": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int, C.c_int, _vp, C.c_int]),
    "qcb_ecmc_create": (C.c_int, [_vp, C.POINTER(EcmcParams), C.c_uint64, C.POINTER(C.c_void_p)]),
    "qcb_ecmc_destroy": (C.c_int, [_vp]),
    "qcb_ecmc_num_chains": (C.c_int, [_vp, _ip]),
    "qcb_ecmc_set_lanes": (C.c_int, [_vp, C.c_int]),
    "qcb_ecmc_lanes": (C.c_int, [_vp, _ip]),
    "qcb_ecmc_sample": (C.c_int, [_vp, _ip]),
    "qcb_ecmc_sample_n": (C.c_int, [_vp, _ip, C.c_int]),
    "qcb_ecmc_counters": (C.c_int, [_vp, C.POINTER(C.c_uint64), C.c_int]),
    "qcb_ecmc_get_chains": (C.c_int, [_vp, _vp, C.POINTER(C.c_uint64)]),
    "qcb_ecmc_set_chains": (C.c_int, [_vp, _vp, C.c_uint64]),
    "qcb_params_default": (C.c_int, [C.POINTER(HbParams)]),
    "qcb_params_load": (C.c_int, [C.c_char_p, C.POINTER(HbParams)]),
    "qcb_ecmc_run_params_default": (C.c_int, [C.POINTER(EcmcRunParams)]),
    "qcb_ecmc_run_params_load": (C.c_int, [C.c_char_p, C.POINTER(EcmcRunParams)]),
}


def lib():
    """Load libqcb.so and declare its signatures (raises if the build is missing)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise QcbError(2, f"libqcb.so not found at {LIB_PATH}: run ecmc-qncb_b200/build.py")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != QCB_OK:
        msg = lib().qcb_last_error()
        raise QcbError(rc, msg.decode() if msg else "")
