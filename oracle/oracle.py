"""ctypes loader for the FP64 CPU oracle (oracle/qcb_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline / reference arm, as the checker.  The product (libqcb and the qcb package) never
imports it.  Parity unpinned: the reference itself cannot be built here (no MPI, Eigen or
c-lime), so this restatement is checked against known answers, not reference outputs.

Arrays use the ILDG site order of the reference: shape (Lt, Lz, Ly, Lx, 4, 3, 3) complex128,
i.e. 72 doubles per site.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "liborc.so"

_lib = None
_build_kind = "checker"


def build() -> Path:
    """Compile liborc.so, the checker, with the committed Makefile (g++, FP64, -O2, no FMA
    contraction on the baseline x86-64 target, so its rounding is fixed)."""
    subprocess.run(["make", "-s", "-f", str(HERE / "Makefile")], check=True)
    return LIB_PATH


def _host_tag() -> str:
    """Short hash of the host CPU's model and feature flags: the timing build targets the
    host it runs on (-march=native), so each kind of host gets its own file."""
    import hashlib

    info = ""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith(("model name", "flags")):
                info += line
                if line.startswith("flags"):
                    break
    except OSError:
        pass
    return hashlib.sha1(info.encode()).hexdigest()[:12]


def fast_lib_path() -> Path:
    return HERE / "_build" / f"liborc_fast-{_host_tag()}.so"


def build_fast() -> Path:
    """Compile the timing build of the same source as the reference's release build is
    compiled (CMakeLists.txt:88-102: -O3 with the host's instruction set): -O3 -march=native
    -fcx-limited-range (complex products without the __muldc3 call).  Only the CPU baseline
    uses it; its rounding differs from the checker's (FMA contraction)."""
    out = fast_lib_path()
    subprocess.run(["make", "-s", "-f", str(HERE / "Makefile"), "fast", f"FAST_OUT={out}"], check=True)
    return out


def select_build(kind: str) -> None:
    """'checker' (default): liborc.so.  'fast': the timing build for this host, built on
    first use.  Must be called before the first call into the oracle in this process."""
    global _build_kind
    if _lib is not None and kind != _build_kind:
        raise RuntimeError("the oracle library is already loaded")
    if kind not in ("checker", "fast"):
        raise ValueError(kind)
    _build_kind = kind


def build_flags() -> str:
    return "-O2 (checker)" if _build_kind == "checker" else "-O3 -march=native -fcx-limited-range, neighbour table"


def lib():
    global _lib
    if _lib is None:
        if _build_kind == "fast":
            path = fast_lib_path()
            if not path.exists():
                build_fast()
        else:
            path = LIB_PATH
            if not path.exists():
                build()
        L = C.CDLL(str(path))
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
        u32p = C.POINTER(C.c_uint32)
        L.orc_plaquette.argtypes = [dp, ip, dp]
        L.orc_topo_qe.argtypes = [dp, ip, dp, dp]
        L.orc_flow_measure.argtypes = [dp, ip, C.c_double, C.c_int, C.c_int, dp]
        L.orc_flow_steps.argtypes = [dp, ip, C.c_double, C.c_int]
        L.orc_staple.argtypes = [dp, ip, C.c_long, C.c_int, dp]
        L.orc_exp_su3.argtypes = [dp, C.c_double, dp]
        L.orc_proj_lie.argtypes = [dp, dp]
        L.orc_philox.argtypes = [u32p, u32p, u32p]
        L.orc_mt19937_64_nth.argtypes = [C.c_uint64, C.c_int]
        L.orc_mt19937_64_nth.restype = C.c_uint64
        L.orc_heatbath_cb.argtypes = [dp, ip, C.c_double, C.c_int, C.c_int, C.c_uint64, C.c_uint64]
        L.orc_heatbath_cb.restype = C.c_uint64
        L.orc_heatbath_cb_frozen.argtypes = [dp, ip, C.c_double, C.c_int, C.c_int, C.c_uint64, C.c_uint64,
                                             C.c_int, ip]
        L.orc_heatbath_cb_frozen.restype = C.c_uint64
        L.orc_shift_sequence.argtypes = [C.c_uint64, C.c_int, C.c_int, ip]
        L.orc_hot_start_philox.argtypes = [dp, ip, C.c_uint64]
        L.orc_gauge_transform_philox.argtypes = [dp, ip, C.c_uint64]
        L.orc_kp_samples.argtypes = [C.c_double, C.c_double, C.c_int, C.c_uint64, dp]
        L.orc_ref_create.argtypes = [C.c_int, C.c_int, C.c_int]
        L.orc_ref_create.restype = C.c_void_p
        L.orc_ref_destroy.argtypes = [C.c_void_p]
        L.orc_ref_run.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int, C.c_int, dp]
        L.orc_ref_sweeps.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int]
        L.orc_ref_get_links.argtypes = [C.c_void_p, dp]
        L.orc_ref_set_links.argtypes = [C.c_void_p, dp]
        L.orc_ecmc_solve_reject.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int, dp]
        L.orc_ecmc_compute_ds.argtypes = [dp, dp, dp]
        L.orc_ecmc_set.argtypes = [C.c_double, C.c_uint64, C.c_uint32, C.c_uint64, C.c_uint32, dp]
        L.orc_ecmc_sample.argtypes = [dp, ip, dp, ip, C.c_uint64, C.c_uint64, ip, C.c_void_p]
        L.orc_ecmc_ref_create.argtypes = [C.c_int, C.c_int, C.c_int, dp, ip]
        L.orc_ecmc_ref_create.restype = C.c_void_p
        L.orc_ecmc_ref_destroy.argtypes = [C.c_void_p]
        L.orc_ecmc_ref_run.argtypes = [C.c_void_p, C.c_int, dp, C.POINTER(C.c_uint64)]
        L.orc_ecmc_ref_get_links.argtypes = [C.c_void_p, dp]
        L.orc_ecmc_ref_set_links.argtypes = [C.c_void_p, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _dims(dims):
    return (C.c_int * 4)(*dims)


def shape(dims):
    lx, ly, lz, lt = dims
    return (lt, lz, ly, lx, 4, 3, 3)


def cold(dims) -> np.ndarray:
    u = np.zeros(shape(dims), np.complex128)
    u[..., 0, 0] = u[..., 1, 1] = u[..., 2, 2] = 1.0
    return u


def hot_philox(dims, seed: int) -> np.ndarray:
    u = np.zeros(shape(dims), np.complex128)
    lib().orc_hot_start_philox(_dp(u), _dims(dims), C.c_uint64(seed))
    return u


def plaquette(u, dims) -> float:
    u = np.ascontiguousarray(u, np.complex128)
    out = C.c_double()
    lib().orc_plaquette(_dp(u), _dims(dims), C.byref(out))
    return out.value


def topo_qe(u, dims):
    u = np.ascontiguousarray(u, np.complex128)
    q, e = C.c_double(), C.c_double()
    lib().orc_topo_qe(_dp(u), _dims(dims), C.byref(q), C.byref(e))
    return q.value, e.value


def flow_measure(u, dims, eps, n_steps_gf, n_rk_steps) -> np.ndarray:
    u = np.ascontiguousarray(u, np.complex128)
    out = np.zeros(3 * n_steps_gf)
    lib().orc_flow_measure(_dp(u), _dims(dims), eps, n_steps_gf, n_rk_steps, _dp(out))
    return out


def flow_steps(u, dims, eps, n) -> np.ndarray:
    u = np.array(u, np.complex128, copy=True)
    lib().orc_flow_steps(_dp(u), _dims(dims), eps, n)
    return u


def staple(u, dims, site, mu) -> np.ndarray:
    u = np.ascontiguousarray(u, np.complex128)
    out = np.zeros((3, 3), np.complex128)
    lib().orc_staple(_dp(u), _dims(dims), site, mu, _dp(out))
    return out


def exp_su3(z, coeff) -> np.ndarray:
    z = np.ascontiguousarray(z, np.complex128)
    out = np.zeros((3, 3), np.complex128)
    lib().orc_exp_su3(_dp(z), coeff, _dp(out))
    return out


def proj_lie(a) -> np.ndarray:
    a = np.ascontiguousarray(a, np.complex128)
    out = np.zeros((3, 3), np.complex128)
    lib().orc_proj_lie(_dp(a), _dp(out))
    return out


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox(c, k, o)
    return list(o)


def mt19937_64_nth(seed: int, n: int) -> int:
    return lib().orc_mt19937_64_nth(seed, n)


def heatbath_cb(u, dims, beta, n_sweeps, n_hits, seed, sweep_offset=0):
    """The library's checkerboard/Philox heatbath restated in FP64; returns (links, kp_fails)."""
    u = np.array(u, np.complex128, copy=True)
    fails = lib().orc_heatbath_cb(_dp(u), _dims(dims), beta, n_sweeps, n_hits, C.c_uint64(seed),
                                  C.c_uint64(sweep_offset))
    return u, int(fails)


def heatbath_cb_frozen(u, dims, beta, n_sweeps, n_hits, seed, sweep_offset, lcore, shift):
    """heatbath_cb with the reference's frozen links of lcore blocks after the cumulative
    translation `shift` (links with (c_d + shift_d) % lcore == 0 for some d != mu stay)."""
    u = np.array(u, np.complex128, copy=True)
    fails = lib().orc_heatbath_cb_frozen(_dp(u), _dims(dims), beta, n_sweeps, n_hits, C.c_uint64(seed),
                                         C.c_uint64(sweep_offset), int(lcore), (C.c_int * 4)(*shift))
    return u, int(fails)


def shift_sequence(seed: int, L: int, n: int) -> np.ndarray:
    """The first n shift vectors (x, y, z, t) the reference draws from mt19937_64(seed)."""
    out = (C.c_int * (4 * n))()
    lib().orc_shift_sequence(C.c_uint64(seed), int(L), int(n), out)
    return np.array(out[:], dtype=np.int64).reshape(n, 4)


def gauge_transform_philox(u, dims, seed):
    u = np.array(u, np.complex128, copy=True)
    lib().orc_gauge_transform_philox(_dp(u), _dims(dims), C.c_uint64(seed))
    return u


def kp_samples(beta, k, n, seed) -> np.ndarray:
    out = np.zeros(n)
    lib().orc_kp_samples(beta, k, n, C.c_uint64(seed), _dp(out))
    return out


class RefChain:
    """Single-rank reference schedule: frozen links + random shift + lexicographic sweep
    with std::mt19937_64 (src/bin/gauge_hb_ncb.cpp:18-179)."""

    def __init__(self, L: int, seed: int, cold_start: bool):
        self.L = L
        self.h = lib().orc_ref_create(L, seed, 1 if cold_start else 0)

    def run(self, beta, n_shift, n_sweeps=1, n_hits=1) -> np.ndarray:
        out = np.zeros(n_shift)
        lib().orc_ref_run(self.h, beta, n_shift, n_sweeps, n_hits, _dp(out))
        return out

    def sweeps(self, beta, n_sweeps, n_hits=1):
        lib().orc_ref_sweeps(self.h, beta, n_sweeps, n_hits)

    def links(self) -> np.ndarray:
        u = np.zeros(shape((self.L,) * 4), np.complex128)
        lib().orc_ref_get_links(self.h, _dp(u))
        return u

    def set_links(self, u):
        u = np.ascontiguousarray(u, np.complex128)
        lib().orc_ref_set_links(self.h, _dp(u))

    def updates_per_sweep(self) -> int:
        L = self.L
        return 4 * L * (L - 1) ** 3

    def __del__(self):
        try:
            lib().orc_ref_destroy(self.h)
        except Exception:
            pass


# ---- ILDG / LIME restatement (src/io/ildg.cpp:13-237) ------------------------------------
_LIME_MAGIC = 0x456789AB


def ildg_xml(dims) -> bytes:
    """generate_ildg_xml (src/io/ildg.cpp:13-22) with per-axis extents."""
    lx, ly, lz, lt = dims
    return ('<?xml version="1.0" encoding="UTF-8"?>\n'
            '<ildgFormat><version>1.0</version><field>su3gauge</field>'
            f'<precision>64</precision><lx>{lx}</lx><ly>{ly}</ly><lz>{lz}</lz><lt>{lt}</lt>'
            '</ildgFormat>').encode()


def _lime_header(mb: bool, me: bool, rtype: str, nbytes: int) -> bytes:
    import struct
    flags = (0x8000 if mb else 0) | (0x4000 if me else 0)
    return struct.pack(">IHHQ", _LIME_MAGIC, 1, flags, nbytes) + rtype.encode().ljust(128, b"\0")


def write_ildg(path, u, dims) -> None:
    """LIME file: 'ildg-format' record (MB=1, ME=1), padding, 'ildg-binary-data' header
    (MB=0, ME=1), then big-endian FP64 links in t, z, y, x, mu, i, j, (re, im) order."""
    xml = ildg_xml(dims)
    data = np.ascontiguousarray(u, np.complex128).view(np.float64).astype(">f8").tobytes()
    with open(path, "wb") as f:
        f.write(_lime_header(True, True, "ildg-format", len(xml)))
        f.write(xml)
        f.write(b"\0" * ((8 - len(xml) % 8) % 8))
        f.write(_lime_header(False, True, "ildg-binary-data", len(data)))
        f.write(data)


def read_ildg(path, dims) -> np.ndarray:
    """Scan LIME records for 'ildg-binary-data', check its size, decode big-endian FP64."""
    import struct
    raw = open(path, "rb").read()
    pos = 0
    expected = int(np.prod(dims)) * 72 * 8
    while pos + 144 <= len(raw):
        magic, _ver, _flags, n = struct.unpack(">IHHQ", raw[pos:pos + 16])
        if magic != _LIME_MAGIC:
            raise ValueError("bad LIME magic")
        rtype = raw[pos + 16:pos + 144].split(b"\0")[0].decode()
        pos += 144
        if rtype == "ildg-binary-data":
            if n != expected:
                raise ValueError("binary data size mismatch")
            buf = np.frombuffer(raw[pos:pos + n], dtype=">f8").astype(np.float64)
            if buf.size * 8 != n:
                raise ValueError("truncated binary data")
            return buf.view(np.complex128).reshape(shape(dims)).copy()
        pos += n + (8 - n % 8) % 8
    raise ValueError("record 'ildg-binary-data' not found")


# ---- input-file parser restatement (src/io/io.cpp:290-295, 353-399) -----------------------
def _stoi(s: str) -> int:
    import re
    m = re.match(r"[\s]*([+-]?\d+)", s)
    if not m:
        raise ValueError("stoi")
    v = int(m.group(1))
    if not -2**31 <= v < 2**31:
        raise OverflowError("stoi")
    return v


def _stod(s: str) -> float:
    import re
    m = re.match(r"[\s]*([+-]?(\d+\.?\d*([eE][+-]?\d+)?|\.\d+([eE][+-]?\d+)?|inf(inity)?|nan))", s, re.I)
    if not m:
        raise ValueError("stod")
    return float(m.group(1))


HB_DEFAULTS = dict(L_core=6, n_core_dims=2, cold_start=1, N_switch_eo=3, N_shift=2, seed=123, beta=6.0,
                   N_samples=10, N_hits=1, N_sweeps=1, N_therm=100, topo=1, N_shift_plaquette=2,
                   N_shift_topo=10, N_steps_gf=10, N_rk_steps=40, save_each_shifts=2, run_name="c",
                   run_dir="data")


def load_params(path) -> dict:
    """io::load_params(..., RunParamsHbCB&): returns the parameter dict (defaults from
    src/io/params.h:46-63); raises ValueError/OverflowError where std::stoi/stod throw."""
    cfg = {}
    with open(path, "rb") as f:
        for raw in f.read().split(b"\n"):
            line = raw.decode("latin-1")
            if not line or line[0] == "#":
                continue
            if "=" not in line:
                continue
            key, value = line.split("=", 1)
            if value == "":
                continue
            cfg[key.strip(" \t")] = value.strip(" \t")
    p = dict(HB_DEFAULTS)
    ints = {"L_core": "L_core", "n_core_dims": "n_core_dims", "seed": "seed", "N_shift": "N_shift",
            "N_sweeps": "N_sweeps", "N_hits": "N_hits", "N_shift_plaquette": "N_shift_plaquette",
            "N_shift_therm": "N_therm", "N_shift_topo": "N_shift_topo", "N_steps_gf": "N_steps_gf",
            "N_rk_steps": "N_rk_steps", "save_each_shifts": "save_each_shifts"}
    for k, dst in ints.items():
        if k in cfg:
            p[dst] = _stoi(cfg[k])
    if "cold_start" in cfg:
        p["cold_start"] = int(cfg["cold_start"] == "true")
    if "topo" in cfg:
        p["topo"] = int(cfg["topo"] == "true")
    if "beta" in cfg:
        p["beta"] = _stod(cfg["beta"])
    p["N_samples"] = 1
    for k in ("run_name", "run_dir"):
        if k in cfg:
            p[k] = cfg[k]
    return p


# ---- event-chain Monte Carlo (library form of mpi::ecmccb::sample_persistant) ------------
# One record per chain, the layout of qcb_ecmc_chain in include/qcb.h (256 bytes).
ECMC_CHAIN_DTYPE = np.dtype([
    ("R", np.complex128, (3, 3)),
    ("theta_refresh_site", np.float64), ("theta_refresh_R", np.float64),
    ("travelled_site", np.float64), ("travelled_R", np.float64),
    ("draws", np.uint64), ("events", np.uint64), ("lifts", np.uint64), ("revs", np.uint64),
    ("site", np.int32, (4,)), ("mu", np.int32), ("epsilon", np.int32),
    ("initialized", np.int32), ("status", np.int32), ("set_counter", np.int32), ("pad", np.int32, (3,)),
])
assert ECMC_CHAIN_DTYPE.itemsize == 256
ECMC_SET_SIZE = 10001


def ecmc_solve_reject(A, B, gamma, eps) -> float:
    out = C.c_double()
    lib().orc_ecmc_solve_reject(A, B, gamma, int(eps), C.byref(out))
    return out.value


def ecmc_compute_ds(P, R) -> float:
    P = np.ascontiguousarray(P, np.complex128)
    R = np.ascontiguousarray(R, np.complex128)
    out = C.c_double()
    lib().orc_ecmc_compute_ds(_dp(P), _dp(R), C.byref(out))
    return out.value


def ecmc_set(epsilon, seed, call, chain=0, gen=1) -> np.ndarray:
    """The set of near-identity elements of chain `chain`, generation `gen`, call `call`."""
    out = np.zeros((ECMC_SET_SIZE, 3, 3), np.complex128)
    lib().orc_ecmc_set(epsilon, C.c_uint64(seed), chain, C.c_uint64(call), gen, _dp(out))
    return out


def ecmc_chains(dims, l_core) -> np.ndarray:
    """Fresh (uninitialised) chain records, one per l_core^4 block."""
    n = int(np.prod([d // l_core for d in dims]))
    return np.zeros(n, ECMC_CHAIN_DTYPE)


def ecmc_sample(u, dims, params: dict, seed, call, cum, chains):
    """One sample call of every chain on a copy of u; returns (links, chains)."""
    u = np.array(u, np.complex128, copy=True)
    ch = np.array(chains, ECMC_CHAIN_DTYPE, copy=True)
    dp = np.array([params["beta"], params["theta_sample"], params["theta_refresh_site"],
                   params["theta_refresh_R"], params["epsilon_set"]], np.float64)
    ip = (C.c_int * 2)(int(params.get("poisson", 0)), int(params["l_core"]))
    rc = lib().orc_ecmc_sample(_dp(u), _dims(dims), _dp(dp), ip, C.c_uint64(seed), C.c_uint64(call),
                               (C.c_int * 4)(*[int(c) for c in cum]), ch.ctypes.data_as(C.c_void_p))
    if rc:
        raise ValueError("l_core must be >= 3 and divide every extent")
    return u, ch


class EcmcRefRun:
    """generate_ecmc_cb on one rank with the reference's own generator (std::mt19937_64,
    std:: distributions, Householder random_su3, the rank's set regenerated per call and every
    10000 lifts): an L^4 lattice as one block with frozen faces, moved by random_shift before
    each sample_persistant call."""

    def __init__(self, L: int, seed: int, cold_start: bool, params: dict):
        dp = np.array([params["beta"], params["theta_sample"], params["theta_refresh_site"],
                       params["theta_refresh_R"], params["epsilon_set"]], np.float64)
        ip = (C.c_int * 2)(int(params.get("poisson", 0)), int(L))
        self.L = L
        self.h = lib().orc_ecmc_ref_create(L, seed, 1 if cold_start else 0, _dp(dp), ip)

    def run(self, n_shift: int):
        """n_shift shifts; returns (plaquette after each, (events, lifts, same-site lifts))."""
        plaq = np.zeros(n_shift)
        c = (C.c_uint64 * 3)()
        lib().orc_ecmc_ref_run(self.h, n_shift, _dp(plaq), c)
        return plaq, (int(c[0]), int(c[1]), int(c[2]))

    def links(self) -> np.ndarray:
        u = np.zeros(shape((self.L,) * 4), np.complex128)
        lib().orc_ecmc_ref_get_links(self.h, _dp(u))
        return u

    def set_links(self, u) -> None:
        u = np.ascontiguousarray(u, np.complex128)
        lib().orc_ecmc_ref_set_links(self.h, _dp(u))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_ecmc_ref_destroy(self.h)
            self.h = None
