"""CPU tests of libqcb.so's host side: exported symbols, error paths without a GPU, the
input-file parser and the ILDG container probe (no kernel launches)."""
import ctypes as C
import re
import sys
from pathlib import Path

import pytest

import oracle
import qcb
from qcb import _lib

ROOT = Path(__file__).resolve().parent.parent


def declared_symbols():
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\**\s*(qcb_[a-z_0-9]+)\s*\(", text, flags=re.M))
    return names


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing
    # and the Python binding declares them all
    assert names <= set(_lib.SIGNATURES), sorted(names - set(_lib.SIGNATURES))


def test_abi_version():
    assert _lib.lib().qcb_abi_version() == 1


def test_null_arguments_are_rejected():
    L = _lib.lib()
    assert L.qcb_ctx_create(0, 0, None) == 1
    assert b"null" in L.qcb_last_error()
    assert L.qcb_plaquette(None, None) == 1
    assert L.qcb_heatbath(None, 6.0, 1, 1, 0, 0) == 1
    assert L.qcb_heatbath_plaquette(None, 6.0, 1, 1, 0, 0, None) == 1
    assert L.qcb_ecmc_set_lanes(None, 3) == 1
    assert L.qcb_ecmc_lanes(None, None) == 1
    assert L.qcb_ecmc_sample_n(None, None, 1) == 1
    assert L.qcb_ecmc_num_chains(None, None) == 1


def test_noalloc_plaquette_rejects_misaligned_pointers_before_any_launch():
    L = _lib.lib()
    dims = (C.c_int * 4)(8, 8, 8, 8)
    for prec, nr, ptr in ((0, 18, 24), (1, 12, 40), (1, 18, 20)):
        assert L.qcb_plaquette_noalloc(C.c_void_p(ptr), dims, prec, nr, 2048, C.c_void_p(16), None) == 1
        assert b"aligned" in L.qcb_last_error()
    assert L.qcb_plaquette_noalloc(C.c_void_p(16), dims, 0, 18, 2048, C.c_void_p(4), None) == 1
    assert b"out must be 8-byte aligned" in L.qcb_last_error()


def test_context_creation_without_gpu_fails_cleanly():
    if qcb.device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(qcb.QcbError) as e:
        qcb.Context(0)
    assert e.value.code == 2
    assert "CUDA" in str(e.value) or "device" in str(e.value)


QUIRKY = """# comment
L_core=8
n_core_dims = 1
cold_start=hot
seed = 1234 trailing
N_shift=200
N_switch_eo=1
beta = 6.0
\tN_sweeps\t=\t1
N_hits = 1
N_shift_plaquette = 1
N_shift_therm = 0
topo = true
N_shift_topo = 1
N_steps_gf = 50
N_rk_steps = 1
run_name = cfg1
run_dir = data
save_each_shifts =
no_equals_line
# last one wins
N_hits = 2
"""


def write(tmp_path, text, name="in.txt"):
    p = tmp_path / name
    p.write_bytes(text.encode())
    return p


def test_params_match_reference_semantics(tmp_path):
    p = write(tmp_path, QUIRKY)
    got = qcb.io.load_params(p).as_dict()
    ref = oracle.load_params(p)
    for k, v in ref.items():
        assert got[k] == v, (k, got[k], v)
    assert got["cold_start"] == 0          # "hot" is not "true"
    assert got["N_hits"] == 2              # later keys override
    assert got["save_each_shifts"] == 2    # empty value: default kept
    assert got["N_samples"] == 1           # forced (io.cpp:381)
    assert got["seed"] == 1234             # std::stoi ignores trailing text


def test_params_defaults_and_crlf(tmp_path):
    p = write(tmp_path, "cold_start=true\r\nbeta=5.7\r\n")
    got = qcb.io.load_params(p).as_dict()
    ref = oracle.load_params(p)
    assert got["cold_start"] == ref["cold_start"] == 0   # trailing \r is not trimmed
    assert got["beta"] == ref["beta"] == 5.7
    assert got["N_therm"] == 100 and got["topo"] == 1    # params.h defaults


def test_params_errors(tmp_path):
    with pytest.raises(qcb.QcbError) as e:
        qcb.io.load_params(tmp_path / "missing.txt")
    assert e.value.code == 3
    p = write(tmp_path, "L_core = eight\n")
    with pytest.raises(qcb.QcbError) as e:
        qcb.io.load_params(p)
    assert e.value.code == 4
    with pytest.raises(ValueError):
        oracle.load_params(p)


def test_reference_example_inputs_parse(tmp_path):
    # the reference's inputs/hcold6.txt keys, restated
    text = ("#Lattice params\nL_core=4\nn_core_dims=2\ncold_start=true\n\n#Run params\nseed=12345\n"
            "N_shift_therm = 0\nN_shift=50000\n\n#Heatbath params\nbeta = 6.0\nN_sweeps = 2\nN_hits = 1\n\n"
            "#Plaquette params\nN_shift_plaquette = 1\n\n#Topo params\ntopo = false\nN_shift_topo = 25\n"
            "N_steps_gf = 10\nN_rk_steps = 40\n\n#Save params\nrun_name = hcold62\nrun_dir = data\n"
            "save_each_shifts = 2000\n")
    p = write(tmp_path, text)
    got = qcb.io.load_params(p).as_dict()
    assert got == {**got, **{k: v for k, v in oracle.load_params(p).items()}}
    assert got["topo"] == 0 and got["N_sweeps"] == 2 and got["run_name"] == "hcold62"


def test_ildg_probe(tmp_path):
    dims = (4, 4, 4, 4)
    u = oracle.cold(dims)
    p = tmp_path / "conf"
    oracle.write_ildg(p, u, dims)
    off, n = qcb.io.ildg_probe(p)
    assert n == 256 * 72 * 8
    xml = oracle.ildg_xml(dims)
    assert off == 144 + len(xml) + (8 - len(xml) % 8) % 8 + 144
    # truncated header and bad magic are format errors
    raw = p.read_bytes()
    (tmp_path / "bad").write_bytes(b"\0" * 200)
    with pytest.raises(qcb.QcbError) as e:
        qcb.io.ildg_probe(tmp_path / "bad")
    assert e.value.code == 4
    (tmp_path / "short").write_bytes(raw[:100])
    with pytest.raises(qcb.QcbError) as e:
        qcb.io.ildg_probe(tmp_path / "short")
    assert e.value.code == 4
    with pytest.raises(qcb.QcbError) as e:
        qcb.io.ildg_probe(tmp_path / "nope")
    assert e.value.code == 3


def test_driver_rejects_bad_input(tmp_path):
    """The drop-in driver reports input errors before touching the GPU (io.cpp:454-461)."""
    import subprocess

    driver = ROOT / "ecmc-qncb_b200" / "bin" / "gauge_hb_ncb"
    if not driver.exists():
        subprocess.run([sys.executable, str(ROOT / "ecmc-qncb_b200" / "build.py")], check=True)
    bad = tmp_path / "bad.txt"
    bad.write_text("L_core = eight\n")
    r = subprocess.run([str(driver), str(bad)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Error reading input" in r.stderr
    r = subprocess.run([str(driver), str(tmp_path / "missing.txt")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Can't open file" in r.stderr
    r = subprocess.run([str(driver)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Usage" in r.stderr
    bad.write_text("L_core = 4\nschedule = lexicographic\n")
    r = subprocess.run([str(driver), str(bad)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "schedule must be" in r.stderr


def test_ecmc_params_parse_reference_example(tmp_path):
    """The reference's inputs/ecold6.txt keys (io.cpp:298-341); unset keys keep the
    RunParamsECB / ECMCParams defaults (params.h:9-44)."""
    text = ("#Lattice params\nL_core=4\nn_core_dims=2\ncold_start=true\n\n#Run params\nseed=12345\n"
            "N_shift_therm = 10\nN_shift=20\n\n#ECMC params\nbeta=6.0\nparam_theta_sample=1000\n"
            "param_theta_refresh_site=500\nparam_theta_refresh_R=3.3\npoisson=false\nepsilon_set=0.15\n\n"
            "#Plaquette params\nN_shift_plaquette = 2\n\n#Topo params\ntopo = false\nN_shift_topo = 25\n"
            "N_steps_gf = 10\nN_rk_steps = 40\n\n#Save params\nrun_name = ecold58e\nrun_dir = data\n"
            "save_each_shifts = 2000\n")
    p = tmp_path / "ecold6.txt"
    p.write_text(text)
    got = qcb.io.load_ecmc_params(p).as_dict()
    want = dict(L_core=4, n_core_dims=2, cold_start=1, seed=12345, N_shift=20, beta=6.0, theta_sample=1000.0,
                theta_refresh_site=500.0, theta_refresh_R=3.3, poisson=0, epsilon_set=0.15, l_core=4, N_therm=10,
                topo=0, N_shift_plaquette=2, N_shift_topo=25, N_steps_gf=10, N_rk_steps=40, run_name="ecold58e",
                run_dir="data", save_each_shifts=2000)
    assert got == want
    p.write_text("poisson = true\nL_core = 5\n")
    got = qcb.io.load_ecmc_params(p).as_dict()
    assert got["poisson"] == 1 and got["l_core"] == 5 and got["theta_sample"] == 100.0 and got["N_therm"] == 100
    p.write_text("param_theta_sample = abc\n")
    with pytest.raises(qcb.QcbError) as e:
        qcb.io.load_ecmc_params(p)
    assert e.value.code == 4


def test_ecmc_driver_rejects_bad_input(tmp_path):
    """The event-chain driver reports input errors before touching the GPU."""
    import subprocess

    driver = ROOT / "ecmc-qncb_b200" / "bin" / "gauge_ecmc_ncb"
    if not driver.exists():
        subprocess.run([sys.executable, str(ROOT / "ecmc-qncb_b200" / "build.py")], check=True)
    bad = tmp_path / "bad.txt"
    bad.write_text("param_theta_sample = many\n")
    r = subprocess.run([str(driver), str(bad)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Error reading input" in r.stderr
    bad.write_text("L_core = 2\n")
    r = subprocess.run([str(driver), str(bad)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "L_core must be at least 3" in r.stderr
    r = subprocess.run([str(driver)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "Usage" in r.stderr
