"""CPU checks of the FP64 oracle against known answers and an independent numpy restatement.

The reference ships no tests or golden vectors and cannot be built here, so the oracle is
pinned by: the C++ standard's mt19937_64 value, the Philox4x32-10 known-answer vectors of
Salmon et al., scipy's expm, exact cold-start values, and gauge / translation invariance.
"""
import json
from pathlib import Path

import numpy as np
import pytest
import scipy.linalg as sl

import np_ref

GOLDEN = Path(__file__).resolve().parent / "golden"


def rand_su3_alg(rng):
    a = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
    b = 0.5 * (a - a.conj().T)
    return b - np.trace(b) / 3 * np.eye(3)


def test_mt19937_64_known_value(orc):
    # C++ standard [rand.predef]: the 10000th output of a default-constructed mt19937_64.
    assert orc.mt19937_64_nth(5489, 10000) == 9981545732273789042


def test_philox_known_answers(orc):
    kat = json.loads((GOLDEN / "philox4x32_10_kat.json").read_text())
    for case in kat:
        got = orc.philox(case["ctr"], case["key"])
        assert got == case["out"], case


def test_exp_su3_matches_expm(orc):
    rng = np.random.default_rng(11)
    for coeff in (0.005, 0.02, 0.1, 0.25, 0.5):
        for _ in range(20):
            Z = rand_su3_alg(rng)
            got = orc.exp_su3(Z, coeff)
            ref = sl.expm(coeff * Z)
            assert np.abs(got - ref).max() < 1e-14
            assert abs(np.linalg.det(got) - 1) < 1e-14


def test_proj_lie(orc):
    rng = np.random.default_rng(3)
    A = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
    P = orc.proj_lie(A)
    assert abs(np.trace(P)) < 1e-15
    assert np.abs(P + P.conj().T).max() == 0.0
    assert np.abs(orc.proj_lie(P) - P).max() < 1e-15


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (4, 6, 2, 8)])
def test_cold_start_exact(orc, dims):
    u = orc.cold(dims)
    assert orc.plaquette(u, dims) == 1.0
    assert orc.topo_qe(u, dims) == (0.0, 0.0)


def test_hot_start_is_su3_and_haar_moments(orc):
    dims = (8, 8, 8, 8)
    u = orc.hot_philox(dims, 7).reshape(-1, 3, 3)
    eye = np.einsum("nij,nkj->nik", u, u.conj())
    assert np.abs(eye - np.eye(3)).max() < 1e-14
    assert np.abs(np.linalg.det(u) - 1).max() < 1e-14
    # Haar on SU(3): E[tr U] = 0, E[|U_ij|^2] = 1/3, E[|tr U|^2] = 1
    n = u.shape[0]
    tr = np.trace(u, axis1=1, axis2=2)
    assert abs(tr.mean()) < 5 / np.sqrt(n)
    assert abs((np.abs(u) ** 2).mean() - 1 / 3) < 5 * 0.3 / np.sqrt(9 * n)
    assert abs((np.abs(tr) ** 2).mean() - 1) < 5 * 1.0 / np.sqrt(n)


def test_observables_match_numpy_restatement(orc):
    dims = (4, 4, 4, 4)
    u = orc.hot_philox(dims, 5)
    # heat it a little so the clover fields are not pure noise
    u, _ = orc.heatbath_cb(u, dims, 6.0, 3, 1, 99)
    assert abs(orc.plaquette(u, dims) - np_ref.plaquette(u)) < 1e-13
    q, e = orc.topo_qe(u, dims)
    qn, en = np_ref.topo_qe(u)
    assert abs(q - qn) < 1e-12 and abs(e - en) < 1e-12 * max(1, abs(en))
    for site, mu in ((0, 0), (17, 2), (255, 3)):
        s = orc.staple(u, dims, site, mu)
        t, rest = divmod(site, 64)
        z, rest = divmod(rest, 16)
        y, x = divmod(rest, 4)
        assert np.abs(s - np_ref.staple(u, mu)[t, z, y, x]).max() < 1e-13


def test_rk3_matches_numpy_expm_restatement(orc):
    dims = (4, 4, 4, 4)
    u, _ = orc.heatbath_cb(orc.hot_philox(dims, 21), dims, 6.0, 4, 1, 3)
    got = orc.flow_steps(u, dims, 0.02, 2)
    ref = np_ref.rk3_step(np_ref.rk3_step(u, 0.02), 0.02)
    assert np.abs(got - ref).max() < 1e-13


def test_gauge_and_translation_invariance(orc):
    dims = (4, 4, 6, 4)
    u, _ = orc.heatbath_cb(orc.hot_philox(dims, 8), dims, 5.7, 4, 1, 1)
    p0, (q0, e0) = orc.plaquette(u, dims), orc.topo_qe(u, dims)
    g = orc.gauge_transform_philox(u, dims, 1234)
    assert np.abs(g - u).max() > 0.1
    assert abs(orc.plaquette(g, dims) - p0) < 1e-13
    q1, e1 = orc.topo_qe(g, dims)
    assert abs(q1 - q0) < 1e-12 and abs(e1 - e0) < 1e-12
    for axis, k in ((0, 1), (1, 3), (2, 2), (3, 1)):
        r = np.roll(u, k, axis=axis)
        assert abs(orc.plaquette(r, dims) - p0) < 1e-13
        qr, er = orc.topo_qe(r, dims)
        assert abs(qr - q0) < 1e-12 and abs(er - e0) < 1e-12


def test_flow_measure_semantics(orc):
    dims = (4, 4, 4, 4)
    u, _ = orc.heatbath_cb(orc.hot_philox(dims, 2), dims, 6.0, 5, 1, 0)
    eps, n_gf, n_rk = 0.02, 5, 2
    tqe = orc.flow_measure(u, dims, eps, n_gf, n_rk).reshape(n_gf, 3)
    # records are taken before each group of n_rk steps: t = 0, eps*n_rk, ...
    assert np.allclose(tqe[:, 0], eps * n_rk * np.arange(n_gf), atol=1e-15)
    q0, e0 = orc.topo_qe(u, dims)
    assert tqe[0, 1] == q0 and tqe[0, 2] == e0
    # E decreases monotonically along the flow
    assert np.all(np.diff(tqe[:, 2]) < 0)
    # the flowed record k equals measuring after k*n_rk explicit steps
    w = orc.flow_steps(u, dims, eps, 2 * n_rk)
    q2, e2 = orc.topo_qe(w, dims)
    assert abs(q2 - tqe[2, 1]) < 1e-13 and abs(e2 - tqe[2, 2]) < 1e-13


def test_kp_distribution(orc):
    """KP a0 against the exact density sqrt(1-a^2) exp(alpha a), alpha = 2 beta k / 3."""
    beta, k = 6.0, 1.3
    alpha = 2 * beta * k / 3
    a = orc.kp_samples(beta, k, 200000, 42)
    edges = np.linspace(-1, 1, 41)
    hist, _ = np.histogram(a, edges)
    xs = np.linspace(-1, 1, 200001)
    dens = np.sqrt(np.clip(1 - xs ** 2, 0, None)) * np.exp(alpha * (xs - 1))
    cdf = np.concatenate([[0], np.cumsum((dens[1:] + dens[:-1]) / 2 * np.diff(xs))])
    cdf /= cdf[-1]
    p = np.diff(np.interp(edges, xs, cdf))
    exp = p * a.size
    m = exp > 5
    chi2 = (((hist - exp) ** 2)[m] / exp[m]).sum()
    dof = m.sum() - 1
    assert chi2 < dof + 5 * np.sqrt(2 * dof), (chi2, dof)


def test_reference_schedule_frozen_count(orc):
    # one reference sweep updates 4 L (L-1)^3 links (GeometryCB.cpp:33-56)
    chain = orc.RefChain(4, 12345, True)
    before = chain.links()
    chain.sweeps(6.0, 1)
    after = chain.links()
    changed = (np.abs(after - before).reshape(-1, 4, 9).max(axis=2) > 0).sum()
    assert changed == 4 * 4 * 3 ** 3


def test_ildg_codec_roundtrip(orc, tmp_path):
    dims = (4, 4, 4, 6)
    u = orc.hot_philox(dims, 3)
    p = tmp_path / "conf"
    orc.write_ildg(p, u, dims)
    raw = p.read_bytes()
    assert raw[16:27] == b"ildg-format"
    assert len(raw) % 8 == 0
    assert np.array_equal(orc.read_ildg(p, dims), u)
    with pytest.raises(ValueError):
        orc.read_ildg(p, (4, 4, 4, 4))


def test_checkerboard_schedule_matches_reference_schedule_statistically(orc):
    """The library's schedule (checkerboard passes, Philox) restated in the oracle samples
    the same mean plaquette as the reference's (frozen links + random shifts, mt19937_64)
    on a 4^4 lattice at beta = 6.0."""
    from stats import binned_mean_err, z_score

    dims = (4, 4, 4, 4)
    u = orc.hot_philox(dims, 17)
    cb = []
    for s in range(2400):
        u, fails = orc.heatbath_cb(u, dims, 6.0, 1, 1, 99, s)
        cb.append(orc.plaquette(u, dims))
    ref = orc.RefChain(4, 4242, False).run(6.0, 2400)
    z = z_score(cb[200:], ref[200:])
    print("cb", binned_mean_err(cb[200:]), "ref", binned_mean_err(ref[200:]), "z", z)
    assert z < 3.0
