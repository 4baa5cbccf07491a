"""CPU checks of the oracle's event-chain Monte Carlo (restatement of
src/ecmc/ecmc_mpi_cb.cpp): the reject-angle equation, dS, the near-identity set, the block
decomposition (frozen links never move, chains stay in their blocks) and, statistically,
the equilibrium it samples against the heatbath."""
import numpy as np
import pytest

import oracle as orc

LAMBDA3 = np.diag([1.0, -1.0, 0.0])


def _pos_integral(A, B, eps, theta, n=400001):
    """int_0^theta max(0, dS/dt) dt for S(t) = A cos t + eps B sin t (dense trapezoid)."""
    t = np.linspace(0.0, theta, n)
    d = np.maximum(0.0, -A * np.sin(t) + eps * B * np.cos(t))
    return float(np.sum((d[1:] + d[:-1]) * 0.5 * np.diff(t)))


@pytest.mark.parametrize("seed", range(6))
def test_solve_reject_integral(seed):
    """The reject angle is where the accumulated positive part of the staple's dS/dtheta
    reaches gamma (the factorized Metropolis filter), for both senses of rotation."""
    rng = np.random.default_rng(seed)
    for _ in range(20):
        A, B = rng.normal(0, 2.0, 2)
        gamma = rng.exponential(1.0) * (1.0 + 3 * rng.random())
        for eps in (-1, 1):
            th = orc.ecmc_solve_reject(A, B, gamma, eps)
            assert th >= 0.0
            got = _pos_integral(A, B, eps, th)
            assert abs(got - gamma) < 2e-4 * max(1.0, gamma), (A, B, gamma, eps, th, got)


def test_solve_reject_periods():
    """gamma beyond one period (2 R) adds whole turns of 2 pi."""
    A, B = 0.3, -0.7
    R = np.hypot(A, B)
    t1 = orc.ecmc_solve_reject(A, B, 0.25 * R, 1)
    t2 = orc.ecmc_solve_reject(A, B, 0.25 * R + 3 * 2 * R, 1)
    assert abs(t2 - t1 - 3 * 2 * np.pi) < 1e-9


def _su3(rng):
    z = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
    q, r = np.linalg.qr(z)
    q = q * (np.diag(r) / np.abs(np.diag(r)))
    return q / np.linalg.det(q) ** (1 / 3)


def test_compute_ds_definition():
    rng = np.random.default_rng(3)
    for _ in range(10):
        P = rng.normal(size=(3, 3)) + 1j * rng.normal(size=(3, 3))
        R = _su3(rng)
        want = np.trace(LAMBDA3 @ R.conj().T @ P @ R).imag
        assert abs(orc.ecmc_compute_ds(P, R) - want) < 1e-12


def test_set_structure():
    s = orc.ecmc_set(0.15, 7, 3)
    assert s.shape == (orc.ECMC_SET_SIZE, 3, 3)
    assert np.allclose(s[0], np.eye(3))
    assert np.allclose(s[2::2], np.conj(np.transpose(s[1::2], (0, 2, 1))))
    uu = np.einsum("nij,nkj->nik", s, s.conj())
    assert np.abs(uu - np.eye(3)).max() < 1e-13
    assert np.abs(np.linalg.det(s) - 1).max() < 1e-13
    dist = np.linalg.norm((s[1:] - np.eye(3)).reshape(len(s) - 1, -1), axis=1)
    assert 0.1 < dist.mean() < 0.5  # three SU(2) rotations of size 0.15 each
    assert not np.allclose(orc.ecmc_set(0.15, 7, 4)[1], s[1])  # a new set per call
    assert not np.allclose(orc.ecmc_set(0.15, 7, 3, chain=1)[1], s[1])  # one set per chain
    assert not np.allclose(orc.ecmc_set(0.15, 7, 3, gen=2)[1], s[1])  # renewed every 10000 lifts


def test_chain_set_counter_counts_lifts_mod_10000():
    """Each chain keeps its set_counter (lifts since its set was last renewed) across calls, as
    the reference's LocalChainState does (ecmc_mpi_cb.cpp:560-566): after a call it is the lift
    count mod 10000 (the first event of the first call renews the set and zeroes it)."""
    dims = (8, 8, 8, 8)
    u = orc.hot_philox(dims, 5)
    chains = orc.ecmc_chains(dims, 4)
    total = np.zeros(len(chains), np.int64)
    for call in range(3):
        u, chains = orc.ecmc_sample(u, dims, PARAMS, 9, call, (call, 0, 2 * call, 1), chains)
        total = chains["lifts"].astype(np.int64)
        assert np.array_equal(chains["set_counter"], total % 10000)


PARAMS = dict(beta=6.0, theta_sample=20.0, theta_refresh_site=10.0, theta_refresh_R=3.0, epsilon_set=0.15,
              poisson=0, l_core=4)


def _frozen_mask(dims, l, cum):
    """(Lt, Lz, Ly, Lx, 4) mask of the links frozen by the l-block faces after shift cum."""
    lx, ly, lz, lt = dims
    t, z, y, x = np.meshgrid(np.arange(lt), np.arange(lz), np.arange(ly), np.arange(lx), indexing="ij")
    c = [x, y, z, t]
    m = np.zeros((lt, lz, ly, lx, 4), bool)
    for mu in range(4):
        for d in range(4):
            if d != mu:
                m[..., mu] |= (c[d] + cum[d]) % l == 0
    return m


@pytest.mark.parametrize("dims,l,poisson", [((8, 8, 8, 8), 4, 0), ((6, 9, 6, 3), 3, 1), ((10, 5, 5, 10), 5, 0)])
def test_blocks_frozen_links_and_confinement(dims, l, poisson):
    p = dict(PARAMS, l_core=l, poisson=poisson)
    u = orc.hot_philox(dims, 5)
    ch = orc.ecmc_chains(dims, l)
    cum = np.zeros(4, int)
    rng = np.random.default_rng(1)
    for call in range(4):
        cum = (cum + rng.integers(0, l, 4)) % np.array(dims)
        before = u.copy()
        u, ch = orc.ecmc_sample(u, dims, p, 11, call, cum, ch)
        frozen = _frozen_mask(dims, l, cum)
        assert np.array_equal(u[frozen], before[frozen])
        assert not np.array_equal(u[~frozen], before[~frozen])
        assert (ch["initialized"] == 1).all() and (ch["status"] == 0).all()
        assert ((ch["site"] >= 0) & (ch["site"] < l)).all()
        assert ((ch["mu"] >= 0) & (ch["mu"] < 4)).all() and set(np.unique(ch["epsilon"])) <= {-1, 1}
        assert (ch["events"] >= ch["lifts"]).all() and (ch["lifts"] > 0).all()
    U = u.reshape(-1, 3, 3)
    assert np.abs(np.einsum("nij,nkj->nik", U, U.conj()) - np.eye(3)).max() < 1e-12
    assert np.abs(np.linalg.det(U) - 1).max() < 1e-12


def test_sample_is_deterministic():
    """A sample call is a pure function of (links, chain records, seed, call, shift)."""
    dims, l = (8, 8, 8, 8), 4
    u = orc.hot_philox(dims, 9)
    ch = orc.ecmc_chains(dims, l)
    a, ca = orc.ecmc_sample(u, dims, PARAMS, 3, 0, (1, 2, 3, 0), ch)
    b, cb = orc.ecmc_sample(u, dims, PARAMS, 3, 0, (1, 2, 3, 0), ch)
    assert np.array_equal(a, b) and np.array_equal(ca, cb)
    c, _ = orc.ecmc_sample(u, dims, PARAMS, 4, 0, (1, 2, 3, 0), ch)
    assert not np.array_equal(a, c)


def test_resume_is_exact():
    """Two calls = one call, save the chain records, second call from them."""
    dims = (8, 8, 8, 8)
    u = orc.hot_philox(dims, 4)
    ch = orc.ecmc_chains(dims, 4)
    a1, c1 = orc.ecmc_sample(u, dims, PARAMS, 5, 0, (0, 1, 0, 2), ch)
    a2, c2 = orc.ecmc_sample(a1, dims, PARAMS, 5, 1, (3, 1, 2, 2), c1)
    saved = c1.copy()
    b2, d2 = orc.ecmc_sample(a1.copy(), dims, PARAMS, 5, 1, (3, 1, 2, 2), saved)
    assert np.array_equal(a2, b2) and np.array_equal(c2, d2)


def test_equilibrium_matches_heatbath_strong_coupling():
    """At beta = 2 (fast decorrelation) the ECMC plaquette agrees with the heatbath's on the
    same 6^4 lattice.  The ECMC error comes from the scatter of four independent runs (keys and
    translation sequences), which also covers correlations longer than a run's bins."""
    dims, beta = (6, 6, 6, 6), 2.0
    uh = orc.cold(dims)
    hp = []
    for s in range(160):
        uh, _ = orc.heatbath_cb(uh, dims, beta, 1, 1, 17, s)
        if s >= 40:
            hp.append(orc.plaquette(uh, dims))
    p = dict(PARAMS, beta=beta, theta_sample=15.0, l_core=3)
    runs = []
    for k in range(4):
        u, ch = uh.copy(), orc.ecmc_chains(dims, 3)
        rng = np.random.default_rng(8 + k)
        cum = np.zeros(4, int)
        ep = []
        for call in range(150):
            cum = (cum + rng.integers(0, 3, 4)) % 6
            u, ch = orc.ecmc_sample(u, dims, p, 23 + k, call, cum, ch)
            if call >= 20:
                ep.append(orc.plaquette(u, dims))
        runs.append(np.mean(ep))
    e_mean, e_err = np.mean(runs), np.std(runs, ddof=1) / np.sqrt(len(runs))

    def err(x, nb=10):
        x = np.asarray(x)
        n = len(x) // nb
        return x[:n * nb].reshape(nb, n).mean(1).std() / np.sqrt(nb)

    diff = abs(e_mean - np.mean(hp))
    assert diff < 3 * np.hypot(e_err, err(hp)) + 1e-4, (runs, np.mean(hp), e_err, err(hp))


def _binned_err(x, nb=10):
    x = np.asarray(x)
    n = len(x) // nb
    return x[:n * nb].reshape(nb, n).mean(1).std() / np.sqrt(nb)


def test_reference_generator_chain_matches_heatbath():
    """The restatement with the reference's own generator (std::mt19937_64, std::
    distributions, Householder random_su3, per-rank set regenerated per call and every 10000
    lifts) on one rank: 6^4 as one block with frozen faces, moved by random_shift each call.
    From a heatbath-equilibrated start at beta = 2 it keeps the heatbath's mean plaquette;
    links stay unitary."""
    dims, beta = (6, 6, 6, 6), 2.0
    uh = orc.cold(dims)
    hp = []
    for s in range(160):
        uh, _ = orc.heatbath_cb(uh, dims, beta, 1, 1, 29, s)
        if s >= 40:
            hp.append(orc.plaquette(uh, dims))
    run = orc.EcmcRefRun(6, 4321, True, dict(PARAMS, beta=beta, theta_sample=40.0))
    run.set_links(uh)  # from the heatbath's equilibrium
    plaq, (events, lifts, revs) = run.run(500)
    ep = plaq[50:]
    assert events >= lifts > revs > 0
    assert abs(np.mean(ep) - np.mean(hp)) < 4 * np.hypot(_binned_err(ep), _binned_err(hp)) + 1e-4, \
        (np.mean(ep), np.mean(hp))
    U = run.links().reshape(-1, 3, 3)
    assert np.abs(np.einsum("nij,nkj->nik", U, U.conj()) - np.eye(3)).max() < 1e-11


def test_non_finite_angle_stops_the_chain():
    dims = (8, 8, 8, 8)
    u = np.full(orc.shape(dims), np.nan + 0j)
    _, ch = orc.ecmc_sample(u, dims, PARAMS, 3, 0, (0, 0, 0, 0), orc.ecmc_chains(dims, 4))
    assert (ch["status"] & 1).all() and (ch["events"] == 0).all() and (ch["initialized"] == 1).all()
