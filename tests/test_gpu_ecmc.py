"""Event-chain Monte Carlo on the GPU (qcb_ecmc_*) against the oracle's restatement of
mpi::ecmccb::sample_persistant (src/ecmc/ecmc_mpi_cb.cpp:496-637).

Both draw every random number from the same Philox counters, so the GPU chains take the
oracle's events one for one: counters, positions and draw counts agree exactly, links and
chain matrices to rounding.  Plus: frozen links stay bit-identical, FP32 storage, resume
from saved records, argument checks, and the equilibrium plaquette against the heatbath.
"""
import numpy as np
import pytest

import oracle as orc
import qcb
from qcb.ecmc import CHAIN_DTYPE

pytestmark = pytest.mark.gpu

# Budgets with no common multiple near theta_sample: with commensurate budgets (the
# reference's defaults 100 / 50, for instance) the sample and site-refresh budgets run out on
# the same event and the last rounding of the summed angles decides which fires first, which
# transcendental functions of different libraries resolve differently.
BASE = dict(beta=6.0, theta_sample=20.0, theta_refresh_site=7.3, theta_refresh_R=3.1, epsilon_set=0.15,
            poisson=0, l_core=4)
EXACT = ["draws", "events", "lifts", "revs", "site", "mu", "epsilon", "initialized", "status", "set_counter"]


def _compare(rec, ref, tol=1e-9):
    for k in EXACT:
        assert np.array_equal(rec[k], ref[k]), k
    for k in ("R", "theta_refresh_site", "theta_refresh_R", "travelled_site", "travelled_R"):
        assert np.abs(rec[k] - ref[k]).max() < tol, k


def test_set_renewal_after_10000_lifts_matches_oracle(ctx):
    """A chain's near-identity set is renewed at the top of the event loop whenever its
    set_counter is a multiple of 10000 (ecmc_mpi_cb.cpp:560-566), besides the renewal at every
    call.  Chains restarted with set_counter 9998 renew their set after two lifts inside the
    call: the GPU takes the oracle's events and ends with the oracle's set_counter."""
    dims, l = (8, 8, 8, 8), 4
    p = dict(BASE, l_core=l)
    u = orc.hot_philox(dims, 31)
    f = qcb.GaugeField(ctx, dims)
    f.set_links(u)
    ch = qcb.EventChains(f, p, 41)
    ch.sample((1, 2, 0, 3))
    ref_u, ref_c = orc.ecmc_sample(u, dims, p, 41, 0, (1, 2, 0, 3), orc.ecmc_chains(dims, l))
    rec, calls = ch.chains()
    _compare(rec, ref_c)
    rec["set_counter"] = 9998
    ref_c["set_counter"] = 9998
    ch.set_chains(rec, calls)
    ch.sample((3, 1, 2, 0))
    ref_u, ref_c = orc.ecmc_sample(ref_u, dims, p, 41, 1, (3, 1, 2, 0), ref_c)
    rec, _ = ch.chains()
    _compare(rec, ref_c)
    assert np.abs(f.get_links() - ref_u).max() < 1e-9
    assert (rec["set_counter"] < 9998).all()  # every chain lifted at least twice and renewed
    ch.close()
    f.close()


@pytest.mark.parametrize("dims,l,poisson,beta,eps_set", [((8, 8, 8, 8), 4, 0, 6.0, 0.15),
                                                        ((6, 6, 12, 6), 3, 1, 5.7, 0.15),
                                                        ((8, 8, 8, 16), 4, 0, 2.0, 0.15),
                                                        ((10, 10, 10, 10), 5, 0, 6.2, 0.3),
                                                        ((8, 8, 8, 8), 4, 1, 6.0, 0.0)])
def test_matches_oracle_event_for_event(ctx, dims, l, poisson, beta, eps_set):
    p = dict(BASE, l_core=l, poisson=poisson, beta=beta, epsilon_set=eps_set)
    u = orc.hot_philox(dims, 21)
    f = qcb.GaugeField(ctx, dims)
    f.set_links(u)
    ch = qcb.EventChains(f, p, 77)
    ref_u, ref_c = u, orc.ecmc_chains(dims, l)
    rng = np.random.default_rng(4)
    cum = np.zeros(4, int)
    for call in range(4):
        cum = (cum + rng.integers(0, l, 4)) % np.array(dims)
        ch.sample(cum)
        ref_u, ref_c = orc.ecmc_sample(ref_u, dims, p, 77, call, cum, ref_c)
        rec, calls = ch.chains()
        assert calls == call + 1
        _compare(rec, ref_c)
        assert np.abs(f.get_links() - ref_u).max() < 1e-9
    ev, lifts, revs = ch.counters()
    assert (ev, lifts, revs) == (int(ref_c["events"].sum()), int(ref_c["lifts"].sum()), int(ref_c["revs"].sum()))
    ch.close()
    f.close()


def test_commensurate_budgets_differ_only_at_the_tie(ctx):
    """theta_sample = 2 theta_refresh_site: at the end of a call the two budgets tie; a chain
    of the GPU and of the oracle may resolve it differently, by one site refresh (its six
    gammas and six site draws), and otherwise take the same events."""
    dims = (8, 8, 8, 8)
    p = dict(BASE, theta_refresh_site=10.0)
    u = orc.hot_philox(dims, 21)
    f = qcb.GaugeField(ctx, dims)
    f.set_links(u)
    ch = qcb.EventChains(f, p, 77)
    ch.sample((1, 2, 3, 0))
    rec, _ = ch.chains()
    _, ref = orc.ecmc_sample(u, dims, p, 77, 0, (1, 2, 3, 0), orc.ecmc_chains(dims, 4))
    d = rec["draws"].astype(np.int64) - ref["draws"].astype(np.int64)
    assert set(np.unique(d)) <= {-12, 0, 12}
    assert np.array_equal(rec["lifts"], ref["lifts"])
    ch.close()
    f.close()


def test_frozen_links_bit_identical(ctx):
    dims, l, cum = (8, 8, 8, 8), 4, (3, 1, 0, 2)
    u = orc.hot_philox(dims, 2)
    f = qcb.GaugeField(ctx, dims)
    f.set_links(u)
    ch = qcb.EventChains(f, BASE, 5)
    ch.sample(cum)
    got = f.get_links()
    lx, ly, lz, lt = dims
    t, z, y, x = np.meshgrid(np.arange(lt), np.arange(lz), np.arange(ly), np.arange(lx), indexing="ij")
    c = [x, y, z, t]
    for mu in range(4):
        frozen = np.zeros((lt, lz, ly, lx), bool)
        for d in range(4):
            if d != mu:
                frozen |= (c[d] + cum[d]) % l == 0
        assert np.array_equal(got[frozen, mu], u[frozen, mu])
        assert not np.array_equal(got[~frozen, mu], u[~frozen, mu])
    ch.close()
    f.close()


@pytest.mark.parametrize("precision,storage,tol", [("fp32", 12, 1e-5), ("fp64", 12, 1e-9), ("fp32", 18, 1e-5)])
def test_other_storages_track_the_oracle(ctx, precision, storage, tol):
    """The chains compute in FP64 on the unpacked links whatever the storage: the same events
    as the oracle from the stored (rounded or 12-real) start, links to the storage's rounding."""
    dims = (8, 8, 8, 8)
    u = orc.hot_philox(dims, 8)
    f = qcb.GaugeField(ctx, dims, precision, storage)
    f.set_links(u)
    start = f.get_links()
    ch = qcb.EventChains(f, BASE, 9)
    ch.sample((1, 1, 1, 1))
    ref_u, ref_c = orc.ecmc_sample(start, dims, BASE, 9, 0, (1, 1, 1, 1), orc.ecmc_chains(dims, 4))
    rec, _ = ch.chains()
    assert np.array_equal(rec["events"], ref_c["events"])
    assert np.array_equal(rec["draws"], ref_c["draws"])
    assert np.abs(f.get_links() - ref_u).max() < tol
    for o in (ch, f):
        o.close()


def test_resume_from_saved_records(ctx):
    dims = (8, 8, 8, 8)
    u = orc.hot_philox(dims, 6)
    f = qcb.GaugeField(ctx, dims)
    f.set_links(u)
    a = qcb.EventChains(f, BASE, 31)
    a.sample((0, 1, 2, 3))
    rec, calls = a.chains()
    mid = f.get_links()
    a.sample((2, 2, 2, 2))
    want = f.get_links()
    f.set_links(mid)
    b = qcb.EventChains(f, BASE, 31)
    b.set_chains(rec, calls)
    b.sample((2, 2, 2, 2))
    assert np.array_equal(f.get_links(), want)
    assert np.array_equal(b.chains()[0], a.chains()[0])
    for o in (a, b, f):
        o.close()


def test_counters_reset(ctx):
    dims = (8, 8, 8, 8)
    f = qcb.GaugeField(ctx, dims)
    f.hot_start(3)
    ch = qcb.EventChains(f, BASE, 1)
    ch.sample()
    ev, lifts, revs = ch.counters(reset=True)
    assert ev >= lifts > revs > 0
    assert ch.counters() == (0, 0, 0)
    ch.sample((1, 0, 0, 0))
    assert ch.counters()[0] > 0
    ch.close()
    f.close()


def test_argument_checks(ctx):
    f = qcb.GaugeField(ctx, (8, 8, 8, 8))
    for bad in (dict(BASE, l_core=2), dict(BASE, l_core=3), dict(BASE, beta=0.0), dict(BASE, theta_sample=-1.0),
                dict(BASE, epsilon_set=1.5)):
        with pytest.raises(qcb.QcbError) as e:
            qcb.EventChains(f, bad, 1)
        assert e.value.code == 1
    ch = qcb.EventChains(f, BASE, 1)
    rec = np.zeros(ch.n_chains, CHAIN_DTYPE)
    rec["initialized"] = 1
    rec["epsilon"] = 1
    for field, value in (("mu", 4), ("mu", -1), ("epsilon", 0), ("epsilon", 2)):
        bad = rec.copy()
        bad[field] = value
        with pytest.raises(qcb.QcbError) as e:
            ch.set_chains(bad, 0)
        assert e.value.code == 1
    ch.close()
    f.close()


def test_equilibrium_matches_heatbath(ctx):
    """From a heatbath-equilibrated 8^4 field at beta = 6.0, the ECMC keeps the heatbath's
    mean plaquette (within the combined statistical error)."""
    dims, beta = (8, 8, 8, 8), 6.0
    f = qcb.GaugeField(ctx, dims)
    f.cold_start()
    hp = []
    for s in range(1200):
        qcb._lib.check(qcb._lib.lib().qcb_heatbath(f.h, beta, 1, 1, 13, s))
        if s >= 200:
            hp.append(qcb.observables.mean_plaquette_global(f))
    ch = qcb.EventChains(f, dict(BASE, theta_sample=100.0, theta_refresh_site=50.0, theta_refresh_R=15.0), 19)
    # the reference's default budgets (src/io/params.h:12-14)
    rng = np.random.default_rng(5)
    cum = np.zeros(4, int)
    ep = []
    for call in range(3000):
        cum = (cum + rng.integers(0, 4, 4)) % 8
        ch.sample(cum)
        if call >= 500:
            ep.append(qcb.observables.mean_plaquette_global(f))

    def err(x, nb=20):
        x = np.asarray(x)
        n = len(x) // nb
        return x[:n * nb].reshape(nb, n).mean(1).std() / np.sqrt(nb)

    assert abs(np.mean(ep) - np.mean(hp)) < 4 * np.hypot(err(ep), err(hp)), (np.mean(ep), np.mean(hp))
    ch.close()
    f.close()


def test_gpu_chains_sample_as_the_reference_generator(ctx):
    """The GPU chain (Philox, the library's shared set) and the restatement with the
    reference's own generator (std::mt19937_64) on the same setup, one rank's 6^4 block with
    frozen faces at beta = 2, from the same heatbath-equilibrated start, keep the same mean
    plaquette."""
    dims, beta = (6, 6, 6, 6), 2.0
    p = dict(BASE, beta=beta, theta_sample=40.0, l_core=6)
    start, _ = orc.heatbath_cb(orc.cold(dims), dims, beta, 60, 1, 31, 0)  # equilibrated start
    ref = orc.EcmcRefRun(6, 4321, True, p)
    ref.set_links(start)
    rplaq, _ = ref.run(600)
    f = qcb.GaugeField(ctx, dims)
    f.set_links(start)
    ch = qcb.EventChains(f, p, 17)
    rng = np.random.default_rng(3)
    cum = np.zeros(4, int)
    gp = []
    for call in range(600):
        cum = (cum + rng.integers(0, 6, 4)) % 6
        ch.sample(cum)
        gp.append(qcb.observables.mean_plaquette_global(f))
    a, b = np.asarray(gp[100:]), rplaq[100:]

    def err(x, nb=10):
        n = len(x) // nb
        return x[:n * nb].reshape(nb, n).mean(1).std() / np.sqrt(nb)

    assert abs(a.mean() - b.mean()) < 4 * np.hypot(err(a), err(b)) + 1e-4, (a.mean(), b.mean())
    ch.close()
    f.close()


def test_non_finite_angle_stops_the_chain_and_is_reported(ctx):
    """Links with NaN give a non-finite event angle: every chain stops at its first event,
    records status bit 0, and qcb_ecmc_counters reports QCB_ERR_STATE once; with valid links
    the same object samples again."""
    dims = (8, 8, 8, 8)
    f = qcb.GaugeField(ctx, dims)
    f.set_links(np.full(orc.shape(dims), np.nan + 0j))
    ch = qcb.EventChains(f, BASE, 3)
    ch.sample((0, 0, 0, 0))
    with pytest.raises(qcb.QcbError) as e:
        ch.counters(reset=True)
    assert e.value.code == 7 and "non-finite" in str(e.value)
    rec, _ = ch.chains()
    assert (rec["status"] & 1).all() and (rec["events"] == 0).all()
    u = orc.hot_philox(dims, 4)
    f.set_links(u)
    ch.set_chains(rec, 1)
    ch.sample((1, 0, 0, 0))
    assert ch.counters()[0] > 0
    assert (ch.chains()[0]["status"] == 0).all()
    ref_u, _ = orc.ecmc_sample(u, dims, BASE, 3, 1, (1, 0, 0, 0), rec)
    assert np.abs(f.get_links() - ref_u).max() < 1e-9
    ch.close()
    f.close()


def test_sample_n_equals_single_calls(ctx):
    """qcb_ecmc_sample_n (one pack and unpack for several calls) = the same calls one by one."""
    dims = (8, 8, 8, 8)
    u = orc.hot_philox(dims, 12)
    shifts = np.array([[1, 0, 2, 3], [2, 3, 2, 0], [3, 1, 1, 1]])
    fa = qcb.GaugeField(ctx, dims)
    fa.set_links(u)
    a = qcb.EventChains(fa, BASE, 41)
    for s in shifts:
        a.sample(s)
    fb = qcb.GaugeField(ctx, dims)
    fb.set_links(u)
    b = qcb.EventChains(fb, BASE, 41)
    b.sample_n(shifts)
    ra, ca = a.chains()
    rb, cb = b.chains()
    assert ca == cb == 3
    assert np.array_equal(ra, rb)
    assert np.array_equal(fa.get_links(), fb.get_links())
    for o in (a, b, fa, fb):
        o.close()


@pytest.mark.parametrize("dims,l,poisson,eps_set", [((8, 8, 8, 8), 4, False, 0.15), ((12, 12, 12, 12), 3, False, 0.15),
                                                     ((8, 8, 8, 8), 4, True, 0.15), ((10, 10, 10, 10), 5, True, 0.3)])
def test_lanes_per_chain_give_identical_results(ctx, dims, l, poisson, eps_set):
    """One, three or six lanes per chain (qcb_ecmc_set_lanes) and the automatic choice run
    the same operations per chain: links and chain records agree bit for bit."""
    u = orc.hot_philox(dims, 5)
    shifts = np.array([[1, 0, 2, 1], [2, 1, 0, 0], [0, 2, 1, 1]]) % l
    out = {}
    for lanes in (0, 1, 3, 6):
        f = qcb.GaugeField(ctx, dims)
        f.set_links(u)
        ch = qcb.EventChains(f, qcb.ecmc.params(theta_sample=20.0, theta_refresh_site=7.3, theta_refresh_R=3.1,
                                                poisson=poisson, epsilon_set=eps_set, l_core=l), 77)
        ch.lanes = lanes
        assert ch.lanes == (lanes or ch.lanes) and ch.lanes in (1, 3, 6)
        for s in shifts:
            ch.sample(s)
        rec, _ = ch.chains()
        assert ch.counters()[0] > 0
        out[lanes] = (f.get_links(), rec)
        ch.close()
        f.close()
    for lanes in (1, 3, 6):
        assert np.array_equal(out[lanes][0], out[0][0]), lanes
        assert np.array_equal(out[lanes][1], out[0][1]), lanes


def test_lanes_argument_checked(ctx):
    f = qcb.GaugeField(ctx, (8, 8, 8, 8))
    ch = qcb.EventChains(f, BASE, 1)
    for bad in (-1, 2, 4, 32):
        with pytest.raises(qcb.QcbError):
            ch.lanes = bad
    ch.close()
    f.close()


def test_automatic_lanes_follow_the_chain_count(ctx):
    """Few chains run on six lanes each; past what the device holds at once, on three."""
    for dims, l, lanes in (((8, 8, 8, 8), 4, 6), ((30, 30, 30, 30), 3, 3)):
        f = qcb.GaugeField(ctx, dims, "fp32", 12)
        ch = qcb.EventChains(f, BASE | {"l_core": l}, 1)
        assert ch.lanes == lanes, (ch.n_chains, ch.lanes)
        ch.lanes = 1
        assert ch.lanes == 1
        ch.lanes = 0
        assert ch.lanes == lanes
        ch.close()
        f.close()
