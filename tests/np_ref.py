"""Vectorised numpy restatement of staple / plaquette / clover / RK3 flow (scipy expm).

A second, independent restatement used only to cross-check the C++ oracle on tiny
lattices.  Links: complex array (Lt, Lz, Ly, Lx, 4, 3, 3); direction mu = 0..3 is x, y, z, t,
so the array axis of direction mu is 3 - mu.
"""
import numpy as np
import scipy.linalg as sl


def _ax(mu):
    return 3 - mu


def shift(a, mu, d):
    """a(x + d*mu) for a site field a[t, z, y, x, ...]."""
    return np.roll(a, -d, axis=_ax(mu))


def dag(a):
    return np.conj(np.swapaxes(a, -1, -2))


def mm(a, b):
    return np.einsum("...ij,...jk->...ik", a, b)


def staple(U, mu):
    A = np.zeros(U.shape[:4] + (3, 3), complex)
    for nu in range(4):
        if nu == mu:
            continue
        Unu, Umu = U[..., nu, :, :], U[..., mu, :, :]
        A += mm(mm(shift(Unu, mu, 1), dag(shift(Umu, nu, 1))), dag(Unu))
        Unu_m = shift(Unu, nu, -1)
        A += mm(mm(dag(shift(Unu_m, mu, 1)), dag(shift(Umu, nu, -1))), Unu_m)
    return A


def plaquette(U):
    s = 0.0
    V = np.prod(U.shape[:4])
    for mu in range(4):
        for nu in range(mu + 1, 4):
            Umu, Unu = U[..., mu, :, :], U[..., nu, :, :]
            P = mm(mm(mm(Umu, shift(Unu, mu, 1)), dag(shift(Umu, nu, 1))), dag(Unu))
            s += np.trace(P, axis1=-2, axis2=-1).real.sum() / 3.0
    return s / (6.0 * V)


def clover_F(U, mu, nu):
    Umu, Unu = U[..., mu, :, :], U[..., nu, :, :]
    s = lambda a, m, d: shift(a, m, d)  # noqa: E731
    C = mm(mm(mm(Umu, s(Unu, mu, 1)), dag(s(Umu, nu, 1))), dag(Unu))
    C += mm(mm(mm(Unu, dag(s(s(Umu, mu, -1), nu, 1))), dag(s(Unu, mu, -1))), s(Umu, mu, -1))
    C += mm(mm(mm(dag(s(Umu, mu, -1)), dag(s(s(Unu, mu, -1), nu, -1))), s(s(Umu, mu, -1), nu, -1)), s(Unu, nu, -1))
    C += mm(mm(mm(dag(s(Unu, nu, -1)), s(Umu, nu, -1)), s(s(Unu, mu, 1), nu, -1)), dag(Umu))
    return 0.125 * (C - dag(C))


def topo_qe(U):
    F = {(m, n): clover_F(U, m, n) for m in range(4) for n in range(m + 1, 4)}
    tr = lambda a, b: np.trace(mm(a, b), axis1=-2, axis2=-1).real  # noqa: E731
    q = tr(F[0, 1], F[2, 3]) - tr(F[0, 2], F[1, 3]) + tr(F[0, 3], F[1, 2])
    e = 0.5 * sum((np.abs(f) ** 2).sum(axis=(-1, -2)) for f in F.values())
    V = np.prod(U.shape[:4])
    return q.sum() / (4 * np.pi ** 2), e.sum() / V


def proj_ta(M):
    B = 0.5 * (M - dag(M))
    tr = np.trace(B, axis1=-2, axis2=-1) / 3.0
    return B - tr[..., None, None] * np.eye(3)


def force(U):
    Z = np.zeros_like(U)
    for mu in range(4):
        Z[..., mu, :, :] = proj_ta(-mm(U[..., mu, :, :], staple(U, mu)))
    return Z


def expm_batch(X):
    flat = X.reshape(-1, 3, 3)
    return np.stack([sl.expm(x) for x in flat]).reshape(X.shape)


def rk3_step(U, eps):
    Z0 = force(U)
    W1 = mm(expm_batch(0.25 * eps * Z0), U)
    Z1 = force(W1)
    W2 = mm(expm_batch(8.0 / 9.0 * eps * Z1 - 17.0 / 36.0 * eps * Z0), W1)
    Z2 = force(W2)
    W3 = mm(expm_batch(0.75 * eps * Z2 - 8.0 / 9.0 * eps * Z1 + 17.0 / 36.0 * eps * Z0), W2)
    return W3
