"""Deterministic input recipes and dense restatements of the reference's
in-test oracles (LatticeMatrices.jl test/*.jl).

These are the reference tests' own known-answer constructions, restated in
numpy so that the C oracle (oracle/lmb_oracle.c) can be pinned against them.
They are written for clarity (dense gamma matrices, explicit path products),
independently of the oracle's projector/half-spin formulation.  Arrays use the
reference's index order (NC1, NC2, X, Y, Z, T), Fortran-ordered, and 1-based
lattice coordinates in the recipes exactly as the Julia tests use them.
"""
from __future__ import annotations

import itertools

import numpy as np

GAMMA = [
    np.array([[0, 0, 0, -1j], [0, 0, -1j, 0], [0, 1j, 0, 0], [1j, 0, 0, 0]]),
    np.array([[0, 0, 0, -1], [0, 0, 1, 0], [0, 1, 0, 0], [-1, 0, 0, 0]],
             dtype=complex),
    np.array([[0, 0, -1j, 0], [0, 0, 0, 1j], [1j, 0, 0, 0], [0, -1j, 0, 0]]),
    np.array([[0, 0, -1, 0], [0, 0, 0, -1], [-1, 0, 0, 0], [0, -1, 0, 0]],
             dtype=complex),
]  # Operators.jl:44-66
GAMMA5 = GAMMA[0] @ GAMMA[1] @ GAMMA[2] @ GAMMA[3]
PLANES = ((0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3))


def zeros(nc1, nc2, L, dtype=np.complex128):
    return np.zeros((nc1, nc2) + tuple(L), dtype=dtype, order="F")


def sites(L):
    """1-based coordinate tuples in column-major (x fastest) order."""
    for t, z, y, x in itertools.product(*[range(1, n + 1) for n in L[::-1]]):
        yield (x, y, z, t)


def idx(x):
    return tuple(v - 1 for v in x)


def shift(x, direction, amount, L):
    # test/staggered_dirac.jl:1-4
    return tuple(((x[d] + amount - 1) % L[d]) + 1 if d == direction else x[d]
                 for d in range(4))


def fermion_shift(x, direction, amount, L, phases):
    # test/staggered_dirac.jl:6-11 (phase^wraps with floor division)
    shifted = shift(x, direction, amount, L)
    wraps = (x[direction] + amount - 1) // L[direction]
    return shifted, complex(phases[direction]) ** wraps


def eta(x, direction):
    # test/staggered_dirac.jl:13-17 (zero-based sum of preceding coordinates)
    if direction == 0:
        return 1
    return 1 if sum(x[nu] - 1 for nu in range(direction)) % 2 == 0 else -1


# ---------------------------------------------------------------------------
# input recipes
# ---------------------------------------------------------------------------
def staggered_test_links(L, NC=3, dtype=np.complex128):
    # test/staggered_dirac.jl:19-35
    links = [zeros(NC, NC, L, dtype) for _ in range(4)]
    rt = np.float32 if dtype == np.complex64 else np.float64
    for x in sites(L):
        coordinate = x[0] + 3 * x[1] + 5 * x[2] + 7 * x[3]
        for mu in range(1, 5):
            for col in range(1, NC + 1):
                for row in range(1, NC + 1):
                    re = rt(0.013 * (2 * row - col + coordinate + 3 * mu))
                    im = rt(0.017 * (row + 2 * col - coordinate + mu))
                    links[mu - 1][(row - 1, col - 1) + idx(x)] = re + 1j * im
    return links


def staggered_test_fermion(L, NC=3, offset=0.0, dtype=np.complex128):
    # test/staggered_dirac.jl:37-51
    psi = zeros(NC, 1, L, dtype)
    rt = np.float32 if dtype == np.complex64 else np.float64
    for x in sites(L):
        coordinate = x[0] + 2 * x[1] + 4 * x[2] + 8 * x[3]
        for color in range(1, NC + 1):
            re = rt(offset + 0.019 * (color + coordinate))
            im = rt(0.023 * (2 * color - coordinate))
            psi[(color - 1, 0) + idx(x)] = re + 1j * im
    return psi


def clover_test_su2(angle, phase):
    # test/wilson_clover.jl:12-17
    c, s, z = np.cos(angle), np.sin(angle), np.exp(1j * phase)
    return np.array([[c, s * z], [-s * np.conj(z), c]])


def clover_test_links(L):
    # test/wilson_clover.jl:19-31
    links = [zeros(2, 2, L) for _ in range(4)]
    for x in sites(L):
        coordinate = x[0] + 2 * x[1] + 3 * x[2] + 5 * x[3]
        for mu in range(1, 5):
            links[mu - 1][(slice(None), slice(None)) + idx(x)] = \
                clover_test_su2(0.071 * (coordinate + 2 * mu),
                                0.113 * (2 * coordinate - mu))
    return links


def clover_test_spinor(L, offset=0.0, NC=2):
    # test/wilson_clover.jl:33-45
    psi = zeros(NC, 4, L)
    for x in sites(L):
        coordinate = x[0] + 2 * x[1] + 3 * x[2] + 5 * x[3]
        for spin in range(1, 5):
            for color in range(1, NC + 1):
                psi[(color - 1, spin - 1) + idx(x)] = (
                    offset + 0.031 * (color + 2 * spin + coordinate) +
                    1j * 0.047 * (2 * color - spin + coordinate))
    return psi


def hisq_test_links(L, NC=3):
    # test/hisq_dirac.jl:1-25
    fat = [zeros(NC, NC, L) for _ in range(4)]
    lng = [zeros(NC, NC, L) for _ in range(4)]
    for x in sites(L):
        coordinate = x[0] + 3 * x[1] + 5 * x[2] + 7 * x[3]
        for mu in range(1, 5):
            for col in range(1, NC + 1):
                for row in range(1, NC + 1):
                    fat[mu - 1][(row - 1, col - 1) + idx(x)] = (
                        0.011 * (2 * row - col + coordinate + 3 * mu) +
                        1j * 0.014 * (row + 2 * col - coordinate + mu))
                    lng[mu - 1][(row - 1, col - 1) + idx(x)] = (
                        0.007 * (row - 3 * col + 2 * coordinate + mu) +
                        1j * 0.009 * (2 * row + col - coordinate - 2 * mu))
    return fat, lng


def unit_links(L, NC, scale=1.0):
    U = zeros(NC, NC, L)
    for c in range(NC):
        U[c, c] = scale
    return U


def near_identity_links(L):
    # test/hisq_full_smearing.jl:58-65 (0.05 * recipe + identity)
    U = staggered_test_links(L, 3)
    for u in U:
        u *= 0.05
        for c in range(3):
            u[c, c] += 1.0
    return U


# ---------------------------------------------------------------------------
# dense oracles
# ---------------------------------------------------------------------------
def mat(U, x):
    return U[(slice(None), slice(None)) + idx(x)]


def clover_field_strength_dense(links):
    # test/wilson_clover.jl:47-80
    L = links[0].shape[2:]
    NC = links[0].shape[0]
    fields = [zeros(NC, NC, L) for _ in range(6)]
    for plane, (mu, nu) in enumerate(PLANES):
        Um, Un = links[mu], links[nu]
        for x in sites(L):
            xpmu = shift(x, mu, 1, L)
            xpnu = shift(x, nu, 1, L)
            xmmu = shift(x, mu, -1, L)
            xmnu = shift(x, nu, -1, L)
            xpnu_mmu = shift(xpnu, mu, -1, L)
            xmmu_mnu = shift(xmmu, nu, -1, L)
            xpmu_mnu = shift(xmnu, mu, 1, L)
            d = lambda a: a.conj().T
            Q = (mat(Um, x) @ mat(Un, xpmu) @ d(mat(Um, xpnu)) @ d(mat(Un, x)) +
                 mat(Un, x) @ d(mat(Um, xpnu_mmu)) @ d(mat(Un, xmmu)) @ mat(Um, xmmu) +
                 d(mat(Um, xmmu)) @ d(mat(Un, xmmu_mnu)) @ mat(Um, xmmu_mnu) @ mat(Un, xmnu) +
                 d(mat(Un, xmnu)) @ mat(Um, xmnu) @ mat(Un, xpmu_mnu) @ d(mat(Um, x)))
            fields[plane][(slice(None), slice(None)) + idx(x)] = 0.125 * (Q - Q.conj().T)
    return fields


def wilson_clover_dense(links, psi, kappa, csw, phases, dagger=False):
    """test/wilson_clover.jl:82-112; dagger via gamma5 D gamma5."""
    if dagger:
        return apply_gamma5(wilson_clover_dense(links, apply_gamma5(psi),
                                                kappa, csw, phases))
    L = psi.shape[2:]
    fields = clover_field_strength_dense(links)
    result = np.empty_like(psi)
    gp = [GAMMA[mu] @ GAMMA[nu] for mu, nu in PLANES]
    eye = np.eye(4)
    for x in sites(L):
        value = psi[(slice(None), slice(None)) + idx(x)].copy()
        for mu in range(4):
            xp, php = fermion_shift(x, mu, 1, L, phases)
            xm, phm = fermion_shift(x, mu, -1, L, phases)
            value -= kappa * mat(links[mu], x) @ (
                php * psi[(slice(None), slice(None)) + idx(xp)]) @ (eye - GAMMA[mu]).T
            value -= kappa * mat(links[mu], xm).conj().T @ (
                phm * psi[(slice(None), slice(None)) + idx(xm)]) @ (eye + GAMMA[mu]).T
        for plane in range(6):
            value -= kappa * csw * mat(fields[plane], x) @ \
                psi[(slice(None), slice(None)) + idx(x)] @ gp[plane].T
        result[(slice(None), slice(None)) + idx(x)] = value
    return result


def apply_gamma5(psi):
    # test/wilson_clover.jl:114-123
    out = np.empty_like(psi)
    for x in sites(psi.shape[2:]):
        out[(slice(None), slice(None)) + idx(x)] = \
            psi[(slice(None), slice(None)) + idx(x)] @ GAMMA5.T
    return out


def staggered_dense(links, psi, mass, phases, dagger=False):
    # test/staggered_dirac.jl:53-77
    L = psi.shape[2:]
    result = np.empty_like(psi)
    hop = -0.5 if dagger else 0.5
    for x in sites(L):
        value = mass * psi[(slice(None), 0) + idx(x)].copy()
        for mu in range(4):
            xp, php = fermion_shift(x, mu, 1, L, phases)
            xm, phm = fermion_shift(x, mu, -1, L, phases)
            value = value + hop * eta(x, mu) * (
                mat(links[mu], x) @ (php * psi[(slice(None), 0) + idx(xp)]) -
                mat(links[mu], xm).conj().T @ (phm * psi[(slice(None), 0) + idx(xm)]))
        result[(slice(None), 0) + idx(x)] = value
    return result


def hisq_dense(fat, lng, psi, mass, eps, phases, dagger=False):
    # test/hisq_dirac.jl:30-62
    L = psi.shape[2:]
    result = np.empty_like(psi)
    sign = -1.0 if dagger else 1.0
    fc, lc = sign / 2, -sign * (1 + eps) / 48
    for x in sites(L):
        value = mass * psi[(slice(None), 0) + idx(x)].copy()
        for mu in range(4):
            e = eta(x, mu)
            for links, dist, coef in ((fat, 1, fc), (lng, 3, lc)):
                xp, php = fermion_shift(x, mu, dist, L, phases)
                xm, phm = fermion_shift(x, mu, -dist, L, phases)
                value = value + coef * e * (
                    mat(links[mu], x) @ (php * psi[(slice(None), 0) + idx(xp)]) -
                    mat(links[mu], xm).conj().T @ (phm * psi[(slice(None), 0) + idx(xm)]))
        result[(slice(None), 0) + idx(x)] = value
    return result


def path_dense(links, origin, path):
    # test/hisq_smearing.jl:1-23
    L = links[0].shape[2:]
    NC = links[0].shape[0]
    T = np.eye(NC, dtype=complex)
    site = origin
    for d in path:
        axis = abs(d) - 1
        if d > 0:
            T = T @ mat(links[axis], site)
            site = shift(site, axis, 1, L)
        else:
            site = shift(site, axis, -1, L)
            T = T @ mat(links[axis], site).conj().T
    return T


def fat7_dense(links, coefficients):
    """Level-1 reference (test/hisq_smearing.jl:25-77) generalised with the
    Lepage term of test/hisq_full_smearing.jl:14-36."""
    c1, c3, c5, c7, cl = coefficients
    L = links[0].shape[2:]
    NC = links[0].shape[0]
    out = [zeros(NC, NC, L) for _ in range(4)]
    for x in sites(L):
        for mu in range(1, 5):
            value = c1 * mat(links[mu - 1], x).copy()
            for nu in range(1, 5):
                if nu == mu:
                    continue
                for sn in (-1, 1):
                    value += c3 * path_dense(links, x, (sn * nu, mu, -sn * nu))
                    if cl:
                        value += cl * path_dense(
                            links, x, (sn * nu, sn * nu, mu, -sn * nu, -sn * nu))
                for rho in range(1, 5):
                    if rho in (mu, nu):
                        continue
                    for sn in (-1, 1):
                        for sr in (-1, 1):
                            value += c5 * path_dense(
                                links, x, (sn * nu, sr * rho, mu, -sr * rho, -sn * nu))
                    for sigma in range(1, 5):
                        if sigma in (mu, nu, rho):
                            continue
                        for sn, sr, ss in itertools.product((-1, 1), repeat=3):
                            value += c7 * path_dense(
                                links, x, (sn * nu, sr * rho, ss * sigma, mu,
                                           -ss * sigma, -sr * rho, -sn * nu))
            out[mu - 1][(slice(None), slice(None)) + idx(x)] = value
    return out


def project_u3_dense(V):
    # test/hisq_full_smearing.jl:1-12 (SVD polar factor U Vt)
    out = [np.empty_like(v) for v in V]
    L = V[0].shape[2:]
    for mu in range(4):
        for x in sites(L):
            u, _, vt = np.linalg.svd(mat(V[mu], x))
            out[mu][(slice(None), slice(None)) + idx(x)] = u @ vt
    return out


def naik_dense(W):
    # test/hisq_full_smearing.jl:38-50
    L = W[0].shape[2:]
    out = [np.empty_like(w) for w in W]
    for mu in range(1, 5):
        for x in sites(L):
            out[mu - 1][(slice(None), slice(None)) + idx(x)] = \
                path_dense(W, x, (mu, mu, mu))
    return out


def fingerprint(field):
    # test/staggered_dirac.jl:139-148 (column-major vec, 1-based weights)
    v = np.asarray(field).reshape(-1, order="F")
    i = np.arange(1, v.size + 1, dtype=np.float64)
    return np.array([v.real.sum(), v.imag.sum(), (i * v.real).sum(),
                     (i * v.imag).sum(), (np.abs(v) ** 2).sum()])


def gauge_transformations(L, NC=3):
    # test/staggered_dirac.jl:79-96
    G = zeros(NC, NC, L)
    for x in sites(L):
        coordinate = x[0] + 3 * x[1] + 5 * x[2] + 7 * x[3]
        if NC == 3:
            angles = (0.031 * coordinate, -0.047 * (coordinate + 1),
                      0.047 * (coordinate + 1) - 0.031 * coordinate)
        else:
            angles = tuple((-1) ** c * 0.037 * coordinate for c in range(1, NC + 1))
        for c in range(NC):
            G[(c, c) + idx(x)] = np.exp(1j * angles[c])
    return G


def gauge_transform(links, G, distance=1):
    L = links[0].shape[2:]
    out = [np.empty_like(u) for u in links]
    for x in sites(L):
        for mu in range(4):
            xp = shift(x, mu, distance, L)
            out[mu][(slice(None), slice(None)) + idx(x)] = \
                mat(G, x) @ mat(links[mu], x) @ mat(G, xp).conj().T
    return out


def transform_field(G, psi):
    out = np.empty_like(psi)
    for x in sites(psi.shape[2:]):
        out[(slice(None), slice(None)) + idx(x)] = \
            mat(G, x) @ psi[(slice(None), slice(None)) + idx(x)]
    return out


def plane_wave(L, momentum):
    w = zeros(1, 1, L)
    for x in sites(L):
        w[(0, 0) + idx(x)] = np.exp(1j * sum(momentum[m] * (x[m] - 1)
                                             for m in range(4)))
    return w


def rel_err(a, b):
    return float(np.linalg.norm((a - b).ravel()) /
                 max(np.linalg.norm(np.asarray(b).ravel()), 1e-300))


# ---------------------------------------------------------------------------
# domain wall (test/domainwall.jl:1-127): recipe and dense oracle
# ---------------------------------------------------------------------------
def domainwall_test_values(n1, n2, size, offset):
    """test/domainwall.jl:20-32 over a lattice of any rank (1-based coords)."""
    out = np.zeros((n1, n2) + tuple(size), dtype=np.complex128, order="F")
    for pos in itertools.product(*[range(1, n + 1) for n in size]):
        coordinate = sum((2 * (d + 1) - 1) * pos[d] for d in range(len(size)))
        for second in range(1, n2 + 1):
            for first in range(1, n1 + 1):
                out[(first - 1, second - 1) + tuple(p - 1 for p in pos)] = (
                    0.013 * (first + 2 * second + coordinate + offset) +
                    1j * 0.017 * (2 * first - second - coordinate + offset))
    return out


def domainwall_F_dense(psi, mass, adjoint=False):
    """test/domainwall.jl:34-55."""
    L5 = psi.shape[6]
    out = np.empty_like(psi)
    for s in range(1, L5 + 1):
        if adjoint:
            lo, hi = (s % L5) + 1, ((s - 2) % L5) + 1
            clo = -mass if s == L5 else 1.0
            chi = -mass if s == 1 else 1.0
        else:
            lo, hi = ((s - 2) % L5) + 1, (s % L5) + 1
            clo = -mass if s == 1 else 1.0
            chi = -mass if s == L5 else 1.0
        out[:, 0:2, ..., s - 1] = clo * psi[:, 0:2, ..., lo - 1]
        out[:, 2:4, ..., s - 1] = chi * psi[:, 2:4, ..., hi - 1]
    return out


def domainwall_DW_dense(links, psi, M, phases, adjoint=False):
    """test/domainwall.jl:57-86: (4+M) psi - 1/2 sum_mu hops on every slice."""
    L = psi.shape[2:6]
    L5 = psi.shape[6]
    out = np.empty_like(psi)
    eye = np.eye(4, dtype=complex)
    for s in range(L5):
        for x in sites(L):
            value = (4 + M) * psi[(slice(None), slice(None)) + idx(x) + (s,)].copy()
            for mu in range(4):
                xp, php = fermion_shift(x, mu, 1, L, phases)
                xm, phm = fermion_shift(x, mu, -1, L, phases)
                gf = eye + GAMMA[mu] if adjoint else eye - GAMMA[mu]
                gb = eye - GAMMA[mu] if adjoint else eye + GAMMA[mu]
                value -= 0.5 * mat(links[mu], x) @ (php * psi[(slice(None), slice(None)) + idx(xp) + (s,)]) @ gf.T
                value -= 0.5 * mat(links[mu], xm).conj().T @ (
                    phm * psi[(slice(None), slice(None)) + idx(xm) + (s,)]) @ gb.T
            out[(slice(None), slice(None)) + idx(x) + (s,)] = value
    return out


def domainwall_dense(links, psi, mass, M, a, b, c, phases, adjoint=False):
    """test/domainwall.jl:107-127 (generalised operator and its adjoint)."""
    A = np.asarray(a).reshape((1,) * 6 + (-1,))
    B = np.asarray(b).reshape((1,) * 6 + (-1,))
    C = np.asarray(c).reshape((1,) * 6 + (-1,))
    if adjoint:
        q = A * psi
        Fq = domainwall_F_dense(q, mass, adjoint=True)
        Dq = domainwall_DW_dense(links, q, M, phases, adjoint=True)
        return q - Fq + B * Dq + domainwall_F_dense(C * Dq, mass, adjoint=True)
    Fpsi = domainwall_F_dense(psi, mass)
    return A * (psi - Fpsi + domainwall_DW_dense(links, B * psi + C * Fpsi, M, phases))


# ---------------------------------------------------------------------------
# halo fill (LatticeMatrices_core.jl:550-567, 707-723)
# ---------------------------------------------------------------------------
def set_halo_dense(A, nw, phases):
    """set_halo! on one process, dimension by dimension as
    exchange_dim_local! does: the minus ghost slab takes the plus face divided
    by phase_d, the plus ghost slab the minus face times phase_d; slabs span
    the full padded extent of the other dimensions.  A: padded array in the
    reference's order (NC1, NC2, X+2nw, ...)."""
    A = np.array(A, copy=True)
    for d in range(A.ndim - 2):
        ax = d + 2
        n = A.shape[ax]

        def sl(r):
            return tuple(r if i == ax else slice(None) for i in range(A.ndim))
        A[sl(slice(0, nw))] = A[sl(slice(n - 2 * nw, n - nw))] / phases[d]
        A[sl(slice(n - nw, n))] = A[sl(slice(nw, 2 * nw))] * phases[d]
    return A
