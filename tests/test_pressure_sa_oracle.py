"""The smoothed-aggregation oracle (oracle/pressure_sa.py) against
independent sparse-matrix constructions: the stencil form of the pressure
operator, its transpose, the smoothed prolongator and restriction, the
Galerkin coarse operators on two levels (9-point stencils computed by
coloured probes), and a PCG solve."""
import numpy as np
import pytest
import scipy.sparse as sp


def pressure_state(Ny=24, Nx=48, iters=20):
    from oracle import Oracle

    from coldplate_b200 import cases
    c = cases.density_field(Ny, Nx, seed=0)
    prm = c.params()
    o = Oracle("f64", prm, cellType=c.cellType, hy=c.hy, hx=c.hx, U=c.U, Ht=c.Ht)
    o.run(iters)
    return o.get("dE"), o.get("dN"), prm["rho"], c.hx, c.hy


def csr_pressure(dE, dN, rho, hx, hy):
    """The reference's pressure rows, built row by row (simple_oracle.c
    pcg_matvec): S, W, P, E, N on the unknowns i in [1, M-1], j in [1, N-2]."""
    M, N = dN.shape[0], dE.shape[1]
    ni, nj = M - 1, N - 2
    k = lambda i, j: (i - 1) * nj + (j - 1)
    rows, cols, vals = [], [], []
    for i in range(1, M):
        for j in range(1, N - 1):
            aE = rho * dE[i, j] * hy
            aW = rho * dE[i, j - 1] * hy if j > 1 else 0.0
            aN = rho * dN[i, j] * hx if i < M - 1 else 0.0
            aS = rho * dN[i - 1, j] * hx if i > 1 else 0.0
            aP = aE + aW + aN + aS
            aP = 1.0 if aP < 1e-20 else aP
            rows.append(k(i, j)); cols.append(k(i, j)); vals.append(aP)
            for cond, c, a in ((i > 1, k(i - 1, j), aS), (j > 1, k(i, j - 1), aW), (j + 1 < N - 1, k(i, j + 1), aE),
                               (i < M - 1, k(i + 1, j), aN)):
                if cond:
                    rows.append(k(i, j)); cols.append(c); vals.append(-a)
    return sp.csr_matrix((vals, (rows, cols)), shape=(ni * nj, ni * nj)), ni, nj


def csr_of(A):
    from pressure_sa import dense
    return sp.csr_matrix(dense(A))


def p_matrices(lv):
    """P0 and P = (I - w D^-1 A) P0 as sparse matrices."""
    from pressure_sa import coarse_shape
    ni, nj = lv.shape
    ci, cj = coarse_shape(ni, nj)
    I, J = np.meshgrid(np.arange(ni) // 3, np.arange(nj) // 3, indexing="ij")
    P0 = sp.csr_matrix((np.ones(ni * nj), (np.arange(ni * nj), (I * cj + J).ravel())), shape=(ni * nj, ci * cj))
    A = csr_of(lv.A)
    P = (sp.identity(ni * nj) - lv.w * sp.diags(1.0 / lv.d.ravel()) @ A) @ P0
    return P0, P, A


def close(a, b, tol=1e-13):
    """Equal to rounding: the sums run in different orders."""
    assert np.abs(a - b).max() <= tol * np.abs(b).max(), np.abs(a - b).max() / np.abs(b).max()


@pytest.fixture(scope="module")
def state():
    return pressure_state()


def test_stencil_operator_equals_the_reference_rows(state):
    from pressure_sa import apply, apply_t, pressure_stencil
    dE, dN, rho, hx, hy = state
    A = pressure_stencil(dE, dN, rho, hx, hy)
    Acsr, ni, nj = csr_pressure(dE, dN, rho, hx, hy)
    rng = np.random.default_rng(1)
    x, y = rng.random((ni, nj)), rng.random((ni, nj))
    close(apply(A, x).ravel(), Acsr @ x.ravel())
    close(apply_t(A, y).ravel(), Acsr.T @ y.ravel())
    assert abs(Acsr - Acsr.T).max() == 0.0           # the pressure operator is symmetric


def test_prolongation_restriction_and_galerkin_on_two_levels(state):
    from pressure_sa import Level, coarse_shape, galerkin, lambda_max, pressure_stencil
    dE, dN, rho, hx, hy = state
    A = pressure_stencil(dE, dN, rho, hx, hy)
    rng = np.random.default_rng(2)
    for _ in range(2):                                  # level 0 (5-point) and level 1 (9-point)
        lv = Level(A, 4.0 / (3.0 * lambda_max(A)))
        P0, P, Acsr = p_matrices(lv)
        e = rng.random(coarse_shape(*lv.shape))
        r = rng.random(lv.shape)
        close(lv.prolong(e).ravel(), P @ e.ravel())
        close(lv.restrict(r).ravel(), P.T @ r.ravel())
        Ac = galerkin(lv)
        ref = (P.T @ Acsr @ P).toarray()
        got = csr_of(Ac).toarray()
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()
        assert np.count_nonzero(np.abs(ref) > 1e-14 * np.abs(ref).max(), axis=1).max() <= 9   # 9-point
        A = Ac


def test_sa_pcg_converges_fast(state):
    from pressure_sa import apply, hierarchy, pcg, pressure_stencil, vcycle
    dE, dN, rho, hx, hy = state
    A = pressure_stencil(dE, dN, rho, hx, hy)
    levels = hierarchy(A)
    b = np.random.default_rng(3).standard_normal(A[(0, 0)].shape)
    x, its = pcg(A, b, lambda r: vcycle(levels, r), tol=1e-6)
    assert np.linalg.norm(b - apply(A, x)) <= 1e-6 * np.linalg.norm(b)
    assert its <= 15, its
