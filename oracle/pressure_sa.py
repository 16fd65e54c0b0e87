"""CPU restatement of a smoothed-aggregation multigrid preconditioner for the
pressure-correction system, in the structured stencil form a GPU kernel
would use.  Test infrastructure only: it is the checker for that
preconditioner and for the claims made about it; nothing in the product
calls it.

The pressure system is the reference's (pressure_solver.cpp:462-816, the
matrix-free form of oracle/simple_oracle.c pcg_matvec): unknowns p'(i, j),
i in [1, M-1], j in [1, N-2], face coefficients rho dE hy (east/west) and
rho dN hx (north/south), no coupling across walls, the Dirichlet outlet
column p'(:, N-1) = 0 folded into the diagonal.  Here it is indexed on the
unknown grid (ni = M - 1 rows, nj = N - 2 columns, 0-based).

Operators are 9-point stencils: A[(di, dj)] is an ni x nj array and
(A x)[i, j] = sum over offsets (di, dj) in {-1, 0, 1}^2 of
A[(di, dj)][i, j] x[i + di, j + dj] (zero outside the grid).  The fine
operator uses only the five offsets of the 5-point stencil.

Smoothed aggregation with 3 x 3 aggregates (the cycle AMGCL's type-4
preconditioner runs, with geometric aggregates):
  P0        piecewise constant on aggregates i // 3, j // 3;
  P         = (I - w D^-1 A) P0 with w = 4 / (3 lambda_max(D^-1 A));
  A_c       = P^T A P, again a 9-point stencil on the coarse grid: the
              smoothed support of an aggregate is 5 x 5 fine cells, so two
              aggregates two coarse cells apart never meet through A.
A_c is computed exactly by nine probes: the aggregates of one colour
(I mod 3, J mod 3) have disjoint smoothed supports at least two cells
apart, so P applied to the indicator of a colour, then A, then P^T gives
every coarse row's entry towards its one neighbour of that colour.
"""
from __future__ import annotations

import numpy as np

OFFSETS = [(di, dj) for di in (-1, 0, 1) for dj in (-1, 0, 1)]


def pressure_stencil(dE, dN, rho: float, hx: float, hy: float) -> dict:
    """The pressure-correction operator as 9-point stencil arrays (corners
    zero) from the staggered dE ((M+1) x N) and dN (M x (N+1)), following
    the reference's row assembly (pressure_solver.cpp:733-742, as
    simple_oracle.c pcg_matvec restates it)."""
    dE = np.asarray(dE, dtype=np.float64)
    dN = np.asarray(dN, dtype=np.float64)
    M = dN.shape[0]
    N = dE.shape[1]
    ni, nj = M - 1, N - 2
    i = np.arange(1, M)[:, None]
    j = np.arange(1, N - 1)[None, :]
    aE = rho * dE[i, j] * hy
    aW = np.where(j > 1, rho * dE[i, np.maximum(j - 1, 0)] * hy, 0.0)
    aN = np.where(i < M - 1, rho * dN[np.minimum(i, M - 1), j] * hx, 0.0)
    aS = np.where(i > 1, rho * dN[np.maximum(i - 1, 0), j] * hx, 0.0)
    aP = aE + aW + aN + aS
    aP = np.where(aP < 1e-20, 1.0, aP)
    A = {o: np.zeros((ni, nj)) for o in OFFSETS}
    A[(0, 0)] = aP
    A[(0, -1)] = -aW
    A[(0, 1)] = np.where(j + 1 < N - 1, -aE, 0.0)     # no east entry at the last unknown column
    A[(-1, 0)] = -aS
    A[(1, 0)] = -aN
    return A


def apply(A: dict, x: np.ndarray) -> np.ndarray:
    """y = A x for a 9-point stencil operator."""
    ni, nj = x.shape
    xp = np.zeros((ni + 2, nj + 2))
    xp[1:-1, 1:-1] = x
    y = np.zeros_like(x)
    for (di, dj), a in A.items():
        y += a * xp[1 + di:1 + di + ni, 1 + dj:1 + dj + nj]
    return y


def apply_t(A: dict, x: np.ndarray) -> np.ndarray:
    """y = A^T x: row (i, j) of A^T takes entry (-di, -dj) of the neighbour."""
    ni, nj = x.shape
    y = np.zeros_like(x)
    for (di, dj), a in A.items():
        c = np.zeros((ni + 2, nj + 2))
        c[1 + di:1 + di + ni, 1 + dj:1 + dj + nj] = a * x        # contribution of row (i, j) to column (i+di, j+dj)
        y += c[1:-1, 1:-1]
    return y


def coarse_shape(ni: int, nj: int) -> tuple[int, int]:
    return (ni + 2) // 3, (nj + 2) // 3


def p0(e: np.ndarray, ni: int, nj: int) -> np.ndarray:
    """P0 e: the coarse value of each fine cell's aggregate."""
    return np.repeat(np.repeat(e, 3, axis=0), 3, axis=1)[:ni, :nj]


def p0t(r: np.ndarray) -> np.ndarray:
    """P0^T r: sums over the aggregates."""
    ni, nj = r.shape
    ci, cj = coarse_shape(ni, nj)
    out = np.zeros((ci, cj))
    np.add.at(out, (np.arange(ni)[:, None] // 3, np.arange(nj)[None, :] // 3), r)
    return out


def lambda_max(A: dict, iters: int = 30, seed: int = 0) -> float:
    """Largest eigenvalue of D^-1 A by power iteration (A symmetric
    positive definite, D^-1 A similar to a symmetric matrix)."""
    d = A[(0, 0)]
    x = np.random.default_rng(seed).random(d.shape) + 0.5
    lam = 1.0
    for _ in range(iters):
        y = apply(A, x) / d
        lam = float(np.linalg.norm(y) / np.linalg.norm(x))
        x = y / np.linalg.norm(y)
    return lam


class Level:
    def __init__(self, A: dict, w: float | None):
        self.A = A
        self.d = A[(0, 0)]
        self.w = w            # prolongator smoothing weight (None: coarsest level)

    @property
    def shape(self):
        return self.d.shape

    def prolong(self, e: np.ndarray) -> np.ndarray:
        """P e = P0 e - w D^-1 A P0 e."""
        ni, nj = self.shape
        q = p0(e, ni, nj)
        return q - self.w * apply(self.A, q) / self.d

    def restrict(self, r: np.ndarray) -> np.ndarray:
        """P^T r = P0^T (r - w A^T D^-1 r)."""
        return p0t(r - self.w * apply_t(self.A, r / self.d))


def galerkin(lv: Level) -> dict:
    """A_c = P^T A P as 9-point stencil arrays, by nine coloured probes."""
    ni, nj = lv.shape
    ci, cj = coarse_shape(ni, nj)
    I = np.arange(ci)[:, None]
    J = np.arange(cj)[None, :]
    Ac = {o: np.zeros((ci, cj)) for o in OFFSETS}
    for a in range(3):
        for b in range(3):
            ind = ((I % 3 == a) & (J % 3 == b)).astype(np.float64)
            col = lv.restrict(apply(lv.A, lv.prolong(ind)))        # row (I, J): entry towards its colour-(a, b) neighbour
            for (DI, DJ) in OFFSETS:
                m = ((I + DI) % 3 == a) & ((J + DJ) % 3 == b)
                m &= (I + DI >= 0) & (I + DI < ci) & (J + DJ >= 0) & (J + DJ < cj)
                Ac[(DI, DJ)] += np.where(m, col, 0.0)
    return Ac


def hierarchy(A: dict, coarsest: int = 64) -> list[Level]:
    """Levels down to at most `coarsest` unknowns (solved directly)."""
    levels = []
    while A[(0, 0)].size > coarsest:
        lv = Level(A, 4.0 / (3.0 * lambda_max(A)))
        levels.append(lv)
        A = galerkin(lv)
    levels.append(Level(A, None))
    return levels


def dense(A: dict) -> np.ndarray:
    """The stencil operator as a dense matrix (small levels and tests)."""
    ni, nj = A[(0, 0)].shape
    n = ni * nj
    out = np.zeros((n, n))
    for k in range(n):
        e = np.zeros(n)
        e[k] = 1.0
        out[:, k] = apply(A, e.reshape(ni, nj)).ravel()
    return out


def vcycle(levels: list[Level], b: np.ndarray, omega: float = 0.9, l: int = 0) -> np.ndarray:
    """One V(1,1) cycle with damped Jacobi smoothing from zero; a direct
    solve on the coarsest level."""
    lv = levels[l]
    if lv.w is None:
        return np.linalg.solve(dense(lv.A), b.ravel()).reshape(b.shape)
    x = omega * b / lv.d
    r = b - apply(lv.A, x)
    x = x + lv.prolong(vcycle(levels, lv.restrict(r), omega, l + 1))
    return x + omega * (b - apply(lv.A, x)) / lv.d


def pcg(A: dict, b: np.ndarray, precond, tol: float = 1e-6, maxit: int = 500) -> tuple[np.ndarray, int]:
    """CG with AMGCL's relative stop rule ||r|| <= tol ||b|| from x = 0;
    returns the solution and the completed iterations."""
    x = np.zeros_like(b)
    r = b.copy()
    z = precond(r)
    p = z.copy()
    rz = float(np.sum(r * z))
    bn = float(np.linalg.norm(b))
    for it in range(1, maxit + 1):
        Ap = apply(A, p)
        a = rz / float(np.sum(p * Ap))
        x += a * p
        r -= a * Ap
        if np.linalg.norm(r) <= tol * bn:
            return x, it
        z = precond(r)
        rz2 = float(np.sum(r * z))
        p = z + (rz2 / rz) * p
        rz = rz2
    return x, maxit
