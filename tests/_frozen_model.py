"""Test infrastructure: the fixed-point model the adjoint differentiates,
restated on the FP64 oracle, with its Jacobian by central differences.

At a converged state X = (u, v, p) of the SIMPLE iteration the model is
  G_u = x_s - u   on every U / V unknown whose sweep result x_s lies inside
                  the clamp (x_s: s Jacobi sweeps of the momentum system
                  assembled at X, from x_0 = u; iterations.cpp:160,
                  momentum_solver.cpp:197-351, jacobi_solver.cpp:20-75),
  G_u = u -+ maxVel on the unknowns the scatter clamps,
  G_c = rho hy (u(i,j-1) - u(i,j)) + rho hx (v(i-1,j) - v(i,j)), the mass
        imbalance of the pressure unknowns (pressure_solver.cpp:733-742),
with s and the clamped set frozen at the state.  The sweeps run in the
oracle (momentumTol 0, maxMomentumIter s).  Ghost values follow the
reference's boundary conditions (boundaries.cpp:50-146): u(i,N-1) = u(i,N-2),
v(i,N) = v(i,N-1), p(i,0) = p(i,1), p(0,j) = p(1,j), p(M,j) = p(M-1,j),
p(i,N-1) = p(i,N) = 0.  The objective is the full-system total-pressure drop
of the boundary patches (postprocessing.cpp:245-327).
"""
import numpy as np

from oracle import Oracle


class FrozenModel:
    def __init__(self, case, base_prm: dict, state: dict, sweeps_u: int, sweeps_v: int):
        mk = lambda prm: Oracle("f64", prm, cellType=case.cellType, hy=case.hy, hx=case.hx, U=case.U, Ht=case.Ht)
        self.o = mk(base_prm)
        self.oU = mk(dict(base_prm, momentumTol=0.0, maxMomentumIter=int(sweeps_u)))
        self.oV = mk(dict(base_prm, momentumTol=0.0, maxMomentumIter=int(sweeps_v)))
        for q in (self.o, self.oU, self.oV):
            q.set_inlet_velocity(case.U)
        M, N = self.o.M, self.o.N
        self.M, self.N = M, N
        self.u0, self.v0, self.p0 = (np.array(state[f], dtype=np.float64) for f in ("u", "v", "p"))
        self.uI = [(i, j) for i in range(1, M) for j in range(1, N - 1)]
        self.vI = [(i, j) for i in range(1, M - 1) for j in range(1, N)]
        self.pI = [(i, j) for i in range(1, M) for j in range(1, N - 1)]
        self.keys = [("u", a) for a in self.uI] + [("v", a) for a in self.vI] + [("p", a) for a in self.pI]
        self.nu, self.nv = len(self.uI), len(self.vI)
        self.rh, self.rx = base_prm["rho"] * case.hy, base_prm["rho"] * case.hx
        self.mv = 3.0 * max(abs(case.U), 0.1)
        self.X0 = self.pack({"u": self.u0, "v": self.v0, "p": self.p0})
        us, vs = self._stars(self.u0, self.v0, self.p0)
        self.cu = np.array([abs(abs(us[a]) - self.mv) <= 1e-12 * self.mv for a in self.uI])
        self.cv = np.array([abs(abs(vs[a]) - self.mv) <= 1e-12 * self.mv for a in self.vI])

    def pack(self, d: dict) -> np.ndarray:
        return np.array([d[f][a] for (f, a) in self.keys])

    def fields(self, X):
        M, N = self.M, self.N
        u, v, p = self.u0.copy(), self.v0.copy(), self.p0.copy()
        for k, a in enumerate(self.uI):
            u[a] = X[k]
        for k, a in enumerate(self.vI):
            v[a] = X[self.nu + k]
        for k, a in enumerate(self.pI):
            p[a] = X[self.nu + self.nv + k]
        u[:, N - 1] = u[:, N - 2]
        v[:, N] = v[:, N - 1]
        p[1:M, 0] = p[1:M, 1]
        p[0, 1:N] = p[1, 1:N]
        p[M, 1:N] = p[M - 1, 1:N]
        p[1:M, N - 1] = 0.0
        p[1:M, N] = 0.0
        return u, v, p

    def _stars(self, u, v, p):
        out = []
        for q, isU in ((self.oU, True), (self.oV, False)):
            q.set("u", u)
            q.set("v", v)
            q.set("p", p)
            q.momentum(isU)
            out.append(q.get("uStar" if isU else "vStar"))
        return out

    def G(self, X):
        u, v, p = self.fields(X)
        us, vs = self._stars(u, v, p)
        gu = np.array([us[a] - u[a] for a in self.uI])
        gv = np.array([vs[a] - v[a] for a in self.vI])
        uu = np.array([u[a] for a in self.uI])
        vv = np.array([v[a] for a in self.vI])
        gu[self.cu] = uu[self.cu] - np.sign(uu[self.cu]) * self.mv
        gv[self.cv] = vv[self.cv] - np.sign(vv[self.cv]) * self.mv
        gc = np.array([self.rh * (u[i, j - 1] - u[i, j]) + self.rx * (v[i - 1, j] - v[i, j]) for (i, j) in self.pI])
        return np.concatenate([gu, gv, gc])

    def J(self, X):
        u, v, p = self.fields(X)
        for f, a in (("u", u), ("v", v), ("p", p)):
            self.o.set(f, a)
        return self.o.sample_patch(True)[4] - self.o.sample_patch(False)[4]

    def jacobians(self, rel_step: float = 1e-6):
        """Dense dG/dX and dJ/dX by central differences; steps rel_step x
        max(|x|, 1) for velocities (wide enough to straddle the kinks of
        faces whose velocity is zero up to rounding) and x max(|p|, 1e-3)
        for pressures."""
        X0 = self.X0
        n = len(X0)
        floor = np.r_[np.ones(self.nu + self.nv), 1e-3 * np.ones(len(self.pI))]
        scale = np.maximum(np.abs(X0), floor)
        GX, JX = np.zeros((n, n)), np.zeros(n)
        for k in range(n):
            h = rel_step * scale[k]
            Xp, Xm = X0.copy(), X0.copy()
            Xp[k] += h
            Xm[k] -= h
            GX[:, k] = (self.G(Xp) - self.G(Xm)) / (2 * h)
            JX[k] = (self.J(Xp) - self.J(Xm)) / (2 * h)
        return GX, JX
