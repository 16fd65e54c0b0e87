// Discrete adjoint of the pressure drop with respect to the density field.
//
// The reference has no flow adjoint (its only adjoint is the 2-D conduction
// toy in AdjointMethod/thermal_adjoint.py); this is new.  It differentiates
// the fixed point that the reference's SIMPLE iteration actually reaches,
// velocity clamps included.
//
// One outer iteration (iterations.cpp:82-659) assembles the momentum system
// at the current state X = (u, v, p), runs s Jacobi sweeps from x_0 = u
// (jacobi_solver.cpp:20-75, s set by its stop rule), clamps the result to
// +-maxVel (momentum_solver.cpp:335-351), and corrects with p' from the mass
// imbalance (iterations.cpp:556-597).  At a fixed point p' = 0, and with
//   y_0 = 0,  y_{j+1} = D^-1 (r0 + N y_j)   (x_j = u + y_j; D = aP0 / uvAlpha,
//   N the off-diagonal coefficients, r0 = b - A u = -R(X) the unrelaxed
//   momentum residual of the flux form below)
// the state satisfies
//   F_u = y_s = 0                 on every U / V unknown whose sweep result
//                                  lies inside the clamp,
//   u = +-maxVel                  on the unknowns the scatter clamps,
//   R_c = 0                       the mass imbalance of the pressure unknowns.
// Where a velocity sits on the clamp the momentum residual does not vanish
// near it, and y_s depends on the sweep count s and on uvAlpha; with s and
// the clamped set frozen (both are locally constant in gamma) this system
// is smooth, and its derivative is what central differences of converged
// solves measure.  Without clamps it reduces to R = 0.
//
// R_u, the U-momentum balance of momentum_solver.cpp:197-314 with the
// relaxation cancelled, in flux form:
//        De(2uP-uE-uW) + Dn(1+hN)(uP-uN) + Dn(1+hS)(uP-uS)
//        + Fe phi_e - Fw phi_w + Fn phi_n - Fs phi_s + (sink + alpha vol) uP
//        - hy (pP - pE)
// where F are the clamped face-average mass fluxes and phi the SOU face
// values of convection.cpp:53-186 (FOU where the SOU stencil is missing or
// convectionScheme = 0); the same for R_v.  R_c: the mass imbalance
// massW - massE + massS - massN (pressure_solver.cpp:733-742).  Boundary
// values enter through the BCs of boundaries.cpp:50-146: the outlet copies
// u(i,N-1) = u(i,N-2) and v(i,N) = v(i,N-1) map to unknowns, walls, inlet and
// p(:,N-1) = 0 are constants.
//
// J = full-system total-pressure drop (SIMPLE.cpp:432): inlet patch
// mass-flux-weighted total pressure minus the outlet patch's
// (postprocessing.cpp:245-327).
//
// Adjoint: J_X^T lambda = dJ/dX, solved by restarted flexible GMRES.  The
// product J_X^T lambda runs the s sweeps in reverse (stored forward
// iterates), which gives the adjoints of r0 and of the coefficients, then
// scatters them through the assembly: every Newton term of the upwind
// switches, SOU branches and face-velocity clamps.  The preconditioner is a
// transposed SIMPLE step for this system: -1 on the momentum rows (F_u is
// already a Jacobi-preconditioned residual), then a pressure-like solve whose
// operator is uvAlpha times the forward pressure-correction matrix with the
// clamped faces removed (a clamped face carries a fixed flux, so it does not
// couple the pressure on either side), solved by the forward (multigrid)
// PCG kernel with a fixed iteration count; the flexible variant stays exact
// under that.
// Gradient: dJ/dgamma = -lambda^T dF/dgamma, local through
// alpha_face = (alpha(cL) + alpha(cR)) / 2 with
// alpha(g) = alpha_max (1 - g) / (1 + q g + 1e-10) (SIMPLE.cpp:770), which
// enters r0 and D; thresholds on gamma (inlet, half-cell and sampling masks)
// are piecewise constant and contribute nothing.
#pragma once

#include "cp_kernels.cuh"

namespace cp {

struct AdjVecs {
    double *lu, *lv, *lc;      // lambda on U / V / continuity rows
    double *yu, *yv, *yp;      // J^T lambda on U / V / p unknowns
    double *gu, *gv, *gp;      // dJ/dX
    double *du, *dv;           // momentum corrections (Jacobi iterates, ping-pong with eu, ev)
    double *eu, *ev;
};

// atomic add of a contribution to an unknown; `ok` is false for constants
__device__ __forceinline__ void adj_add(double* y, size_t c, double v, bool ok) {
    if (ok && v != 0.0) atomicAdd(y + c, v);
}

// Face value phi and its derivatives for one face, given the upwind side.
// up/dn: the FOU value (upwind cell) and the SOU second point.
struct Phi {
    double val;
    double dUp, dUpUp, dDn;   // d phi / d(upwind), d/d(second upwind), d/d(downwind)
};

// phi for F >= 0 (flow from "lo" to "hi"): FOU lo, SOU 1.5 lo - 0.5 lolo;
// for F < 0: FOU hi, SOU 1.5 hi - 0.5 hihi.  Returns weights on (lo, lolo,
// hi, hihi).
struct FaceW {
    double lo, lolo, hi, hihi, val;
};

// Kinks.  A face whose velocity is zero up to rounding (|x| <= kKinkRel
// maxVel: the symmetry plane of a jet, a stagnant corner) sits on the upwind
// switch, and the sign the rounding gives it picks a branch at random.  There
// the derivative is the mean of the two branches', the one central
// differences of the converged solve measure: F phi and its derivative in F
// take both branches' weights halved (F phi itself is zero there), and the
// coefficients max(0, +-F) change with slope 1/2.  Likewise a face average on
// the clamp (|x| = maxVel, between two clamped velocities) has clamp slope
// 1/2.
constexpr double kKinkRel = 1e-9;
__device__ __forceinline__ bool kink0(double x, double mv) { return fabs(x) <= kKinkRel * mv; }
// d max(0, F) / dF and d max(0, -F) / d(-F) at the face velocity x
__device__ __forceinline__ double upw_pos(double x, double mv) { return kink0(x, mv) ? 0.5 : (x > 0.0 ? 1.0 : 0.0); }
__device__ __forceinline__ double upw_neg(double x, double mv) { return kink0(x, mv) ? 0.5 : (x < 0.0 ? 1.0 : 0.0); }

__device__ __forceinline__ FaceW face_phi(double F, double lo, double lolo, double hi, double hihi, bool souLo,
                                          bool souHi, bool kink = false) {
    FaceW w{0, 0, 0, 0, 0};
    const double wl = kink ? 0.5 : (F >= 0.0 ? 1.0 : 0.0), wh = 1.0 - wl;
    if (souLo) { w.lo = 1.5 * wl; w.lolo = -0.5 * wl; } else { w.lo = wl; }
    if (souHi) { w.hi = 1.5 * wh; w.hihi = -0.5 * wh; } else { w.hi = wh; }
    w.val = w.lo * lo + w.lolo * lolo + w.hi * hi + w.hihi * hihi;
    return w;
}

// clamp derivative: 1 inside [-maxVel, maxVel], 0 where the clamp acts, 1/2
// on it
__device__ __forceinline__ double clampd(double x, double m) {
    const double ax = fabs(x);
    return ax > m * (1.0 + 1e-12) ? 0.0 : (ax >= m * (1.0 - 1e-12) ? 0.5 : 1.0);
}

struct AdjCtx {
    KParams k;
    const double *u, *v, *p, *alpha, *gamma;
    double maxVel;
};

// ---------------------------------------------------------------- J^T lambda
// U row (i, j): accumulate lambda * dR_u/dX into y.  Returns R_u (for tests).
__device__ double adj_row_u(const AdjCtx& a, int i, int j, double lam, AdjVecs V, bool scatter) {
    const KParams& k = a.k;
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const double* u = a.u;
    const double* v = a.v;
    const double hx = k.hx, hy = k.hy, vol = hx * hy;
    const double cs = k.convScale, cE = cs * k.rho * hy, cN = cs * k.rho * hx;
    const double De = k.eta * (hy / hx), Dn = k.eta * (hx / hy);
    // unknown map: U unknowns i in [1,M-1], j in [1,N-2]; u(i,N-1) -> u(i,N-2)
    auto U = [&](int ii, int jj, size_t& c) -> bool {
        if (ii < 1 || ii > M - 1 || jj < 1) return false;
        if (jj == N - 1) jj = N - 2;
        if (jj > N - 2) return false;
        c = at(d, ii, jj);
        return true;
    };
    auto Vk = [&](int ii, int jj, size_t& c) -> bool {  // V unknowns i in [1,M-2], j in [1,N-1]
        if (ii < 1 || ii > M - 2 || jj < 1) return false;
        if (jj == N) jj = N - 1;
        if (jj > N - 1) return false;
        c = at(d, ii, jj);
        return true;
    };
    auto uv = [&](int ii, int jj) -> double { return u[at(d, ii, jj)]; };
    auto vv = [&](int ii, int jj) -> double { return v[at(d, ii, jj)]; };
    const double uP = uv(i, j), uE = uv(i, j + 1), uW = uv(i, j - 1), uN = uv(i + 1, j), uS = uv(i - 1, j);
    const double uEE = (j + 2 < N) ? uv(i, j + 2) : 0.0, uWW = (j >= 2) ? uv(i, j - 2) : 0.0;
    const double uNN = (i + 2 <= M) ? uv(i + 2, j) : 0.0, uSS = (i >= 2) ? uv(i - 2, j) : 0.0;
    const double mv = a.maxVel;
    const double xe = 0.5 * (uP + uE), xw = 0.5 * (uW + uP);
    const double xn = 0.5 * (vv(i, j) + vv(i, j + 1)), xs = 0.5 * (vv(i - 1, j) + vv(i - 1, j + 1));
    const double Fe = cE * dclamp(xe, -mv, mv), Fw = cE * dclamp(xw, -mv, mv);
    const double Fn = cN * dclamp(xn, -mv, mv), Fs = cN * dclamp(xs, -mv, mv);
    const double gE = 0.5 * cE * clampd(xe, mv), gW = 0.5 * cE * clampd(xw, mv);
    const double gN = 0.5 * cN * clampd(xn, mv), gS = 0.5 * cN * clampd(xs, mv);
    const bool sou = k.sou;
    // faces: east (lo = P, hi = E), west (lo = W, hi = P), north (lo = P, hi = N), south (lo = S, hi = P)
    const FaceW pe = face_phi(Fe, uP, uW, uE, uEE, sou && j >= 2, sou && j + 2 < N, kink0(xe, mv));
    const FaceW pw = face_phi(Fw, uW, uWW, uP, uE, sou && j >= 2, sou && j + 1 < N, kink0(xw, mv));
    const FaceW pn = face_phi(Fn, uP, uS, uN, uNN, sou && i >= 1, sou && i + 2 <= M, kink0(xn, mv));
    const FaceW ps = face_phi(Fs, uS, uSS, uP, uN, sou && i >= 2, sou && i + 1 <= M, kink0(xs, mv));
    // half-cell wall flags (boundaries.cpp:148-171), as in the assembly
    const double gF = 0.5 * (a.gamma[at(d, i - 1, j - 1)] + a.gamma[at(d, i - 1, j)]);
    const double vt = 1e-8;
    const bool hS = gF >= 0.999 && i == 1 && fabs(uv(0, j)) <= vt && fabs(vv(0, j)) <= vt && fabs(vv(0, j + 1)) <= vt;
    const bool hN = gF >= 0.999 && i == M - 1 && fabs(uv(M, j)) <= vt && fabs(vv(M - 1, j)) <= vt &&
                    fabs(vv(M - 1, j + 1)) <= vt;
    const double DnN = Dn * (hN ? 2.0 : 1.0), DnS = Dn * (hS ? 2.0 : 1.0);
    const double alphaF = 0.5 * (a.alpha[at(d, i - 1, j - 1)] + a.alpha[at(d, i - 1, j)]);
    const double Kd = k.sinkDiag + alphaF * vol;
    const double pP = a.p[at(d, i, j)], pE = a.p[at(d, i, j + 1)];
    const double R = De * (2 * uP - uE - uW) + DnN * (uP - uN) + DnS * (uP - uS) + Fe * pe.val - Fw * pw.val +
                     Fn * pn.val - Fs * ps.val + Kd * uP - hy * (pP - pE);
    if (!scatter) return R;
    // d/du: diffusion + flux derivative + face-value derivative
    double dP = 2 * De + DnN + DnS + Kd + gE * pe.val - gW * pw.val + Fe * pe.lo - Fw * pw.hi + Fn * pn.lo - Fs * ps.hi;
    double dE_ = -De + gE * pe.val + Fe * pe.hi - Fw * pw.hihi;
    double dW_ = -De + Fe * pe.lolo - gW * pw.val - Fw * pw.lo;
    double dEE = Fe * pe.hihi;
    double dWW = -Fw * pw.lolo;
    double dN_ = -DnN + Fn * pn.hi - Fs * ps.hihi;
    double dNN = Fn * pn.hihi;
    double dS_ = -DnS + Fn * pn.lolo - Fs * ps.lo;
    double dSS = -Fs * ps.lolo;
    size_t c;
    if (U(i, j, c)) adj_add(V.yu, c, lam * dP, true);
    if (U(i, j + 1, c)) adj_add(V.yu, c, lam * dE_, true);
    if (U(i, j - 1, c)) adj_add(V.yu, c, lam * dW_, true);
    if (j + 2 < N && U(i, j + 2, c)) adj_add(V.yu, c, lam * dEE, true);
    if (j >= 2 && U(i, j - 2, c)) adj_add(V.yu, c, lam * dWW, true);
    if (U(i + 1, j, c)) adj_add(V.yu, c, lam * dN_, true);
    if (i + 2 <= M && U(i + 2, j, c)) adj_add(V.yu, c, lam * dNN, true);
    if (U(i - 1, j, c)) adj_add(V.yu, c, lam * dS_, true);
    if (i >= 2 && U(i - 2, j, c)) adj_add(V.yu, c, lam * dSS, true);
    // d/dv through Fn, Fs
    if (Vk(i, j, c)) adj_add(V.yv, c, lam * gN * pn.val, true);
    if (Vk(i, j + 1, c)) adj_add(V.yv, c, lam * gN * pn.val, true);
    if (Vk(i - 1, j, c)) adj_add(V.yv, c, -lam * gS * ps.val, true);
    if (Vk(i - 1, j + 1, c)) adj_add(V.yv, c, -lam * gS * ps.val, true);
    // d/dp: pP always an unknown here; pE unless j + 1 == N - 1 (p(:,N-1) = 0)
    adj_add(V.yp, at(d, i, j), -lam * hy, true);
    if (j + 1 <= N - 2) adj_add(V.yp, at(d, i, j + 1), lam * hy, true);
    return R;
}

// V row (i, j)
__device__ double adj_row_v(const AdjCtx& a, int i, int j, double lam, AdjVecs V, bool scatter) {
    const KParams& k = a.k;
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const double* u = a.u;
    const double* v = a.v;
    const double hx = k.hx, hy = k.hy, vol = hx * hy;
    const double cs = k.convScale, cE = cs * k.rho * hy, cN = cs * k.rho * hx;
    const double De = k.eta * (hy / hx), Dn = k.eta * (hx / hy);
    auto U = [&](int ii, int jj, size_t& c) -> bool {
        if (ii < 1 || ii > M - 1 || jj < 1) return false;
        if (jj == N - 1) jj = N - 2;
        if (jj > N - 2) return false;
        c = at(d, ii, jj);
        return true;
    };
    auto Vk = [&](int ii, int jj, size_t& c) -> bool {
        if (ii < 1 || ii > M - 2 || jj < 1) return false;
        if (jj == N) jj = N - 1;
        if (jj > N - 1) return false;
        c = at(d, ii, jj);
        return true;
    };
    auto uv = [&](int ii, int jj) -> double { return u[at(d, ii, jj)]; };
    auto vv = [&](int ii, int jj) -> double { return v[at(d, ii, jj)]; };
    const double vP = vv(i, j), vE = vv(i, j + 1), vW = vv(i, j - 1), vN = vv(i + 1, j), vS = vv(i - 1, j);
    const double vEE = (j + 2 <= N) ? vv(i, j + 2) : 0.0, vWW = (j >= 2) ? vv(i, j - 2) : 0.0;
    const double vNN = (i + 2 < M) ? vv(i + 2, j) : 0.0, vSS = (i >= 2) ? vv(i - 2, j) : 0.0;
    const double mv = a.maxVel;
    const double xe = 0.5 * (uv(i, j) + uv(i + 1, j)), xw = 0.5 * (uv(i, j - 1) + uv(i + 1, j - 1));
    const double xn = 0.5 * (vP + vN), xs = 0.5 * (vS + vP);
    const double Fe = cE * dclamp(xe, -mv, mv), Fw = cE * dclamp(xw, -mv, mv);
    const double Fn = cN * dclamp(xn, -mv, mv), Fs = cN * dclamp(xs, -mv, mv);
    const double gE = 0.5 * cE * clampd(xe, mv), gW = 0.5 * cE * clampd(xw, mv);
    const double gN = 0.5 * cN * clampd(xn, mv), gS = 0.5 * cN * clampd(xs, mv);
    const bool sou = k.sou;
    const FaceW pe = face_phi(Fe, vP, vW, vE, vEE, sou && j >= 2, sou && j + 2 <= N, kink0(xe, mv));
    const FaceW pw = face_phi(Fw, vW, vWW, vP, vE, sou && j >= 2, sou && j + 1 <= N, kink0(xw, mv));
    const FaceW pn = face_phi(Fn, vP, vS, vN, vNN, sou && i >= 1, sou && i + 2 < M, kink0(xn, mv));
    const FaceW ps = face_phi(Fs, vS, vSS, vP, vN, sou && i >= 2, sou && i + 1 < M, kink0(xs, mv));
    const double gF = 0.5 * (a.gamma[at(d, i - 1, j - 1)] + a.gamma[at(d, i, j - 1)]);
    const double vt = 1e-8;
    const bool hW = gF >= 0.999 && j == 1 && !(fabs(k.targetVel) > vt) && fabs(vv(i, 0)) <= vt &&
                    fabs(uv(i, 0)) <= vt && fabs(uv(i + 1, 0)) <= vt;
    const bool hE = gF >= 0.999 && j == N - 1 && !(fabs(a.p[at(d, i, N)]) <= 1e-8) && fabs(vv(i, N)) <= vt &&
                    fabs(uv(i, N - 1)) <= vt && fabs(uv(i + 1, N - 1)) <= vt;
    const double DeW = De * (hW ? 2.0 : 1.0), DeE = De * (hE ? 2.0 : 1.0);
    const double alphaF = 0.5 * (a.alpha[at(d, i - 1, j - 1)] + a.alpha[at(d, i, j - 1)]);
    const double Kd = k.sinkDiag + alphaF * vol;
    const double pP = a.p[at(d, i, j)], pN = a.p[at(d, i + 1, j)];
    const double R = DeW * (vP - vW) + DeE * (vP - vE) + Dn * (2 * vP - vN - vS) + Fe * pe.val - Fw * pw.val +
                     Fn * pn.val - Fs * ps.val + Kd * vP - hx * (pP - pN);
    if (!scatter) return R;
    double dP = DeW + DeE + 2 * Dn + Kd + Fe * pe.lo - Fw * pw.hi + gN * pn.val - gS * ps.val + Fn * pn.lo - Fs * ps.hi;
    double dE_ = -DeE + Fe * pe.hi - Fw * pw.hihi;
    double dW_ = -DeW + Fe * pe.lolo - Fw * pw.lo;
    double dEE = Fe * pe.hihi;
    double dWW = -Fw * pw.lolo;
    double dN_ = -Dn + gN * pn.val + Fn * pn.hi - Fs * ps.hihi;
    double dNN = Fn * pn.hihi;
    double dS_ = -Dn + Fn * pn.lolo - gS * ps.val - Fs * ps.lo;
    double dSS = -Fs * ps.lolo;
    size_t c;
    if (Vk(i, j, c)) adj_add(V.yv, c, lam * dP, true);
    if (Vk(i, j + 1, c)) adj_add(V.yv, c, lam * dE_, true);
    if (Vk(i, j - 1, c)) adj_add(V.yv, c, lam * dW_, true);
    if (j + 2 <= N && Vk(i, j + 2, c)) adj_add(V.yv, c, lam * dEE, true);
    if (j >= 2 && Vk(i, j - 2, c)) adj_add(V.yv, c, lam * dWW, true);
    if (Vk(i + 1, j, c)) adj_add(V.yv, c, lam * dN_, true);
    if (i + 2 < M && Vk(i + 2, j, c)) adj_add(V.yv, c, lam * dNN, true);
    if (Vk(i - 1, j, c)) adj_add(V.yv, c, lam * dS_, true);
    if (i >= 2 && Vk(i - 2, j, c)) adj_add(V.yv, c, lam * dSS, true);
    // d/du through Fe (u(i,j), u(i+1,j)) and Fw (u(i,j-1), u(i+1,j-1))
    if (U(i, j, c)) adj_add(V.yu, c, lam * gE * pe.val, true);
    if (U(i + 1, j, c)) adj_add(V.yu, c, lam * gE * pe.val, true);
    if (U(i, j - 1, c)) adj_add(V.yu, c, -lam * gW * pw.val, true);
    if (U(i + 1, j - 1, c)) adj_add(V.yu, c, -lam * gW * pw.val, true);
    // d/dp: p(i,j) and p(i+1,j) are unknowns when j <= N-2
    if (j <= N - 2) {
        adj_add(V.yp, at(d, i, j), -lam * hx, true);
        adj_add(V.yp, at(d, i + 1, j), lam * hx, true);
    }
    return R;
}

// continuity row (i, j): R_c = rho hy (u(i,j-1) - u(i,j)) + rho hx (v(i-1,j) - v(i,j))
__device__ double adj_row_c(const AdjCtx& a, int i, int j, double lam, AdjVecs V, bool scatter) {
    const KParams& k = a.k;
    const Dims d = k.d;
    const int M = d.M;
    const double rh = k.rho * k.hy, rx = k.rho * k.hx;
    const double R = rh * (a.u[at(d, i, j - 1)] - a.u[at(d, i, j)]) + rx * (a.v[at(d, i - 1, j)] - a.v[at(d, i, j)]);
    if (!scatter) return R;
    if (j - 1 >= 1) adj_add(V.yu, at(d, i, j - 1), lam * rh, true);
    adj_add(V.yu, at(d, i, j), -lam * rh, true);
    if (i - 1 >= 1) adj_add(V.yv, at(d, i - 1, j), lam * rx, true);
    if (i <= M - 2) adj_add(V.yv, at(d, i, j), -lam * rx, true);
    return R;
}

// ---------------------------------------------------------------- frozen sweeps
// One momentum component's Jacobi system at the converged state and the
// adjoints its reverse sweeps accumulate.
struct AdjSweep {
    const double *aP, *aE, *aW, *aN, *aS;   // relaxed diagonal D, masked off-diagonals N
    const double* clamp;                     // 1 where the scatter clamps the sweep result
    double *r0b, *eb, *wb, *nb, *sb, *db;    // adjoints of r0, aE, aW, aN, aS and D
};

// One forward Jacobi sweep x+ = x + (b - A x) / aP of one component in the
// reference's arithmetic (CSR order S, W, P, E, N; jacobi_solver.cpp:44-60)
// from x = field (x == nullptr) or x; part[block] = the block's sum of r^2
// of the pre-update residual (the stop rule's sum).
template <bool IsU>
__global__ void k_adj_sweep(KParams k, MomSys<double> S, const double* field, const double* x, double* xn,
                            double* part) {
    __shared__ double sm[32];
    const Dims d = k.d;
    int i1, j1;
    mom_range<IsU>(d, i1, j1);
    const int n = i1 * j1;
    const double* X = x ? x : field;
    double acc[1] = {0.0};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int i = 1 + t / j1, j = 1 + t % j1;
        const size_t c = at(d, i, j);
        double Ax = 0.0;
        Ax += (-S.aS[c]) * ((i > 1) ? X[c - d.P] : 0.0);
        Ax += (-S.aW[c]) * ((j > 1) ? X[c - 1] : 0.0);
        Ax += S.aP[c] * X[c];
        Ax += (-S.aE[c]) * ((j < j1) ? X[c + 1] : 0.0);
        Ax += (-S.aN[c]) * ((i < i1) ? X[c + d.P] : 0.0);
        const double r = S.b[c] - Ax;
        xn[c] = X[c] + r / S.aP[c];
        acc[0] += r * r;
    }
    block_sum<1>(acc, sm);
    if (threadIdx.x == 0) part[blockIdx.x] = acc[0];
}

// clamp[c] = 1 where the sweep result lies outside +-maxVel (the scatter
// clamps it, momentum_solver.cpp:342), else 0
template <bool IsU>
__global__ void k_adj_clampmask(KParams k, const double* xs, double maxVel, double* clamp) {
    const Dims d = k.d;
    int i1, j1;
    mom_range<IsU>(d, i1, j1);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < i1 * j1; t += gridDim.x * blockDim.x) {
        const size_t c = at(d, 1 + t / j1, 1 + t % j1);
        clamp[c] = (xs[c] < -maxVel || maxVel < xs[c]) ? 1.0 : 0.0;
    }
}

// part[2 b] = clamped unknowns of block b, part[2 b + 1] = the largest
// |x_s - x_0| over its unclamped unknowns (U and V): how far the state is
// from a fixed point of the frozen iteration
__global__ void k_adj_fixedpoint(KParams k, const double* xsU, const double* u, const double* clampU,
                                 const double* xsV, const double* v, const double* clampV, double* part) {
    __shared__ double sm[64];
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const int nU = (M - 1) * (N - 2), nV = (M - 2) * (N - 1);
    double cnt = 0.0, mx = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nU + nV; t += gridDim.x * blockDim.x) {
        const bool isU = t < nU;
        const int q = isU ? t : t - nU;
        const int w = isU ? N - 2 : N - 1;
        const size_t c = at(d, 1 + q / w, 1 + q % w);
        const double cl = (isU ? clampU : clampV)[c];
        if (cl != 0.0) cnt += 1.0;
        else mx = dmax(mx, fabs((isU ? xsU : xsV)[c] - (isU ? u : v)[c]));
    }
    double a[1] = {cnt};
    block_sum<1>(a, sm);
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0) sm[32 + (threadIdx.x >> 5)] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int q = 0; q < (int)((blockDim.x + 31) >> 5); ++q) m = dmax(m, sm[32 + q]);
        part[2 * blockIdx.x] = a[0];
        part[2 * blockIdx.x + 1] = m;
    }
}

// One reverse sweep of the recurrence y_{j+1} = D^-1 (r0 + N y_j) of one
// component (y_j = x_j - field): with w = ybar / D on the unknowns,
// r0b += w, the coefficient adjoints eb.. += w y_j(neighbour), db -= w y_{j+1},
// and ybar' = N^T w.  seed: ybar is the adjoint vector itself, masked to the
// unclamped unknowns (the rows of y_s that are equations).
template <bool IsU>
__device__ __forceinline__ void adj_rev_comp(const Dims& d, const AdjSweep& S, const double* field,
                                             const double* xj, const double* xj1, const double* yb, bool seed,
                                             double* ybn, int t) {
    int i1, j1;
    mom_range<IsU>(d, i1, j1);
    const int i = 1 + t / j1, j = 1 + t % j1;
    const size_t c = at(d, i, j);
    auto Yb = [&](size_t a) -> double { return seed ? yb[a] * (1.0 - S.clamp[a]) : yb[a]; };
    auto W = [&](size_t a) -> double { return Yb(a) / S.aP[a]; };
    const double wc = W(c);
    if (wc != 0.0) {
        S.r0b[c] += wc;
        if (j < j1) S.eb[c] += wc * (xj[c + 1] - field[c + 1]);
        if (j > 1) S.wb[c] += wc * (xj[c - 1] - field[c - 1]);
        if (i < i1) S.nb[c] += wc * (xj[c + d.P] - field[c + d.P]);
        if (i > 1) S.sb[c] += wc * (xj[c - d.P] - field[c - d.P]);
        S.db[c] -= wc * (xj1[c] - field[c]);
    }
    double y = 0.0;
    if (j < j1) y += S.aW[c + 1] * W(c + 1);
    if (j > 1) y += S.aE[c - 1] * W(c - 1);
    if (i < i1) y += S.aS[c + d.P] * W(c + d.P);
    if (i > 1) y += S.aN[c - d.P] * W(c - d.P);
    ybn[c] = y;
}

__global__ void k_adj_rev(KParams k, AdjSweep U, AdjSweep V, const double* u, const double* v, const double* xUj,
                          const double* xUj1, const double* xVj, const double* xVj1, const double* ybU,
                          const double* ybV, double* ybUn, double* ybVn, int doU, int doV, int seedU, int seedV) {
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const int nU = doU ? (M - 1) * (N - 2) : 0, nV = doV ? (M - 2) * (N - 1) : 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nU + nV; t += gridDim.x * blockDim.x) {
        if (t < nU) adj_rev_comp<true>(d, U, u, xUj, xUj1, ybU, seedU != 0, ybUn, t);
        else adj_rev_comp<false>(d, V, v, xVj, xVj1, ybV, seedV != 0, ybVn, t - nU);
    }
}

// Coefficient adjoints of one momentum row scattered to the face velocities
// the coefficients depend on.  aE = De + max(0, -Fe), aW = De + max(0, Fw),
// aN = Dn + max(0, -Fn), aS = Dn + max(0, Fs) (in-set neighbours only; the
// half-cell doubling is constant), aP0 = sum of all four + (Fe - Fw + Fn - Fs)
// + sink + alpha vol, D = aP0 / uvAlpha (momentum_solver.cpp:204-262).
// F are cs rho h times the clamped face averages.
template <bool IsU>
__device__ void adj_coef_row(const AdjCtx& a, int i, int j, const AdjSweep& S, AdjVecs V) {
    const KParams& k = a.k;
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const size_t c = at(d, i, j);
    const double ap0b = S.db[c] / k.uvAlpha;
    int i1, j1;
    mom_range<IsU>(d, i1, j1);
    const bool eIn = j < j1, wIn = j > 1, nIn = i < i1, sIn = i > 1;
    const double mv = a.maxVel;
    const double cs = k.convScale, cE = cs * k.rho * k.hy, cN = cs * k.rho * k.hx;
    const double* u = a.u;
    const double* v = a.v;
    auto uv = [&](int ii, int jj) -> double { return u[at(d, ii, jj)]; };
    auto vv = [&](int ii, int jj) -> double { return v[at(d, ii, jj)]; };
    double xe, xw, xn, xs;
    if (IsU) {
        xe = 0.5 * (uv(i, j) + uv(i, j + 1)); xw = 0.5 * (uv(i, j - 1) + uv(i, j));
        xn = 0.5 * (vv(i, j) + vv(i, j + 1)); xs = 0.5 * (vv(i - 1, j) + vv(i - 1, j + 1));
    } else {
        xe = 0.5 * (uv(i, j) + uv(i + 1, j)); xw = 0.5 * (uv(i, j - 1) + uv(i + 1, j - 1));
        xn = 0.5 * (vv(i, j) + vv(i + 1, j)); xs = 0.5 * (vv(i - 1, j) + vv(i, j));
    }
    const double Fe = cE * dclamp(xe, -mv, mv), Fw = cE * dclamp(xw, -mv, mv);
    const double Fn = cN * dclamp(xn, -mv, mv), Fs = cN * dclamp(xs, -mv, mv);
    const double sE = upw_neg(xe, mv), sW = upw_pos(xw, mv);
    const double sN = upw_neg(xn, mv), sS = upw_pos(xs, mv);
    const double Feb = (eIn ? -S.eb[c] * sE : 0.0) + ap0b * (1.0 - sE);
    const double Fwb = (wIn ? S.wb[c] * sW : 0.0) + ap0b * (sW - 1.0);
    const double Fnb = (nIn ? -S.nb[c] * sN : 0.0) + ap0b * (1.0 - sN);
    const double Fsb = (sIn ? S.sb[c] * sS : 0.0) + ap0b * (sS - 1.0);
    const double gE = 0.5 * cE * clampd(xe, mv) * Feb, gW = 0.5 * cE * clampd(xw, mv) * Fwb;
    const double gN = 0.5 * cN * clampd(xn, mv) * Fnb, gS = 0.5 * cN * clampd(xs, mv) * Fsb;
    auto Uk = [&](int ii, int jj, size_t& cc) -> bool {  // U unknowns; u(i,N-1) is the copy of u(i,N-2)
        if (ii < 1 || ii > M - 1 || jj < 1) return false;
        if (jj == N - 1) jj = N - 2;
        if (jj > N - 2) return false;
        cc = at(d, ii, jj);
        return true;
    };
    auto Vk = [&](int ii, int jj, size_t& cc) -> bool {  // V unknowns; v(i,N) is the copy of v(i,N-1)
        if (ii < 1 || ii > M - 2 || jj < 1) return false;
        if (jj == N) jj = N - 1;
        if (jj > N - 1) return false;
        cc = at(d, ii, jj);
        return true;
    };
    size_t q;
    if (IsU) {
        if (Uk(i, j, q)) adj_add(V.yu, q, gE + gW, true);
        if (Uk(i, j + 1, q)) adj_add(V.yu, q, gE, true);
        if (Uk(i, j - 1, q)) adj_add(V.yu, q, gW, true);
        if (Vk(i, j, q)) adj_add(V.yv, q, gN, true);
        if (Vk(i, j + 1, q)) adj_add(V.yv, q, gN, true);
        if (Vk(i - 1, j, q)) adj_add(V.yv, q, gS, true);
        if (Vk(i - 1, j + 1, q)) adj_add(V.yv, q, gS, true);
    } else {
        if (Uk(i, j, q)) adj_add(V.yu, q, gE, true);
        if (Uk(i + 1, j, q)) adj_add(V.yu, q, gE, true);
        if (Uk(i, j - 1, q)) adj_add(V.yu, q, gW, true);
        if (Uk(i + 1, j - 1, q)) adj_add(V.yu, q, gW, true);
        if (Vk(i, j, q)) adj_add(V.yv, q, gN + gS, true);
        if (Vk(i + 1, j, q)) adj_add(V.yv, q, gN, true);
        if (Vk(i - 1, j, q)) adj_add(V.yv, q, gS, true);
    }
}

// y = J^T lambda (y zeroed by the caller) after the reverse sweeps:
// momentum rows scatter -r0b through the residual's Jacobian (dr0 = -dR),
// their coefficient adjoints through the assembly, and clamped unknowns add
// lambda itself (their rows are u = +-maxVel); continuity rows scatter lambda.
__global__ void k_adj_jt(AdjCtx a, AdjVecs V, AdjSweep Us, AdjSweep Vs) {
    const Dims d = a.k.d;
    const int M = d.M, N = d.N;
    const int nU = (M - 1) * (N - 2), nV = (M - 2) * (N - 1), nC = (M - 1) * (N - 2);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nU + nV + nC; t += gridDim.x * blockDim.x) {
        if (t < nU) {
            const int i = 1 + t / (N - 2), j = 1 + t % (N - 2);
            const size_t c = at(d, i, j);
            adj_row_u(a, i, j, -Us.r0b[c], V, true);
            adj_coef_row<true>(a, i, j, Us, V);
            if (Us.clamp[c] != 0.0) adj_add(V.yu, c, V.lu[c], true);
        } else if (t < nU + nV) {
            const int q = t - nU;
            const int i = 1 + q / (N - 1), j = 1 + q % (N - 1);
            const size_t c = at(d, i, j);
            adj_row_v(a, i, j, -Vs.r0b[c], V, true);
            adj_coef_row<false>(a, i, j, Vs, V);
            if (Vs.clamp[c] != 0.0) adj_add(V.yv, c, V.lv[c], true);
        } else {
            const int q = t - nU - nV;
            const int i = 1 + q / (N - 2), j = 1 + q % (N - 2);
            adj_row_c(a, i, j, V.lc[at(d, i, j)], V, true);
        }
    }
}

// dJ/dX of the full-system pressure drop (one block).  Inlet patch: rows with
// gamma(i-1, 0) pure fluid; static p(i,0) = p(i,1) (ghost copy of an
// unknown), u(i,0) and v(.,0) are boundary constants.  Outlet patch: rows
// with gamma(i-1, N-2) pure fluid; p(i,N) = 0, u(i,N-1) = u(i,N-2),
// v(.,N) = v(.,N-1).  Also returns J (for checks).
__global__ void __launch_bounds__(1024) k_adj_g(AdjCtx a, AdjVecs V, double* Jout) {
    __shared__ double sm[32 * 5];
    const KParams& k = a.k;
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const double rho = k.rho, hy = k.hy;
    // pass 1: sums of the inlet and outlet patches
    double s[5] = {0, 0, 0, 0, 0};  // in: flux, tot*flux ; out: flux, tot*flux, area
    for (int i = 1 + threadIdx.x; i < M; i += blockDim.x) {
        if (a.gamma[at(d, i - 1, 0)] >= 1.0 - 1e-6) {
            const double un = a.u[at(d, i, 0)];
            const double vt = 0.5 * (a.v[at(d, i - 1, 0)] + a.v[at(d, i, 0)]);
            const double fa = fabs(rho * un * hy);
            const double tot = a.p[at(d, i, 0)] + 0.5 * rho * (un * un + vt * vt);
            if (fa > 0.0) { s[0] += fa; s[1] += tot * fa; }
        }
        if (a.gamma[at(d, i - 1, N - 2)] >= 1.0 - 1e-6) {
            const int vtI = i - 1, vbI = (i < M - 1) ? i : M - 1;
            const double un = a.u[at(d, i, N - 1)];
            const double vt = 0.5 * (a.v[at(d, vtI, N)] + a.v[at(d, vbI, N)]);
            const double fa = fabs(rho * un * hy);
            const double tot = a.p[at(d, i, N)] + 0.5 * rho * (un * un + vt * vt);
            if (fa > 0.0) { s[2] += fa; s[3] += tot * fa; }
            s[4] += hy;
        }
    }
    block_sum<5>(s, sm);
    const double inAvg = s[0] > 0.0 ? s[1] / s[0] : 0.0;
    const double outAvg = s[2] > 0.0 ? s[3] / s[2] : 0.0;
    if (threadIdx.x == 0 && Jout) *Jout = inAvg - outAvg;
    // pass 2: derivatives
    for (int i = 1 + threadIdx.x; i < M; i += blockDim.x) {
        if (s[0] > 0.0 && a.gamma[at(d, i - 1, 0)] >= 1.0 - 1e-6) {
            const double un = a.u[at(d, i, 0)];
            const double fa = fabs(rho * un * hy);
            // d inAvg / d p(i,1) (p(i,0) is the ghost copy of p(i,1))
            if (fa > 0.0) V.gp[at(d, i, 1)] += fa / s[0];
        }
        if (s[2] > 0.0 && a.gamma[at(d, i - 1, N - 2)] >= 1.0 - 1e-6) {
            const int vtI = i - 1, vbI = (i < M - 1) ? i : M - 1;
            const double un = a.u[at(d, i, N - 1)];
            const double vt = 0.5 * (a.v[at(d, vtI, N)] + a.v[at(d, vbI, N)]);
            const double fa = fabs(rho * un * hy);
            if (fa > 0.0) {
                const double tot = a.p[at(d, i, N)] + 0.5 * rho * (un * un + vt * vt);
                const double sg = un > 0.0 ? 1.0 : (un < 0.0 ? -1.0 : 0.0);
                // d outAvg / d un and / d vt; J = in - out
                const double dun = (rho * un * fa + (tot - outAvg) * rho * hy * sg) / s[2];
                const double dvt = rho * vt * fa / s[2];
                // un = u(i,N-1) = u(i,N-2) (outlet copy)
                atomicAdd(V.gu + at(d, i, N - 2), -dun);
                // vt = (v(i-1,N) + v(i,N)) / 2 = (v(i-1,N-1) + v(i,N-1)) / 2; walls are constants
                if (vtI >= 1 && vtI <= M - 2) atomicAdd(V.gv + at(d, vtI, N - 1), -0.5 * dvt);
                if (vbI >= 1 && vbI <= M - 2) atomicAdd(V.gv + at(d, vbI, N - 1), -0.5 * dvt);
            }
        }
    }
}

// r = gs g - ys y on all unknowns; partial sums of r^2 and g^2 per block
// into part[b*2].  (gs, ys) = (1, 1): the adjoint residual; (0, -1): the
// product y = J^T z restricted to the unknowns.
__global__ void k_adj_defect(KParams k, AdjVecs V, double gs, double ys, double* ru, double* rv, double* rp,
                             double* part) {
    __shared__ double sm[64];
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const int nU = (M - 1) * (N - 2), nV = (M - 2) * (N - 1), nP = (M - 1) * (N - 2);
    double acc[2] = {0.0, 0.0};
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nU + nV + nP; t += gridDim.x * blockDim.x) {
        if (t < nU) {
            const size_t c = at(d, 1 + t / (N - 2), 1 + t % (N - 2));
            const double r = gs * V.gu[c] - ys * V.yu[c];
            ru[c] = r; acc[0] += r * r; acc[1] += V.gu[c] * V.gu[c];
        } else if (t < nU + nV) {
            const int q = t - nU;
            const size_t c = at(d, 1 + q / (N - 1), 1 + q % (N - 1));
            const double r = gs * V.gv[c] - ys * V.yv[c];
            rv[c] = r; acc[0] += r * r; acc[1] += V.gv[c] * V.gv[c];
        } else {
            const int q = t - nU - nV;
            const size_t c = at(d, 1 + q / (N - 2), 1 + q % (N - 2));
            const double r = gs * V.gp[c] - ys * V.yp[c];
            rp[c] = r; acc[0] += r * r; acc[1] += V.gp[c] * V.gp[c];
        }
    }
    block_sum<2>(acc, sm);
    if (threadIdx.x == 0) { part[2 * blockIdx.x] = acc[0]; part[2 * blockIdx.x + 1] = acc[1]; }
}

// Momentum part of the preconditioner: z = -r on the unclamped momentum
// unknowns (F_u is a Jacobi-preconditioned residual, dF_u/du ~ -I) and
// z = r on clamped ones (identity rows); zd = r / D on the unclamped
// unknowns and 0 on clamped ones, the input of the pressure-like rhs.
__global__ void k_adj_prec_mom(KParams k, const double* ru, const double* rv, AdjSweep Us, AdjSweep Vs, double* zu,
                               double* zv, double* zdu, double* zdv) {
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const int nU = (M - 1) * (N - 2), nV = (M - 2) * (N - 1);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nU + nV; t += gridDim.x * blockDim.x) {
        const bool isU = t < nU;
        const int q = isU ? t : t - nU;
        const int w = isU ? N - 2 : N - 1;
        const size_t c = at(d, 1 + q / w, 1 + q % w);
        const AdjSweep& S = isU ? Us : Vs;
        const double r = (isU ? ru : rv)[c];
        const bool cl = S.clamp[c] != 0.0;
        (isU ? zu : zv)[c] = cl ? r : -r;
        (isU ? zdu : zdv)[c] = cl ? 0.0 : r / S.aP[c];
    }
}

// dE' = uvAlpha dE, dN' = uvAlpha dN with the clamped faces set to 0: the
// pressure-like operator of the preconditioner in the forward PCG's form
__global__ void k_adj_prec_faces(KParams k, const double* dE, const double* dN, AdjSweep Us, AdjSweep Vs,
                                 double* dEp, double* dNp) {
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const int nU = (M - 1) * (N - 2), nV = (M - 2) * (N - 1);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nU + nV; t += gridDim.x * blockDim.x) {
        const bool isU = t < nU;
        const int q = isU ? t : t - nU;
        const int w = isU ? N - 2 : N - 1;
        const size_t c = at(d, 1 + q / w, 1 + q % w);
        if (isU) dEp[c] = Us.clamp[c] != 0.0 ? 0.0 : k.uvAlpha * dE[c];
        else dNp[c] = Vs.clamp[c] != 0.0 ? 0.0 : k.uvAlpha * dN[c];
    }
}

// rhs of the pressure-like correction: G^T dm* - r_p, with
// (G^T dm)(i,j) = hy (du(i,j-1) - du(i,j)) + hx (dv(i-1,j) - dv(i,j));
// written into the PCG rhs (TV) on the pressure unknowns.
template <typename TV>
__global__ void k_adj_prhs(KParams k, const double* du, const double* dv, const double* rp, TV* rhs) {
    const Dims d = k.d;
    const int M = d.M, N = d.N, w = N - 2;
    const int n = (M - 1) * w;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int i = 1 + t / w, j = 1 + t % w;
        const size_t c = at(d, i, j);
        const double uw = (j > 1) ? du[c - 1] : 0.0;
        const double vs = (i > 1) ? dv[c - d.P] : 0.0;
        const double vn = (i <= M - 2) ? dv[c] : 0.0;
        rhs[c] = (TV)(k.hy * (uw - du[c]) + k.hx * (vs - vn) - rp[c]);
    }
}

// corrections after the pressure-like solve: on unclamped momentum unknowns
// z += (dR_c/dX)^T dc, i.e. u(i,j) += rho hy (dc(i,j+1) - dc(i,j)) and
// v(i,j) += rho hx (dc(i+1,j) - dc(i,j)) (dc zero outside the pressure
// unknowns); clamped unknowns keep z; the continuity part is dc
__global__ void k_adj_update(KParams k, const double* zu, const double* zv, const double* dc, AdjSweep Us,
                             AdjSweep Vs, double* ou, double* ov, double* oc) {
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const int nU = (M - 1) * (N - 2), nV = (M - 2) * (N - 1), nP = (M - 1) * (N - 2);
    auto C = [&](int i, int j) -> double {
        if (i < 1 || i > M - 1 || j < 1 || j > N - 2) return 0.0;
        return dc[at(d, i, j)];
    };
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nU + nV + nP; t += gridDim.x * blockDim.x) {
        if (t < nU) {
            const int i = 1 + t / (N - 2), j = 1 + t % (N - 2);
            const size_t c = at(d, i, j);
            ou[c] = zu[c] + (Us.clamp[c] != 0.0 ? 0.0 : k.rho * k.hy * (C(i, j + 1) - C(i, j)));
        } else if (t < nU + nV) {
            const int q = t - nU;
            const int i = 1 + q / (N - 1), j = 1 + q % (N - 1);
            const size_t c = at(d, i, j);
            ov[c] = zv[c] + (Vs.clamp[c] != 0.0 ? 0.0 : k.rho * k.hx * (C(i + 1, j) - C(i, j)));
        } else {
            const int q = t - nU - nV;
            const int i = 1 + q / (N - 2), j = 1 + q % (N - 2);
            oc[at(d, i, j)] = dc[at(d, i, j)];
        }
    }
}

// ---------------------------------------------------------------- Krylov vectors
// A Krylov vector is three field-layout arrays (U, V, continuity) stored
// back to back, L = 3 * nElem doubles; entries off the unknowns stay zero.
constexpr int kKryMaxDots = 32;

// part[b * 32 + q] = block b's share of <w, B_q>, q < nv, B_q = B + q L
// a block's partial sums of the nv per-thread accumulators (warp shuffles,
// then warps in order) into part[block * 32 + q]
__device__ __forceinline__ void kry_block_partials(const double (&acc)[kKryMaxDots], int nv, double* part) {
    __shared__ double sm[8][kKryMaxDots];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < kKryMaxDots; ++q) {
        if (q < nv) {
            double v = acc[q];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) sm[wid][q] = v;
        }
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double v = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) v += sm[q][threadIdx.x];
        part[(size_t)blockIdx.x * kKryMaxDots + threadIdx.x] = v;
    }
}

__global__ void __launch_bounds__(256) k_kry_mdot(const double* __restrict__ w, const double* __restrict__ B,
                                                  size_t L, int nv, double* part) {
    double acc[kKryMaxDots];
#pragma unroll
    for (int q = 0; q < kKryMaxDots; ++q) acc[q] = 0.0;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < L; t += (size_t)gridDim.x * blockDim.x) {
        const double wt = w[t];
#pragma unroll
        for (int q = 0; q < kKryMaxDots; ++q)
            if (q < nv) acc[q] += B[q * L + t] * wt;
    }
    kry_block_partials(acc, nv, part);
}

// w += sign * sum_q h[q] B_q (k_kry_axpy), then the partials of the updated
// w against B_0 .. B_nd-1, or (selfDot) of its squared norm (k_kry_mdot on
// the new w): one pass over B and w instead of two, with the per-thread
// element order and the block reduction of the two kernels it replaces.
__global__ void __launch_bounds__(256) k_kry_axpy_mdot(double* __restrict__ w, const double* __restrict__ B,
                                                       size_t L, int nv, const double* __restrict__ h, double sign,
                                                       int nd, int selfDot, double* part) {
    __shared__ double hs[kKryMaxDots];
    if (threadIdx.x < nv) hs[threadIdx.x] = sign * h[threadIdx.x];
    __syncthreads();
    double acc[kKryMaxDots];
#pragma unroll
    for (int q = 0; q < kKryMaxDots; ++q) acc[q] = 0.0;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < L; t += (size_t)gridDim.x * blockDim.x) {
        double a = w[t];
        for (int q = 0; q < nv; ++q) a += hs[q] * B[q * L + t];
        w[t] = a;
        if (selfDot) {
            acc[0] += a * a;
        } else {
#pragma unroll
            for (int q = 0; q < kKryMaxDots; ++q)
                if (q < nd) acc[q] += B[q * L + t] * a;
        }
    }
    kry_block_partials(acc, selfDot ? 1 : nd, part);
}

// out[q] = sum over blocks of part[b * 32 + q]; one block of 32 warps, warp q
// sums entry q in a fixed order
__global__ void __launch_bounds__(1024) k_kry_sum(const double* part, int nb, int nv, double* out) {
    const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (q >= nv) return;
    double v = 0.0;
    for (int b = lane; b < nb; b += 32) v += part[(size_t)b * kKryMaxDots + q];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) out[q] = v;
}

// w += sign * sum_q h[q] B_q
__global__ void __launch_bounds__(256) k_kry_axpy(double* __restrict__ w, const double* __restrict__ B, size_t L,
                                                  int nv, const double* __restrict__ h, double sign) {
    __shared__ double hs[kKryMaxDots];
    if (threadIdx.x < nv) hs[threadIdx.x] = sign * h[threadIdx.x];
    __syncthreads();
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < L; t += (size_t)gridDim.x * blockDim.x) {
        double a = w[t];
        for (int q = 0; q < nv; ++q) a += hs[q] * B[q * L + t];
        w[t] = a;
    }
}

// dst = s * src
__global__ void k_kry_scale(double* dst, const double* src, size_t L, double s) {
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < L; t += (size_t)gridDim.x * blockDim.x)
        dst[t] = s * src[t];
}

// dJ/dgamma(cell a, b) = -sum over the faces the cell touches of
// abar_face * 0.5 * alpha'(gamma(a,b)), where abar_face is the adjoint of the
// face's alpha_face: it enters r0 as -alpha_face vol x_face (the Brinkman
// term of R) and D = aP0 / uvAlpha as alpha_face vol / uvAlpha; cells Ny x Nx.
__global__ void k_adj_grad(AdjCtx a, AdjSweep Us, AdjSweep Vs, double alphaMax, double q, double* grad) {
    const KParams& k = a.k;
    const Dims d = k.d;
    const int M = d.M, N = d.N, Ny = M - 1, Nx = N - 1;
    const double vol = k.hx * k.hy, ia = 1.0 / k.uvAlpha;
    auto abU = [&](size_t c) -> double { return vol * (Us.db[c] * ia - a.u[c] * Us.r0b[c]); };
    auto abV = [&](size_t c) -> double { return vol * (Vs.db[c] * ia - a.v[c] * Vs.r0b[c]); };
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < Ny * Nx; t += gridDim.x * blockDim.x) {
        const int ca = t / Nx, cb = t % Nx;
        const double g = a.gamma[at(d, ca, cb)];
        const double den = 1.0 + q * g + 1e-10;
        const double dalpha = -alphaMax * (den + (1.0 - g) * q) / (den * den);
        double s = 0.0;
        // U faces (i, j) with i-1 = ca and j-1 = cb (left cell) or j = cb (right cell); j in [1, N-2]
        const int iu = ca + 1;
        if (iu >= 1 && iu <= M - 1) {
            if (cb + 1 <= N - 2) s += abU(at(d, iu, cb + 1));
            if (cb >= 1 && cb <= N - 2) s += abU(at(d, iu, cb));
        }
        // V faces (i, j) with j-1 = cb and i-1 = ca (top cell) or i = ca (bottom cell); i in [1, M-2]
        const int jv = cb + 1;
        if (jv >= 1 && jv <= N - 1) {
            if (ca + 1 <= M - 2) s += abV(at(d, ca + 1, jv));
            if (ca >= 1 && ca <= M - 2) s += abV(at(d, ca, jv));
        }
        grad[t] = -s * 0.5 * dalpha;
    }
}

// ---------------------------------------------------------------- equations model
// The adjoint of the discretisation R(X) = 0 itself: exact at a state with no
// velocity on the clamp (there the fixed point of the iteration satisfies
// R = 0, whatever the sweep count), the model for states that are not fixed
// points of the iteration, and the one whose preconditioner (Jacobi sweeps on
// the transposed Picard momentum matrix, then the pressure-like correction
// with the forward pressure matrix) converges robustly.

// Equations model: y = J_R^T lambda (y zeroed by the caller); with resid != nullptr also the
// residuals R(X) per row (U, V, C in the field layout).
__global__ void k_adj_jt_eq(AdjCtx a, AdjVecs V, double* rU, double* rV, double* rC) {
    const Dims d = a.k.d;
    const int M = d.M, N = d.N;
    const int nU = (M - 1) * (N - 2), nV = (M - 2) * (N - 1), nC = (M - 1) * (N - 2);
    const bool scatter = (rU == nullptr);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nU + nV + nC; t += gridDim.x * blockDim.x) {
        if (t < nU) {
            const int i = 1 + t / (N - 2), j = 1 + t % (N - 2);
            const double R = adj_row_u(a, i, j, scatter ? V.lu[at(d, i, j)] : 0.0, V, scatter);
            if (!scatter) rU[at(d, i, j)] = R;
        } else if (t < nU + nV) {
            const int q = t - nU;
            const int i = 1 + q / (N - 1), j = 1 + q % (N - 1);
            const double R = adj_row_v(a, i, j, scatter ? V.lv[at(d, i, j)] : 0.0, V, scatter);
            if (!scatter) rV[at(d, i, j)] = R;
        } else {
            const int q = t - nU - nV;
            const int i = 1 + q / (N - 2), j = 1 + q % (N - 2);
            const double R = adj_row_c(a, i, j, scatter ? V.lc[at(d, i, j)] : 0.0, V, scatter);
            if (!scatter) rC[at(d, i, j)] = R;
        }
    }
}

// Equations model: one Jacobi sweep of the transposed, relaxed Picard momentum system for U
// and V: (A_P^T x)(i,j) = aP x(i,j) - aW(i,j+1) x(i,j+1) - aE(i,j-1) x(i,j-1)
// - aS(i+1,j) x(i+1,j) - aN(i-1,j) x(i-1,j) with the masked coefficients of
// the converged assembly (aP = aP0 / uvAlpha).  first: x = 0.
__global__ void k_adj_jacobi_t(KParams k, MomSys<double> Us, MomSys<double> Vs, const double* ru,
                               const double* rv, const double* xu, const double* xv, double* yu, double* yv,
                               int first) {
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const int nU = (M - 1) * (N - 2), nV = (M - 2) * (N - 1);
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nU + nV; t += gridDim.x * blockDim.x) {
        const bool isU = t < nU;
        const int q = isU ? t : t - nU;
        const int w = isU ? N - 2 : N - 1;
        const int i = 1 + q / w, j = 1 + q % w;
        const size_t c = at(d, i, j);
        const MomSys<double>& S = isU ? Us : Vs;
        const double* x = isU ? xu : xv;
        const double* r = isU ? ru : rv;
        double Ax = 0.0;
        if (!first) {
            Ax = S.aP[c] * x[c] - S.aW[c + 1] * x[c + 1] - S.aE[c - 1] * x[c - 1] - S.aS[c + d.P] * x[c + d.P] -
                 S.aN[c - d.P] * x[c - d.P];
        }
        const double xn = (first ? 0.0 : x[c]) + (r[c] - Ax) / S.aP[c];
        (isU ? yu : yv)[c] = xn;
    }
}

// Equations model, corrections: dm = dm* - D_A^-1 D^T dc with (D_A^-1 D^T dc)_u(i,j) =
// rho dE(i,j) (dc(i,j+1) - dc(i,j)) and for v rho dN(i,j) (dc(i+1,j) - dc(i,j))
// (dc zero outside the pressure unknowns); out = (dm, pAlpha dc) on the
// U / V / continuity unknowns
__global__ void k_adj_update_eq(KParams k, const double* du, const double* dv, const double* dc, const double* dE,
                             const double* dN, double relaxC, double* ou, double* ov, double* oc) {
    const Dims d = k.d;
    const int M = d.M, N = d.N;
    const int nU = (M - 1) * (N - 2), nV = (M - 2) * (N - 1), nP = (M - 1) * (N - 2);
    auto C = [&](int i, int j) -> double {
        if (i < 1 || i > M - 1 || j < 1 || j > N - 2) return 0.0;
        return dc[at(d, i, j)];
    };
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nU + nV + nP; t += gridDim.x * blockDim.x) {
        if (t < nU) {
            const int i = 1 + t / (N - 2), j = 1 + t % (N - 2);
            const size_t c = at(d, i, j);
            ou[c] = du[c] - k.rho * dE[c] * (C(i, j + 1) - C(i, j));
        } else if (t < nU + nV) {
            const int q = t - nU;
            const int i = 1 + q / (N - 1), j = 1 + q % (N - 1);
            const size_t c = at(d, i, j);
            ov[c] = dv[c] - k.rho * dN[c] * (C(i + 1, j) - C(i, j));
        } else {
            const int q = t - nU - nV;
            const int i = 1 + q / (N - 2), j = 1 + q % (N - 2);
            oc[at(d, i, j)] = relaxC * dc[at(d, i, j)];
        }
    }
}

// Equations model: dJ/dgamma(cell a, b) = -sum over the faces the cell touches of
// lambda_face * vol * vel_face * 0.5 * alpha'(gamma(a,b)); cells Ny x Nx.
__global__ void k_adj_grad_eq(AdjCtx a, AdjVecs V, double alphaMax, double q, double* grad) {
    const KParams& k = a.k;
    const Dims d = k.d;
    const int M = d.M, N = d.N, Ny = M - 1, Nx = N - 1;
    const double vol = k.hx * k.hy;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < Ny * Nx; t += gridDim.x * blockDim.x) {
        const int ca = t / Nx, cb = t % Nx;
        const double g = a.gamma[at(d, ca, cb)];
        const double den = 1.0 + q * g + 1e-10;
        const double dalpha = -alphaMax * (den + (1.0 - g) * q) / (den * den);
        double s = 0.0;
        // U faces (i, j) with i-1 = ca and j-1 = cb (left cell) or j = cb (right cell); j in [1, N-2]
        const int iu = ca + 1;
        if (iu >= 1 && iu <= M - 1) {
            if (cb + 1 <= N - 2) s += V.lu[at(d, iu, cb + 1)] * a.u[at(d, iu, cb + 1)];
            if (cb >= 1 && cb <= N - 2) s += V.lu[at(d, iu, cb)] * a.u[at(d, iu, cb)];
        }
        // V faces (i, j) with j-1 = cb and i-1 = ca (top cell) or i = ca (bottom cell); i in [1, M-2]
        const int jv = cb + 1;
        if (jv >= 1 && jv <= N - 1) {
            if (ca + 1 <= M - 2) s += V.lv[at(d, ca + 1, jv)] * a.v[at(d, ca + 1, jv)];
            if (ca >= 1 && ca <= M - 2) s += V.lv[at(d, ca, jv)] * a.v[at(d, ca, jv)];
        }
        grad[t] = -s * vol * 0.5 * dalpha;
    }
}

}  // namespace cp
