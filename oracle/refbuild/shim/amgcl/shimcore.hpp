// Minimal stand-in for the part of the AMGCL API (github.com/ddemidov/amgcl,
// not vendored with the reference) that the reference's thermal solver names
// (ThermalSolver/thermal_solver.cpp:77-84, 533-553).  Written here from that
// call site; it is not AMGCL.  Test infrastructure only: it lets the
// reference's own assembly run, then solves the assembled system itself with
// a Jacobi-preconditioned BiCGStab to a tight tolerance (the requested
// tolerance is raised to 1e-14 so that the result pins the discretisation),
// and, when CP_AMGCL_SHIM_DUMP names a file, writes n, the CSR matrix, b and
// the solution there (int32 n, nnz; int32 row_ptr, col_idx; float64 values,
// b, x).
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <tuple>
#include <vector>

namespace amgcl {
namespace backend {
template <class T>
struct builtin {
    struct params {};
};
template <class T>
struct crs {
    int n = 0;
    std::vector<int> ptr, col;
    std::vector<T> val;
    crs(int nr, int nc, const std::vector<int>& p, const std::vector<int>& c, const std::vector<T>& v)
        : n(nr), ptr(p), col(c), val(v) { (void)nc; }
};
}  // namespace backend
namespace coarsening { struct smoothed_aggregation {}; }
namespace relaxation { struct spai0 {}; struct ilu0 {}; }
template <class Backend, class Coarsening, class Relax>
struct amg {
    struct params { bool allow_rebuild = false; };
};
namespace solver {
struct common_params {
    int s = 4;
    bool smoothing = false;
    double tol = 1e-8;
    double abstol = 0.0;
    int maxiter = 100;
};
template <class B> struct idrs { typedef common_params params; };
template <class B> struct bicgstab { typedef common_params params; };
template <class B> struct cg { typedef common_params params; };
}  // namespace solver

template <class Precond, class Solver>
class make_solver {
public:
    struct params {
        typename Precond::params precond;
        typename Solver::params solver;
    };
    make_solver(std::shared_ptr<backend::crs<double>> A, const params& prm) : A_(A), prm_(prm) {}

    std::tuple<int, double> operator()(const std::vector<double>& b, std::vector<double>& x) const {
        const backend::crs<double>& A = *A_;
        const int n = A.n;
        std::vector<double> dinv(n, 1.0);
        for (int r = 0; r < n; ++r)
            for (int q = A.ptr[r]; q < A.ptr[r + 1]; ++q)
                if (A.col[q] == r && A.val[q] != 0.0) dinv[r] = 1.0 / A.val[q];
        auto mv = [&](const std::vector<double>& v, std::vector<double>& out) {
            for (int r = 0; r < n; ++r) {
                double s = 0.0;
                for (int q = A.ptr[r]; q < A.ptr[r + 1]; ++q) s += A.val[q] * v[A.col[q]];
                out[r] = s;
            }
        };
        auto dot = [&](const std::vector<double>& a, const std::vector<double>& c) {
            double s = 0.0;
            for (int r = 0; r < n; ++r) s += a[r] * c[r];
            return s;
        };
        if ((int)x.size() != n) x.assign(n, 0.0);
        std::vector<double> r(n), rh(n), p(n, 0.0), v(n, 0.0), s(n), t(n), ph(n), sh(n);
        mv(x, t);
        for (int q = 0; q < n; ++q) r[q] = b[q] - t[q];
        rh = r;
        const double bn = std::sqrt(dot(b, b)) > 0 ? std::sqrt(dot(b, b)) : 1.0;
        double rho = 1.0, alpha = 1.0, omega = 1.0, res = std::sqrt(dot(r, r)) / bn;
        int it = 0;
        const double tol = 1e-14;
        for (; it < 200000 && res > tol; ++it) {
            const double rho1 = dot(rh, r);
            if (rho1 == 0.0) break;
            const double beta = (rho1 / rho) * (alpha / omega);
            for (int q = 0; q < n; ++q) p[q] = r[q] + beta * (p[q] - omega * v[q]);
            for (int q = 0; q < n; ++q) ph[q] = dinv[q] * p[q];
            mv(ph, v);
            alpha = rho1 / dot(rh, v);
            for (int q = 0; q < n; ++q) s[q] = r[q] - alpha * v[q];
            for (int q = 0; q < n; ++q) sh[q] = dinv[q] * s[q];
            mv(sh, t);
            const double tt = dot(t, t);
            omega = tt > 0 ? dot(t, s) / tt : 0.0;
            for (int q = 0; q < n; ++q) x[q] += alpha * ph[q] + omega * sh[q];
            for (int q = 0; q < n; ++q) r[q] = s[q] - omega * t[q];
            rho = rho1;
            res = std::sqrt(dot(r, r)) / bn;
            if (omega == 0.0) break;
        }
        if (const char* path = std::getenv("CP_AMGCL_SHIM_DUMP")) {
            if (FILE* f = std::fopen(path, "wb")) {
                const int nnz = (int)A.val.size();
                std::fwrite(&n, sizeof(int), 1, f);
                std::fwrite(&nnz, sizeof(int), 1, f);
                std::fwrite(A.ptr.data(), sizeof(int), n + 1, f);
                std::fwrite(A.col.data(), sizeof(int), nnz, f);
                std::fwrite(A.val.data(), sizeof(double), nnz, f);
                std::fwrite(b.data(), sizeof(double), n, f);
                std::fwrite(x.data(), sizeof(double), n, f);
                std::fclose(f);
            }
        }
        (void)prm_;
        return std::make_tuple(it, res);
    }

private:
    std::shared_ptr<backend::crs<double>> A_;
    params prm_;
};
}  // namespace amgcl
