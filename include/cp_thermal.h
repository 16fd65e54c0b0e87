/* C ABI of the B200 3-D conjugate-heat-transfer solve (the reference's
 * ThermalSolver/thermal_solver.cpp, which assembles a 7-point finite-volume
 * system and solves it with AMGCL's IDR(s)).  Every call returns a
 * cp_status (include/cp_simple.h); cp_last_error_string() explains it.
 *
 * Grid: Nx x Ny cells in the plane (the CFD's cropped thermal domain) and
 * Nz = nz_solid + nz_fluid layers (k = 0 the bottom of the base plate,
 * Nz <= 16; the reference's default is 9);
 * temperatures are indexed k * Nx * Ny + j * Nx + i as in the reference. */
#ifndef CP_THERMAL_H
#define CP_THERMAL_H

#include "cp_simple.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Parameters, names and defaults of struct Params (thermal_solver.cpp:148-200);
 * dx, dy are the cell sizes (the reference's thermal_params.txt). */
typedef struct cp_thermal_params {
    int Nx, Ny, nz_solid, nz_fluid;
    double dx, dy, H_b, H_t;
    double k_s, k_f, rho, Cp, T_inlet;
    double rtol;           /* stop when ||b - A T|| <= rtol ||b|| (AMGCL's test)   */
    int maxiter;
    int k_interp_mode;     /* 0 linear, 1 RAMP, 2 harmonic (thermal_solver.cpp:267-295) */
    double qk;             /* RAMP parameter                                        */
    int precision;         /* cp_precision: CP_PREC_FP64 (default) or CP_PREC_MIXED,
                              a float V-cycle inside the FP64 BiCGStab; the solve is
                              restarted from its iterate while the FP64 residual
                              b - A T is above rtol (at most 4 launches)           */
} cp_thermal_params;

typedef struct cp_thermal cp_thermal;

typedef struct cp_thermal_report {
    int iterations;        /* BiCGStab iterations                  */
    int converged;         /* 1 if rtol was reached                */
    double residual;       /* final ||b - A T|| / ||b||            */
    double device_ms;      /* assembly + factorisation + solve     */
} cp_thermal_report;

void cp_thermal_params_default(cp_thermal_params* p);
cp_status cp_thermal_create(const cp_thermal_params* p, cp_thermal** out);
cp_status cp_thermal_destroy(cp_thermal* th);
/* gamma (1 fluid .. 0 solid), cell-centred velocities u_xy, v_xy [m/s] and the
 * bottom heat flux q0 [W/m^2]: Ny x Nx each, row-major, host memory.  The
 * reference reads them from geometry_thermal.txt (as 1 - gamma),
 * u_thermal.txt, v_thermal.txt and power_map.txt (W/cm^2) or a uniform qf. */
cp_status cp_thermal_set_inputs(cp_thermal* th, const double* gamma, const double* u_xy, const double* v_xy,
                                const double* q0);
/* Assembles the system (thermal_solver.cpp:417-520) and solves it from
 * T = T_inlet with BiCGStab right-preconditioned by one V-cycle of 2 x 2
 * column aggregates with z-line smoothing (the reference: AMGCL IDR(8) with
 * smoothed-aggregation AMG, thermal_solver.cpp:534-553). */
cp_status cp_thermal_solve(cp_thermal* th, cp_thermal_report* rep);
/* T: Nz * Ny * Nx doubles (host) */
cp_status cp_thermal_get_T(cp_thermal* th, double* T);
/* The bottom-layer maximum and p-norm (mean of T^p)^(1/p)
 * (thermal_solver.cpp:346-386) of the current solution. */
cp_status cp_thermal_objective(cp_thermal* th, double p, double* Tb_max, double* Tb_pnorm);
/* The discrete adjoint of the p-norm objective: J = Tb_pnorm of the current
 * solution and dJ_dgamma (Ny x Nx, host) = dJ/dgamma of every plane cell,
 * from one solve of A^T lambda = dJ/dT (same solver, rtol and maxiter) with
 * the velocities and the fluid/solid masks held fixed.  The reference's
 * sensitivity (compute_optimization_results, thermal_solver.cpp:361-386;
 * the ThermalAdjointSolver stub, thermal_adjoint.cpp:16-64) is a placeholder
 * of zeros; its dk_dgamma (thermal_solver.cpp:317-321) is used here.  rep
 * describes the adjoint solve. */
cp_status cp_thermal_pnorm_gradient(cp_thermal* th, double p, double* J, double* dJ_dgamma, cp_thermal_report* rep);

#ifdef __cplusplus
}
#endif

#endif /* CP_THERMAL_H */
