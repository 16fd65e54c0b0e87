// Drop-in replacement of the reference's Utilities/iterations.cpp
// (Carloossgg/coldplate-solver): SIMPLE::calculateStep (iterations.cpp:82)
// runs one outer SIMPLE iteration on the GPU through libcoldplate.so
// (include/cp_simple.h) instead of the Eigen/OpenMP code.
//
// Build it in place of iterations.cpp together with the reference's other
// sources and link libcoldplate.so; SIMPLE.h, SIMPLE.cpp and the rest of the
// reference stay unchanged.  SIMPLE::runIterations (SIMPLE.cpp:310-528)
// keeps its host loop: its inlet ramp, pressure-drop sampling on the host
// fields (SIMPLE.cpp:423-432), ΔP-window stop rule (:449-491), logs and
// outputs all work as before, because every call copies u, v and p back into
// the SIMPLE object's matrices after the iteration.
//
// Per SIMPLE object, the first call creates a device context from the
// object's public parameters, its cellType and its current u, v, p (the
// initial fields, or a restart read by reuseInitialFields).  The device runs
// no stop rule of its own: the host loop decides.  The arithmetic is FP64
// (the reference algorithm re-typed); CP_PRECISION=mixed selects FP32 inner
// solves with FP64 fields and reductions.  The residual members (residU ...
// residMass_max, the RMS normalisation references) are filled as the
// reference's calculateStep fills them (iterations.cpp:496-659).
//
// Cost of the drop-in form: three host copies per iteration (u, v, p), which
// the caller's own loop needs.  A driver that samples on the device can call
// cp_step / cp_run directly and read fields only when it saves them.
#include "SIMPLE.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <vector>

#include "cp_simple.h"

namespace {

std::map<const SIMPLE*, cp_ctx*> g_contexts;

void cp_or_exit(cp_status s, const char* what) {
    if (s == CP_OK) return;
    std::cerr << "libcoldplate: " << what << " failed: " << cp_status_string(s) << ": " << cp_last_error_string()
              << std::endl;
    std::exit(1);
}

// Eigen matrix (any scalar, column-major) <-> the C ABI's strided doubles
template <class Mat>
void upload(cp_ctx* c, cp_field f, const Mat& m) {
    const long R = m.rows(), C = m.cols();
    std::vector<double> buf((size_t)(R * C));
    for (long j = 0; j < C; ++j)
        for (long i = 0; i < R; ++i) buf[(size_t)(i + j * R)] = (double)m(i, j);
    cp_or_exit(cp_set_field(c, f, buf.data(), R, C, 1, R), "cp_set_field");
}

template <class Mat>
void download(cp_ctx* c, cp_field f, Mat& m) {
    const long R = m.rows(), C = m.cols();
    std::vector<double> buf((size_t)(R * C));
    cp_or_exit(cp_get_field(c, f, buf.data(), R, C, 1, R), "cp_get_field");
    using Scalar = typename std::decay<decltype(m(0, 0))>::type;
    for (long j = 0; j < C; ++j)
        for (long i = 0; i < R; ++i) m(i, j) = (Scalar)buf[(size_t)(i + j * R)];
}

cp_ctx* context_for(SIMPLE& s) {
    auto it = g_contexts.find(&s);
    if (it != g_contexts.end()) return it->second;
    cp_params p;
    cp_params_default(&p);
    p.Ny = s.M - 1;
    p.Nx = s.N - 1;                                     // SIMPLE.cpp:53-54
    p.hy = s.hy; p.hx = s.hx; p.targetVel = s.targetVel; p.Ht_channel = s.Ht_channel;
    p.N_in_buffer = s.N_in_buffer; p.N_out_buffer = s.N_out_buffer;
    // the host loop applies epsilon, maxIterations and the ΔP window
    p.epsilon = -1.0;
    p.maxIterations = std::max(s.maxIterations, 1) + 1;
    p.historyCapacity = p.maxIterations;
    p.usePressureDropConvergence = 0;
    p.xPlaneCoreInlet = s.xPlaneCoreInlet; p.xPlaneCoreOutlet = s.xPlaneCoreOutlet;
    p.pressureSolverType = s.pressureSolverType; p.maxPressureIter = s.maxPressureIter; p.pTol = s.pTol;
    p.momentumSolverType = s.momentumSolverType; p.momentumTol = s.momentumTol;
    p.maxMomentumIter = s.maxMomentumIter;
    p.convectionScheme = s.convectionScheme;
    p.enableTwoPointFiveD = s.enableTwoPointFiveD ? 1 : 0;
    p.twoPointFiveDConvectionFactor = s.twoPointFiveDConvectionFactor;
    p.twoPointFiveDSinkMultiplier = s.twoPointFiveDSinkMultiplier;
    p.brinkmanKMin = s.brinkmanKMin; p.brinkmanQ = s.brinkmanQ;
    p.rho = s.rho; p.eta = s.eta;
    p.enableInletRamp = s.enableInletRamp ? 1 : 0; p.rampSteps = s.rampSteps;
    p.uvAlpha = s.uvAlpha; p.pAlpha = s.pAlpha;
    p.enableNormalizedResiduals = s.enableNormalizedResiduals ? 1 : 0;
    p.residNormFloorVel = s.residNormFloorVel; p.residNormFloorMass = s.residNormFloorMass;
    const char* prec = std::getenv("CP_PRECISION");
    p.precision = (prec && std::strcmp(prec, "mixed") == 0) ? CP_PREC_MIXED : CP_PREC_FP64;
    cp_ctx* c = nullptr;
    cp_or_exit(cp_create(&p, &c), "cp_create");
    // geometry: the physical (M-1) x (N-1) block of cellType (SIMPLE.cpp:633-690)
    const long Ny = s.M - 1, Nx = s.N - 1;
    std::vector<double> ct((size_t)(Ny * Nx));
    for (long i = 0; i < Ny; ++i)
        for (long j = 0; j < Nx; ++j) ct[(size_t)(i * Nx + j)] = (double)s.cellType(i, j);
    cp_or_exit(cp_set_cell_type(c, ct.data(), Ny, Nx, Nx, 1), "cp_set_cell_type");
    upload(c, CP_FIELD_U, s.u);
    upload(c, CP_FIELD_V, s.v);
    upload(c, CP_FIELD_P, s.p);
    g_contexts[&s] = c;
    return c;
}

}  // namespace

float SIMPLE::calculateStep(int& pressureIterations) {
    cp_ctx* c = context_for(*this);
    cp_iter_report r;
    cp_or_exit(cp_step(c, 1, &r), "cp_step");
    download(c, CP_FIELD_U, u);
    download(c, CP_FIELD_V, v);
    download(c, CP_FIELD_P, p);
    pressureIterations = r.pressureIterations;
    residU_max = (float)r.residU_max; residV_max = (float)r.residV_max; residMass_max = (float)r.residMass_max;
    residU_RMS = (float)r.residU_RMS; residV_RMS = (float)r.residV_RMS; residMass_RMS = (float)r.residMass_RMS;
    // RMS normalisation references and the reported residuals
    // (iterations.cpp:617-659)
    const float velFloor = std::max(residNormFloorVel, 1e-30f);
    const float massFloor = std::max(residNormFloorMass, 1e-30f);
    if (!residU_RMS0_set && residU_RMS > velFloor) { residU_RMS0 = residU_RMS; residU_RMS0_set = true; }
    if (!residV_RMS0_set && residV_RMS > velFloor) { residV_RMS0 = residV_RMS; residV_RMS0_set = true; }
    if (!residMass_RMS0_set && residMass_RMS > massFloor) { residMass_RMS0 = residMass_RMS; residMass_RMS0_set = true; }
    if (!residU_RMS0_set) residU_RMS0 = velFloor;
    if (!residV_RMS0_set) residV_RMS0 = velFloor;
    if (!residMass_RMS0_set) residMass_RMS0 = massFloor;
    residU = (float)r.residU; residV = (float)r.residV; residMass = (float)r.residMass;
    return std::max({residU, residV, residMass});
}
