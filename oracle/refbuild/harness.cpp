// Driver that runs the reference solver's own sources (compiled against the
// Eigen API stand-in in shim/) on a case directory and dumps what the parity
// tests need.  Test infrastructure: it builds the CPU oracle in oracle/_ref/
// and the timed CPU baseline; nothing in the product links it.
//
// The reference keeps its outer loop in SIMPLE::runIterations()
// (SIMPLE.cpp:310-528), which also writes logs and VTK files every iteration.
// This driver keeps the loop's arithmetic and stop rule (inlet ramp
// SIMPLE.cpp:382-386, calculateStep :396, pseudo-time hook :400-409, the four
// pressure samples :423-432, error > epsilon :378) but records the history in
// memory and writes binary dumps at full precision instead of text.
//
// Usage: ref_harness <case_dir> <out_dir> [key=value ...]
//   case_dir holds ExportFiles/fluid_params.txt and ExportFiles/geometry_fluid.txt
//   keys: see applyOverride() below; threads=N sets the OpenMP thread count
//   (the constructor forces numThreads=8, SIMPLE.cpp:101, so it is reset here).
#include "SIMPLE.h"

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unistd.h>
#include <vector>

#ifndef REF_REAL
#define REF_REAL float
#endif
typedef REF_REAL real_t;

namespace {

struct Options {
    int threads = 1;
    int timeOnly = 0;       // 1: only print per-iteration timing, no dumps
    int runNative = 0;      // 1: call runIterations() itself (writes ExportFiles/*)
};

bool applyOverride(SIMPLE& s, Options& o, const std::string& key, const std::string& val) {
    const double d = std::atof(val.c_str());
    const int i = std::atoi(val.c_str());
#define SETR(name) if (key == #name) { s.name = static_cast<real_t>(d); return true; }
#define SETI(name) if (key == #name) { s.name = i; return true; }
#define SETB(name) if (key == #name) { s.name = (i != 0); return true; }
    SETR(rho) SETR(eta) SETR(brinkmanKMin) SETR(brinkmanQ)
    SETI(convectionScheme) SETB(enableTwoPointFiveD) SETR(twoPointFiveDConvectionFactor)
    SETR(twoPointFiveDSinkMultiplier) SETR(Ht_channel)
    SETR(epsilon) SETI(maxIterations) SETI(maxPressureIter) SETR(pTol)
    SETR(momentumTol) SETI(maxMomentumIter) SETR(uvAlpha) SETR(pAlpha)
    SETR(xPlaneCoreInlet) SETR(xPlaneCoreOutlet) SETB(enableInletRamp) SETI(rampSteps)
    SETI(pressureSolverType) SETI(momentumSolverType) SETB(usePressureDropConvergence)
    SETI(dpConvergenceWindow) SETR(dpConvergencePercent) SETI(saveStateInterval)
    SETB(enableNormalizedResiduals)
#undef SETR
#undef SETI
#undef SETB
    if (key == "threads") { o.threads = i; return true; }
    if (key == "time_only") { o.timeOnly = i; return true; }
    if (key == "run_native") { o.runNative = i; return true; }
    return false;
}

void dumpMatrix(FILE* f, const char* name, const Eigen::DenseMatrix<real_t>& m) {
    // header: name (16 bytes), rows, cols (int32); then row-major float64 data
    char tag[16] = {0};
    std::strncpy(tag, name, 15);
    std::fwrite(tag, 1, 16, f);
    int dims[2] = {static_cast<int>(m.rows()), static_cast<int>(m.cols())};
    std::fwrite(dims, sizeof(int), 2, f);
    std::vector<double> row(static_cast<size_t>(m.cols()));
    for (int r = 0; r < dims[0]; ++r) {
        for (int c = 0; c < dims[1]; ++c) row[static_cast<size_t>(c)] = static_cast<double>(m(r, c));
        std::fwrite(row.data(), sizeof(double), row.size(), f);
    }
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s <case_dir> <out_dir> [key=value ...]\n", argv[0]);
        return 2;
    }
    const std::string caseDir = argv[1];
    std::string outDir = argv[2];
    if (!outDir.empty() && outDir[0] != '/') {
        char cwd[4096];
        if (getcwd(cwd, sizeof cwd)) outDir = std::string(cwd) + "/" + outDir;
    }
    if (chdir(caseDir.c_str()) != 0) {
        std::fprintf(stderr, "cannot enter %s\n", caseDir.c_str());
        return 2;
    }

    // Constructor output (banner, geometry counts) goes to stdout; keep it.
    SIMPLE s;
    Options opt;
    // Defaults that make a run reproducible and quiet (see the SIMPLE.h knobs).
    s.usePressureDropConvergence = false;
    s.saveStateInterval = 0;
    for (int a = 3; a < argc; ++a) {
        std::string kv = argv[a];
        size_t eq = kv.find('=');
        if (eq == std::string::npos || !applyOverride(s, opt, kv.substr(0, eq), kv.substr(eq + 1))) {
            std::fprintf(stderr, "bad override '%s'\n", kv.c_str());
            return 2;
        }
    }
    // The 2.5-D switch is validated at load time (SIMPLE.cpp:67-73); repeat
    // that check for a switch turned on by an override.
    if (s.enableTwoPointFiveD && s.Ht_channel <= real_t(0)) s.enableTwoPointFiveD = false;
    // alpha_max depends on eta and K_min (SIMPLE.cpp:78-79); rebuild after overrides.
    s.brinkmanAlphaMax = s.eta / std::max(s.brinkmanKMin, static_cast<real_t>(1e-20));
    s.buildAlphaFromDensity();
    s.numThreads = opt.threads;
    omp_set_num_threads(opt.threads);

    if (opt.runNative) {
        s.runIterations();
        return 0;
    }

    FILE* hist = nullptr;
    if (!opt.timeOnly) {
        hist = std::fopen((outDir + "/history.txt").c_str(), "w");
        if (!hist) { std::fprintf(stderr, "cannot write %s\n", outDir.c_str()); return 2; }
        std::fprintf(hist, "iter error residU_RMS residV_RMS residMass_RMS residU_max residV_max "
                           "residMass_max pIters coreTotal fullTotal coreStatic fullStatic "
                           "inMassFlux outMassFlux seconds\n");
    }

    const real_t domainXMax = (s.N - 1) * s.hx;
    (void)domainXMax;
    int iter = 0;
    real_t error = 1;
    double total = 0.0;
    while (iter < s.maxIterations && error > s.epsilon) {
        auto t0 = std::chrono::steady_clock::now();
        if (s.enableInletRamp && s.rampSteps > 0 && iter < s.rampSteps)
            s.inletVelocity = (static_cast<real_t>(iter + 1) / s.rampSteps) * s.targetVel;
        else
            s.inletVelocity = s.targetVel;
        int pIters = 0;
        error = s.calculateStep(pIters);
        s.updatePseudoTimeController(std::max({s.residU_RMS, s.residV_RMS, s.residMass_RMS}), iter + 1);
        PlaneMetrics ci = samplePlaneAtX(s, s.xPlaneCoreInlet);
        PlaneMetrics co = samplePlaneAtX(s, s.xPlaneCoreOutlet);
        PlaneMetrics fi = sampleBoundaryPatch(s, true);
        PlaneMetrics fo = sampleBoundaryPatch(s, false);
        double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        total += sec;
        if (hist) {
            std::fprintf(hist, "%d %.17g %.17g %.17g %.17g %.17g %.17g %.17g %d %.17g %.17g %.17g %.17g %.17g %.17g %.6f\n",
                         iter, double(error), double(s.residU_RMS), double(s.residV_RMS),
                         double(s.residMass_RMS), double(s.residU_max), double(s.residV_max),
                         double(s.residMass_max), pIters,
                         double(ci.avgTotal - co.avgTotal), double(fi.avgTotal - fo.avgTotal),
                         double(ci.avgStatic - co.avgStatic), double(fi.avgStatic - fo.avgStatic),
                         double(fi.massFlux), double(fo.massFlux), sec);
        } else {
            std::printf("ITER %d %.6f %d %.9g\n", iter, sec, pIters, double(fi.avgTotal - fo.avgTotal));
            std::fflush(stdout);
        }
        iter++;
    }
    if (hist) std::fclose(hist);
    if (!opt.timeOnly) {
        FILE* f = std::fopen((outDir + "/fields.bin").c_str(), "wb");
        if (!f) return 2;
        dumpMatrix(f, "u", s.u);
        dumpMatrix(f, "v", s.v);
        dumpMatrix(f, "p", s.p);
        dumpMatrix(f, "uStar", s.uStar);
        dumpMatrix(f, "vStar", s.vStar);
        dumpMatrix(f, "pStar", s.pStar);
        dumpMatrix(f, "dE", s.dE);
        dumpMatrix(f, "dN", s.dN);
        dumpMatrix(f, "gamma", s.gamma);
        dumpMatrix(f, "alpha", s.alpha);
        std::fclose(f);
    }
    std::printf("DONE iters=%d seconds=%.6f error=%.9g\n", iter, total, double(error));
    return 0;
}
