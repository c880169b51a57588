// Test harness of the DP3 adapter (dp3_b200/dp3/IterativeSolverB200.h): C
// entry points that build one regular solution interval through DP3's own
// SolveData constructor and solve it either with DP3's own
// IterativeDiagonalSolver / IterativeScalarSolver or with the adapter, both
// configured the same way through DP3's SolverBase (Initialize, setters,
// AntennaConstraint / SmoothnessConstraint), so that tests compare the two
// on identical inputs inside one process. DP3's solver sources are compiled
// from the reference tree (tests/adapter/Makefile); the adapter calls
// libddsolve_b200.so on the GPU.
//
// TEST INFRASTRUCTURE: only tests/test_dp3_adapter.py loads this library.
#include <execinfo.h>
#include <signal.h>
#include <unistd.h>

#include <cstdlib>
#include <sstream>
#include <stdexcept>
#include <string>

namespace {
void Trace(const char* what);
}
#define DP3B200_ADAPTER_TRACE(what) Trace(what)
#include "dp3/IterativeSolverB200.h"
#include "ddecal/gain_solvers/IterativeDiagonalSolver.h"
#include "ddecal/gain_solvers/IterativeFullJonesSolver.h"
#include "ddecal/gain_solvers/IterativeScalarSolver.h"
#include "ddecal/linear_solvers/LLSSolver.h"
#include "ref_problem.h"

namespace dp3::ddecal {
// Referenced by SolverBase.cc (direct solvers only); not used by the
// iterative solvers.
std::unique_ptr<LLSSolver> LLSSolver::Make(LLSSolverType, int, int, int) {
  throw std::runtime_error("LLSSolver is not available in this harness");
}
}  // namespace dp3::ddecal

#define HARNESS_API __attribute__((visibility("default")))

namespace {

thread_local std::string g_error;

// With DP3B200_HARNESS_BACKTRACE set: progress lines on stderr around the
// solver calls, and a native backtrace when the process takes SIGSEGV /
// SIGABRT (library offsets, resolvable with addr2line against the same
// build), printed from an alternate signal stack so that a stack overflow is
// reported too; then the default action.
bool g_trace = false;
void Trace(const char* what) {
  if (!g_trace) return;
  const std::string line = std::string("harness: ") + what + "\n";
  (void)!write(2, line.data(), line.size());
}
void CrashReport(int sig, siginfo_t* info, void*) {
  char head[96];
  const int len = snprintf(head, sizeof(head), "harness: signal %d at address %p\n", sig,
                           info ? info->si_addr : nullptr);
  (void)!write(2, head, size_t(len));
  void* frames[64];
  const int n = backtrace(frames, 64);
  backtrace_symbols_fd(frames, n, 2);
  signal(sig, SIG_DFL);
  raise(sig);
}
struct CrashReporter {
  CrashReporter() {
    if (!std::getenv("DP3B200_HARNESS_BACKTRACE")) return;
    g_trace = true;
    static char alt_stack[1 << 16];
    stack_t ss{};
    ss.ss_sp = alt_stack;
    ss.ss_size = sizeof(alt_stack);
    sigaltstack(&ss, nullptr);
    struct sigaction sa {};
    sa.sa_sigaction = CrashReport;
    sa.sa_flags = SA_SIGINFO | SA_ONSTACK;
    sigaction(SIGSEGV, &sa, nullptr);
    sigaction(SIGABRT, &sa, nullptr);
    sigaction(SIGBUS, &sa, nullptr);
  }
} g_crash_reporter;

template <typename Solver, typename V,
          typename Smoothness = dp3::ddecal::SmoothnessConstraint>
int Run(Solver& solver, const ref_problem& p, const ref_settings& s, const ref_constraints* c,
        double* solutions, ref_result* out, double* step_magnitudes, uint32_t n_step_cap) {
  Trace("pack");
  const dp3::ddecal::SolveData<V> data = dp3b200_ref::Pack<V>(p);
  Trace("configure");
  dp3b200_ref::Configure<Smoothness>(solver, p, s, c);
  const size_t n_sub = std::accumulate(p.n_solutions_per_direction,
                                       p.n_solutions_per_direction + p.n_directions, size_t(0));
  const size_t per_cb = size_t(p.n_antennas) * n_sub * solver.NSolutionPolarizations();
  auto sol = dp3b200_ref::ToVectors(solutions, p.n_channel_blocks, per_cb);
  dp3::ddecal::SolverBase::SolveResult r;
  if constexpr (std::is_same_v<Solver, dp3::ddecal::IterativeSolverB200<V, 2>> ||
                std::is_same_v<Solver, dp3::ddecal::IterativeSolverB200<V, 1>> ||
                std::is_same_v<Solver, dp3::ddecal::IterativeSolverB200<V, 4>>) {
    std::ostringstream stats;  // the statistics-stream overload
    Trace("adapter solve");
    r = solver.Solve(data, sol, 0.0, &stats);
    Trace("adapter solve done");
    std::istringstream in(stats.str());
    size_t it;
    double mag;
    while (in >> it >> mag)
      if (step_magnitudes && it >= 1 && it <= n_step_cap) step_magnitudes[it - 1] = mag;
  } else {
    r = solver.Solve(data, sol, 0.0);
  }
  dp3b200_ref::FromVectors(sol, solutions);
  Trace("results copied");
  out->iterations = uint32_t(r.iterations);
  out->constraint_iterations = uint32_t(r.constraint_iterations);
  return 0;
}

template <typename V, size_t NPol>
int Dispatch(int use_b200, int device, const ref_problem& p, const ref_settings& s,
             const ref_constraints* c, double* solutions, ref_result* out, double* mags,
             uint32_t cap) {
  using namespace dp3::ddecal;
  if (use_b200 == 2) {  // smoothness through the adapter's device-capable class
    IterativeSolverB200<V, NPol> solver(device);
    return Run<IterativeSolverB200<V, NPol>, V, SmoothnessConstraintB200>(solver, p, s, c,
                                                                         solutions, out, mags,
                                                                         cap);
  }
  if (use_b200) {
    IterativeSolverB200<V, NPol> solver(device);
    return Run<IterativeSolverB200<V, NPol>, V>(solver, p, s, c, solutions, out, mags, cap);
  }
  if constexpr (NPol == 4) {
    IterativeFullJonesSolver solver;
    return Run<IterativeFullJonesSolver, V>(solver, p, s, c, solutions, out, mags, cap);
  } else if constexpr (NPol == 2) {
    IterativeDiagonalSolver<V> solver;
    return Run<IterativeDiagonalSolver<V>, V>(solver, p, s, c, solutions, out, mags, cap);
  } else {
    IterativeScalarSolver<V> solver;
    return Run<IterativeScalarSolver<V>, V>(solver, p, s, c, solutions, out, mags, cap);
  }
}

}  // namespace

extern "C" HARNESS_API const char* adapter_last_error(void) { return g_error.c_str(); }

namespace {
template <typename V, size_t NPol>
int CorrectAndSubtract(int device, uint32_t n_ant, uint32_t n_dir, uint32_t n_cb,
                       uint32_t n_times, uint32_t n_bl, uint32_t n_ch, const uint32_t* a1,
                       const uint32_t* a2, const double* solutions, float* data,
                       float* models, int subtract, int keep) {
  dp3::ddecal::IterativeSolverB200<V, NPol> solver(device);
  solver.Initialize(n_ant, std::vector<size_t>(n_dir, 1), n_cb);
  const size_t per_cb = size_t(n_ant) * n_dir * NPol;
  const auto sol = dp3b200_ref::ToVectors(solutions, n_cb, per_cb);
  const std::vector<uint32_t> ant1(a1, a1 + n_bl), ant2(a2, a2 + n_bl);
  const size_t per_step = size_t(n_bl) * n_ch * 4;  // complex values of one time step
  auto* d = reinterpret_cast<std::complex<float>*>(data);
  auto* m = reinterpret_cast<std::complex<float>*>(models);
  for (uint32_t t = 0; t < n_times; ++t) {  // one DPBuffer per time step, as DDECal holds them
    std::vector<std::complex<float>*> step_models(n_dir);
    for (uint32_t k = 0; k < n_dir; ++k)
      step_models[k] = m + (size_t(k) * n_times + t) * per_step;
    solver.CorrectAndSubtract(sol, n_bl, n_ch, ant1, ant2, d + t * per_step, step_models,
                              subtract != 0, keep != 0);
  }
  return 0;
}
}  // namespace

// The adapter's CorrectAndSubtract for n_pol 1, 2 or 4 (4-correlation
// buffers): data [n_times][n_bl][n_ch][4] and models [n_dir][n_times][n_bl]
// [n_ch][4] (complex float) are corrected in place, one call per time step.
extern "C" HARNESS_API int adapter_correct_and_subtract(int n_pol, int device, uint32_t n_ant,
                                                        uint32_t n_dir, uint32_t n_cb,
                                                        uint32_t n_times, uint32_t n_bl,
                                                        uint32_t n_ch, const uint32_t* a1,
                                                        const uint32_t* a2,
                                                        const double* solutions, float* data,
                                                        float* models, int subtract, int keep) {
  try {
    switch (n_pol) {
      case 1:
        return CorrectAndSubtract<aocommon::MC2x2F, 1>(device, n_ant, n_dir, n_cb, n_times, n_bl,
                                                       n_ch, a1, a2, solutions, data, models,
                                                       subtract, keep);
      case 2:
        return CorrectAndSubtract<aocommon::MC2x2F, 2>(device, n_ant, n_dir, n_cb, n_times, n_bl,
                                                       n_ch, a1, a2, solutions, data, models,
                                                       subtract, keep);
      case 4:
        return CorrectAndSubtract<aocommon::MC2x2F, 4>(device, n_ant, n_dir, n_cb, n_times, n_bl,
                                                       n_ch, a1, a2, solutions, data, models,
                                                       subtract, keep);
      default:
        g_error = "n_pol must be 1, 2 or 4";
        return 1;
    }
  } catch (const std::exception& e) {
    g_error = e.what();
    return 2;
  }
}

// kind: REF_* of ref_problem.h; use_b200: 0 = DP3's own solver, 1 = the B200
// adapter on CUDA device `device` with DP3's constraint classes (a
// SmoothnessConstraint keeps the loop on the host), 2 = the adapter with its
// SmoothnessConstraintB200 (with DP3's AntennaConstraint: device constraints,
// the loop on the device). step_magnitudes (optional, adapter only):
// the statistics stream's per-iteration step magnitudes, up to n_step_cap.
extern "C" HARNESS_API int adapter_solve(const ref_problem* p, const ref_settings* s, int kind,
                                         int use_b200, int device, uint32_t n_threads,
                                         const ref_constraints* c, double* solutions,
                                         ref_result* out, double* step_magnitudes,
                                         uint32_t n_step_cap) {
  if (!p || !s || !solutions || !out) {
    g_error = "NULL argument";
    return 1;
  }
  schaapcommon::ThreadPool::GetInstance().SetNThreads(std::max<uint32_t>(n_threads, 1));
  try {
    switch (kind) {
      case REF_DIAGONAL_DUO:
        return Dispatch<aocommon::MC2x2FDiag, 2>(use_b200, device, *p, *s, c, solutions, out,
                                                 step_magnitudes, n_step_cap);
      case REF_DIAGONAL_FULL:
        return Dispatch<aocommon::MC2x2F, 2>(use_b200, device, *p, *s, c, solutions, out,
                                             step_magnitudes, n_step_cap);
      case REF_SCALAR_UNI:
        return Dispatch<std::complex<float>, 1>(use_b200, device, *p, *s, c, solutions, out,
                                                step_magnitudes, n_step_cap);
      case REF_SCALAR_DUO:
        return Dispatch<aocommon::MC2x2FDiag, 1>(use_b200, device, *p, *s, c, solutions, out,
                                                 step_magnitudes, n_step_cap);
      case REF_SCALAR_FULL:
        return Dispatch<aocommon::MC2x2F, 1>(use_b200, device, *p, *s, c, solutions, out,
                                             step_magnitudes, n_step_cap);
      case REF_FULL_JONES:
        return Dispatch<aocommon::MC2x2F, 4>(use_b200, device, *p, *s, c, solutions, out,
                                             step_magnitudes, n_step_cap);
      default:
        g_error = "unknown solver kind";
        return 1;
    }
  } catch (const std::exception& e) {
    g_error = e.what();
    return 2;
  }
}
