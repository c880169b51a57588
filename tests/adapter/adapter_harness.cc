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
#include <sstream>
#include <stdexcept>
#include <string>

#include "dp3/IterativeSolverB200.h"
#include "ddecal/gain_solvers/IterativeDiagonalSolver.h"
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

template <typename Solver, typename V>
int Run(Solver& solver, const ref_problem& p, const ref_settings& s, const ref_constraints* c,
        double* solutions, ref_result* out, double* step_magnitudes, uint32_t n_step_cap) {
  const dp3::ddecal::SolveData<V> data = dp3b200_ref::Pack<V>(p);
  dp3b200_ref::Configure(solver, p, s, c);
  const size_t n_sub = std::accumulate(p.n_solutions_per_direction,
                                       p.n_solutions_per_direction + p.n_directions, size_t(0));
  const size_t per_cb = size_t(p.n_antennas) * n_sub * solver.NSolutionPolarizations();
  auto sol = dp3b200_ref::ToVectors(solutions, p.n_channel_blocks, per_cb);
  dp3::ddecal::SolverBase::SolveResult r;
  if constexpr (std::is_same_v<Solver, dp3::ddecal::IterativeSolverB200<V, 2>> ||
                std::is_same_v<Solver, dp3::ddecal::IterativeSolverB200<V, 1>>) {
    std::ostringstream stats;  // the statistics-stream overload
    r = solver.Solve(data, sol, 0.0, &stats);
    std::istringstream in(stats.str());
    size_t it;
    double mag;
    while (in >> it >> mag)
      if (step_magnitudes && it >= 1 && it <= n_step_cap) step_magnitudes[it - 1] = mag;
  } else {
    r = solver.Solve(data, sol, 0.0);
  }
  dp3b200_ref::FromVectors(sol, solutions);
  out->iterations = uint32_t(r.iterations);
  out->constraint_iterations = uint32_t(r.constraint_iterations);
  return 0;
}

template <typename V, size_t NPol>
int Dispatch(int use_b200, int device, const ref_problem& p, const ref_settings& s,
             const ref_constraints* c, double* solutions, ref_result* out, double* mags,
             uint32_t cap) {
  using namespace dp3::ddecal;
  if (use_b200) {
    IterativeSolverB200<V, NPol> solver(device);
    return Run<IterativeSolverB200<V, NPol>, V>(solver, p, s, c, solutions, out, mags, cap);
  }
  if constexpr (NPol == 2) {
    IterativeDiagonalSolver<V> solver;
    return Run<IterativeDiagonalSolver<V>, V>(solver, p, s, c, solutions, out, mags, cap);
  } else {
    IterativeScalarSolver<V> solver;
    return Run<IterativeScalarSolver<V>, V>(solver, p, s, c, solutions, out, mags, cap);
  }
}

}  // namespace

extern "C" HARNESS_API const char* adapter_last_error(void) { return g_error.c_str(); }

// kind: REF_* of ref_problem.h; use_b200: 0 = DP3's own solver, 1 = the B200
// adapter on CUDA device `device`. step_magnitudes (optional, adapter only):
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
      default:
        g_error = "unknown solver kind";
        return 1;
    }
  } catch (const std::exception& e) {
    g_error = e.what();
    return 2;
  }
}
