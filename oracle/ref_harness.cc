// C entry points around the reference's own solver, compiled here from the
// reference sources (oracle/Makefile, target _ref): DP3's
// IterativeDiagonalSolver / IterativeScalarSolver / SolverBase / SolveData /
// SmoothnessConstraint .cc files and AntennaConstraint.h, unmodified, built
// against the project's stand-ins for DP3's external headers
// (dp3_b200/dp3/standin: aocommon, schaapcommon, xtensor, xsimd, DPBuffer).
//
// TEST INFRASTRUCTURE ONLY: this is the reference-code oracle. Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline legs load it.
//
// ref_solve packs one solution interval into DPBuffers (one per time step:
// data "" and one cube per direction, [baseline][channel][4 correlations]),
// builds SolveData<V> through the reference's regular constructor
// (SolveData.cc:77-188: even channel-block split, autocorrelations dropped,
// direction-dependent solution indices), sets up the solver the way DDECal's
// SolverFactory does (SolverFactory.cc:49-146: Initialize, the setters,
// AddConstraint + Constraint::Initialize) and calls Solve(data, solutions,
// time) (SolverBase.h:205-227). The shared steps are in ref_problem.h.
#include <chrono>
#include <stdexcept>
#include <string>

#include "ddecal/gain_solvers/IterativeDiagonalSolver.h"
#include "ddecal/gain_solvers/IterativeFullJonesSolver.h"
#include "ddecal/gain_solvers/IterativeScalarSolver.h"
#include "ddecal/linear_solvers/LLSSolver.h"
#include "ref_problem.h"

namespace dp3::ddecal {
// SolverBase.cc references LLSSolver::Make (CreateLLSSolver, used only by
// the direct solvers); the iterative solvers never call it, and the LAPACK
// solvers behind it are not built here.
std::unique_ptr<LLSSolver> LLSSolver::Make(LLSSolverType, int, int, int) {
  throw std::runtime_error("LLSSolver is not available in the reference-code oracle");
}
}  // namespace dp3::ddecal

#define REF_API __attribute__((visibility("default")))

namespace {

thread_local std::string g_error;

template <typename Solver, typename V>
int Run(const ref_problem& p, const ref_settings& s, uint32_t n_threads,
        const ref_constraints* c, double* solutions, ref_result* out) {
  schaapcommon::ThreadPool::GetInstance().SetNThreads(std::max<uint32_t>(n_threads, 1));
  const auto t0 = std::chrono::steady_clock::now();
  const dp3::ddecal::SolveData<V> data = dp3b200_ref::Pack<V>(p);
  const auto t1 = std::chrono::steady_clock::now();
  Solver solver;
  dp3b200_ref::Configure(solver, p, s, c);
  const size_t n_sub = std::accumulate(p.n_solutions_per_direction,
                                       p.n_solutions_per_direction + p.n_directions, size_t(0));
  const size_t per_cb = size_t(p.n_antennas) * n_sub * solver.NSolutionPolarizations();
  auto sol = dp3b200_ref::ToVectors(solutions, p.n_channel_blocks, per_cb);
  const auto t2 = std::chrono::steady_clock::now();
  const dp3::ddecal::SolverBase::SolveResult r = solver.Solve(data, sol, 0.0);
  const auto t3 = std::chrono::steady_clock::now();
  dp3b200_ref::FromVectors(sol, solutions);
  out->iterations = uint32_t(r.iterations);
  out->constraint_iterations = uint32_t(r.constraint_iterations);
  out->seconds_packing = std::chrono::duration<double>(t1 - t0).count();
  out->seconds_solve = std::chrono::duration<double>(t3 - t2).count();
  return 0;
}

// An interval packed once (SolveData of the solver kind), solved many times.
struct PreparedBase {
  virtual ~PreparedBase() = default;
  virtual int Solve(const ref_problem& p, const ref_settings& s, uint32_t n_threads,
                    const ref_constraints* c, double* solutions, ref_result* out) = 0;
};

template <typename Solver, typename V>
struct Prepared final : PreparedBase {
  explicit Prepared(const ref_problem& p) : data(dp3b200_ref::Pack<V>(p)) {}
  int Solve(const ref_problem& p, const ref_settings& s, uint32_t n_threads,
            const ref_constraints* c, double* solutions, ref_result* out) override {
    schaapcommon::ThreadPool::GetInstance().SetNThreads(std::max<uint32_t>(n_threads, 1));
    Solver solver;
    dp3b200_ref::Configure(solver, p, s, c);
    const size_t n_sub = std::accumulate(
        p.n_solutions_per_direction, p.n_solutions_per_direction + p.n_directions, size_t(0));
    const size_t per_cb = size_t(p.n_antennas) * n_sub * solver.NSolutionPolarizations();
    auto sol = dp3b200_ref::ToVectors(solutions, p.n_channel_blocks, per_cb);
    const auto t0 = std::chrono::steady_clock::now();
    const dp3::ddecal::SolverBase::SolveResult r = solver.Solve(data, sol, 0.0);
    const auto t1 = std::chrono::steady_clock::now();
    dp3b200_ref::FromVectors(sol, solutions);
    out->iterations = uint32_t(r.iterations);
    out->constraint_iterations = uint32_t(r.constraint_iterations);
    out->seconds_packing = 0.0;
    out->seconds_solve = std::chrono::duration<double>(t1 - t0).count();
    return 0;
  }
  const dp3::ddecal::SolveData<V> data;
};

PreparedBase* Prepare(const ref_problem& p, int kind) {
  using namespace dp3::ddecal;
  switch (kind) {
    case REF_DIAGONAL_DUO:
      return new Prepared<IterativeDiagonalSolver<aocommon::MC2x2FDiag>, aocommon::MC2x2FDiag>(p);
    case REF_DIAGONAL_FULL:
      return new Prepared<IterativeDiagonalSolver<aocommon::MC2x2F>, aocommon::MC2x2F>(p);
    case REF_SCALAR_UNI:
      return new Prepared<IterativeScalarSolver<std::complex<float>>, std::complex<float>>(p);
    case REF_SCALAR_DUO:
      return new Prepared<IterativeScalarSolver<aocommon::MC2x2FDiag>, aocommon::MC2x2FDiag>(p);
    case REF_SCALAR_FULL:
      return new Prepared<IterativeScalarSolver<aocommon::MC2x2F>, aocommon::MC2x2F>(p);
    case REF_FULL_JONES:
      return new Prepared<IterativeFullJonesSolver, aocommon::MC2x2F>(p);
    default:
      throw std::runtime_error("unknown solver kind");
  }
}

}  // namespace

typedef struct ref_prepared ref_prepared;

// Packs the interval once (the reference's SolveData constructor, timed into
// *seconds_packing); ref_solve_prepared then solves it with any settings.
extern "C" REF_API int ref_prepare(const ref_problem* p, int kind, ref_prepared** out,
                                   double* seconds_packing) {
  if (!p || !out) {
    g_error = "NULL argument";
    return 1;
  }
  try {
    const auto t0 = std::chrono::steady_clock::now();
    *out = reinterpret_cast<ref_prepared*>(Prepare(*p, kind));
    if (seconds_packing)
      *seconds_packing =
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return 0;
  } catch (const std::exception& e) {
    g_error = e.what();
    return 2;
  }
}

// `p` supplies the dimensions again (the same problem as ref_prepare's).
extern "C" REF_API int ref_solve_prepared(ref_prepared* h, const ref_problem* p,
                                          const ref_settings* s, uint32_t n_threads,
                                          const ref_constraints* c, double* solutions,
                                          ref_result* out) {
  if (!h || !p || !s || !solutions || !out) {
    g_error = "NULL argument";
    return 1;
  }
  try {
    return reinterpret_cast<PreparedBase*>(h)->Solve(*p, *s, n_threads, c, solutions, out);
  } catch (const std::exception& e) {
    g_error = e.what();
    return 2;
  }
}

extern "C" REF_API void ref_release(ref_prepared* h) { delete reinterpret_cast<PreparedBase*>(h); }

extern "C" REF_API const char* ref_last_error(void) { return g_error.c_str(); }

extern "C" REF_API int ref_solve(const ref_problem* p, const ref_settings* s, int kind,
                                 uint32_t n_threads, const ref_constraints* c,
                                 double* solutions, ref_result* out) {
  if (!p || !s || !solutions || !out) {
    g_error = "NULL argument";
    return 1;
  }
  if (p->n_correlations_in != 1 && p->n_correlations_in != 2 && p->n_correlations_in != 4) {
    g_error = "n_correlations_in must be 1, 2 or 4";
    return 1;
  }
  using namespace dp3::ddecal;
  try {
    switch (kind) {
      case REF_DIAGONAL_DUO:
        return Run<IterativeDiagonalSolver<aocommon::MC2x2FDiag>, aocommon::MC2x2FDiag>(
            *p, *s, n_threads, c, solutions, out);
      case REF_DIAGONAL_FULL:
        return Run<IterativeDiagonalSolver<aocommon::MC2x2F>, aocommon::MC2x2F>(
            *p, *s, n_threads, c, solutions, out);
      case REF_SCALAR_UNI:
        return Run<IterativeScalarSolver<std::complex<float>>, std::complex<float>>(
            *p, *s, n_threads, c, solutions, out);
      case REF_SCALAR_DUO:
        return Run<IterativeScalarSolver<aocommon::MC2x2FDiag>, aocommon::MC2x2FDiag>(
            *p, *s, n_threads, c, solutions, out);
      case REF_SCALAR_FULL:
        return Run<IterativeScalarSolver<aocommon::MC2x2F>, aocommon::MC2x2F>(
            *p, *s, n_threads, c, solutions, out);
      case REF_FULL_JONES:
        return Run<IterativeFullJonesSolver, aocommon::MC2x2F>(*p, *s, n_threads, c, solutions,
                                                                out);
      default:
        g_error = "unknown solver kind";
        return 1;
    }
  } catch (const std::exception& e) {
    g_error = e.what();
    return 2;
  }
}
