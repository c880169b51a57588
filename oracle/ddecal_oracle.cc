// CPU oracle for the DDECal direction-iterative gain solve.
//
// TEST INFRASTRUCTURE ONLY: the checker for the CUDA solver in dp3_b200. Only
// tests/, __graft_entry__.smoke() and the cpu-baseline legs of bench.py load
// it; the product never links it.
//
// This is a restatement, in plain C++, of the reference algorithm. Each
// function names the reference lines it follows. The arithmetic of the
// reference is kept (std::complex<float> per visibility, FP32 accumulators in
// the diagonal solver, FP64 accumulators in the scalar solver, FP64 division,
// FP64 step and convergence norm) when precision == 32; precision == 64 runs
// the same algorithm entirely in FP64 and is the "FP64 oracle".
#include "ddecal_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstring>
#include <limits>
#include <numeric>
#include <random>
#include <thread>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// Small fixed-size visibility matrices. NCorr = 1 (complex<float>), 2 (the
// diagonal XX/YY pair, aocommon::MC2x2FDiag) or 4 (row-major 2x2
// [XX XY; YX YY], aocommon::MC2x2F). The reference's operator semantics are
// restated from its call sites: IterativeDiagonalSolver.cc:20-34,160-197,
// SolveData.h:230-241, IterativeScalarSolver.cc:20-27,151-175,213-221.
// ---------------------------------------------------------------------------
template <typename T, int NCorr>
struct Vis {
  std::complex<T> v[NCorr];
};

template <typename T, int NCorr>
Vis<T, NCorr> LoadVis(const float* p) {
  Vis<T, NCorr> r;
  for (int i = 0; i < NCorr; ++i)
    r.v[i] = std::complex<T>(T(p[2 * i]), T(p[2 * i + 1]));
  return r;
}

// Diagonal solution pair (pol 0 = X, pol 1 = Y) cast to T.
template <typename T>
struct DiagGain {
  std::complex<T> g[2];
};

template <typename T>
DiagGain<T> LoadDiagGain(const std::complex<double>* s) {
  return DiagGain<T>{{std::complex<T>(s[0]), std::complex<T>(s[1])}};
}

// contribution = diag(ga) * M * diag(gb)^H   (SolveData.h:236-237)
template <typename T>
Vis<T, 2> DiagContribution(const DiagGain<T>& ga, const Vis<T, 2>& m,
                           const DiagGain<T>& gb) {
  Vis<T, 2> r;
  for (int p = 0; p < 2; ++p) r.v[p] = (ga.g[p] * m.v[p]) * std::conj(gb.g[p]);
  return r;
}
template <typename T>
Vis<T, 4> DiagContribution(const DiagGain<T>& ga, const Vis<T, 4>& m,
                           const DiagGain<T>& gb) {
  // (diag(ga) * M): rows scaled; (... * diag(gb)^H): columns scaled.
  Vis<T, 4> r;
  r.v[0] = (ga.g[0] * m.v[0]) * std::conj(gb.g[0]);
  r.v[1] = (ga.g[0] * m.v[1]) * std::conj(gb.g[1]);
  r.v[2] = (ga.g[1] * m.v[2]) * std::conj(gb.g[0]);
  r.v[3] = (ga.g[1] * m.v[3]) * std::conj(gb.g[1]);
  return r;
}

// Per-visibility numerator / denominator contribution of the diagonal solver
// (IterativeDiagonalSolver.cc:160-197 and AddNormToDenominator :20-34).
// For antenna 1: cor = diag(g2) * M^H,  num += Diagonal(D * cor)
// For antenna 2: cor = diag(g1) * M,    num += Diagonal(D^H * cor)
template <typename T, typename Acc>
void DiagSolveContribution(const Vis<T, 2>& d, const Vis<T, 2>& m,
                           const DiagGain<T>& g_ant1, const DiagGain<T>& g_ant2,
                           std::complex<Acc>* num1, Acc* den1,
                           std::complex<Acc>* num2, Acc* den2) {
  for (int p = 0; p < 2; ++p) {
    const std::complex<T> cor1 = g_ant2.g[p] * std::conj(m.v[p]);
    num1[p] += std::complex<Acc>(d.v[p] * cor1);
    den1[p] += Acc(std::norm(cor1));
    const std::complex<T> cor2 = g_ant1.g[p] * m.v[p];
    num2[p] += std::complex<Acc>(std::conj(d.v[p]) * cor2);
    den2[p] += Acc(std::norm(cor2));
  }
}
template <typename T, typename Acc>
void DiagSolveContribution(const Vis<T, 4>& d, const Vis<T, 4>& m,
                           const DiagGain<T>& g_ant1, const DiagGain<T>& g_ant2,
                           std::complex<Acc>* num1, Acc* den1,
                           std::complex<Acc>* num2, Acc* den2) {
  // cor1 = diag(g2) * M^H = [g2x conj(m0), g2x conj(m2); g2y conj(m1), g2y conj(m3)]
  const std::complex<T> c1_0 = g_ant2.g[0] * std::conj(m.v[0]);
  const std::complex<T> c1_1 = g_ant2.g[0] * std::conj(m.v[2]);
  const std::complex<T> c1_2 = g_ant2.g[1] * std::conj(m.v[1]);
  const std::complex<T> c1_3 = g_ant2.g[1] * std::conj(m.v[3]);
  // Diagonal(D * cor1)
  num1[0] += std::complex<Acc>(d.v[0] * c1_0 + d.v[1] * c1_2);
  num1[1] += std::complex<Acc>(d.v[2] * c1_1 + d.v[3] * c1_3);
  den1[0] += Acc(std::norm(c1_0) + std::norm(c1_2));
  den1[1] += Acc(std::norm(c1_1) + std::norm(c1_3));
  // cor2 = diag(g1) * M = [g1x m0, g1x m1; g1y m2, g1y m3]
  const std::complex<T> c2_0 = g_ant1.g[0] * m.v[0];
  const std::complex<T> c2_1 = g_ant1.g[0] * m.v[1];
  const std::complex<T> c2_2 = g_ant1.g[1] * m.v[2];
  const std::complex<T> c2_3 = g_ant1.g[1] * m.v[3];
  // Diagonal(D^H * cor2), D^H = [conj(d0), conj(d2); conj(d1), conj(d3)]
  num2[0] += std::complex<Acc>(std::conj(d.v[0]) * c2_0 +
                               std::conj(d.v[2]) * c2_2);
  num2[1] += std::complex<Acc>(std::conj(d.v[1]) * c2_1 +
                               std::conj(d.v[3]) * c2_3);
  den2[0] += Acc(std::norm(c2_0) + std::norm(c2_2));
  den2[1] += Acc(std::norm(c2_1) + std::norm(c2_3));
}

// Scalar solver per-visibility terms (IterativeScalarSolver.cc:151-175):
// num1 += Trace(D * M^H * g2), den1 += Norm(M^H * g2)
// num2 += Trace(D^H * M * g1), den2 += Norm(M * g1)
// Trace(D * M^H) = sum_i d_i conj(m_i) for the diagonal and full layouts.
template <typename T, int NCorr, typename Acc>
void ScalarSolveContribution(const Vis<T, NCorr>& d, const Vis<T, NCorr>& m,
                             std::complex<T> g1, std::complex<T> g2,
                             std::complex<Acc>& num1, Acc& den1,
                             std::complex<Acc>& num2, Acc& den2) {
  std::complex<T> t1(0, 0), t2(0, 0);
  T n1 = 0, n2 = 0;
  for (int i = 0; i < NCorr; ++i) {
    // HermTranspose(M) * g2 has elements conj(m_j) * g2; the trace pairs
    // d_i with conj(m_i).
    const std::complex<T> c1 = std::conj(m.v[i]) * g2;
    t1 += d.v[i] * c1;
    n1 += std::norm(c1);
    const std::complex<T> c2 = m.v[i] * g1;
    t2 += std::conj(d.v[i]) * c2;
    n2 += std::norm(c2);
  }
  num1 += std::complex<Acc>(t1);
  den1 += Acc(n1);
  num2 += std::complex<Acc>(t2);
  den2 += Acc(n2);
}

// ---------------------------------------------------------------------------
// Minimal fork/join helper: runs fn(task) for task in [0, n_tasks) on up to
// n_threads threads (task order per thread is static, like StaticFor).
// ---------------------------------------------------------------------------
template <typename Fn>
void ParallelTasks(size_t n_tasks, size_t n_threads, Fn&& fn) {
  n_threads = std::max<size_t>(1, std::min(n_threads, n_tasks));
  if (n_threads == 1) {
    for (size_t t = 0; t != n_tasks; ++t) fn(t);
    return;
  }
  std::vector<std::thread> threads;
  threads.reserve(n_threads);
  for (size_t th = 0; th != n_threads; ++th) {
    threads.emplace_back([&, th] {
      const size_t begin = n_tasks * th / n_threads;
      const size_t end = n_tasks * (th + 1) / n_threads;
      for (size_t t = begin; t != end; ++t) fn(t);
    });
  }
  for (std::thread& t : threads) t.join();
}

struct Problem {
  size_t n_ant, n_dir, n_cb, n_corr, n_pol, n_sub;
  std::vector<uint32_t> n_sol_per_dir;
  const oracle_channel_block* cbs;
};

Problem MakeProblem(const oracle_dims* dims, const oracle_channel_block* cbs) {
  Problem p;
  p.n_ant = dims->n_antennas;
  p.n_dir = dims->n_directions;
  p.n_cb = dims->n_channel_blocks;
  p.n_corr = dims->n_correlations;
  p.n_pol = dims->n_solution_polarizations;
  p.n_sol_per_dir.assign(dims->n_solutions_per_direction,
                         dims->n_solutions_per_direction + p.n_dir);
  p.n_sub = std::accumulate(p.n_sol_per_dir.begin(), p.n_sol_per_dir.end(),
                            size_t(0));
  p.cbs = cbs;
  return p;
}

// ---------------------------------------------------------------------------
// PerformIteration for one chunk of visibilities of one channel block.
// Restates IterativeDiagonalSolver.cc:100-127 (and the scalar twin
// IterativeScalarSolver.cc:91-115): subtract all directions, then for every
// direction add it back to a copy of the residual and accumulate that
// direction's normal equations (SolveDirection :130-204 / :117-182).
// Accumulators are laid out [dir][ant * n_dir_solutions + rel][pol].
// ---------------------------------------------------------------------------
template <typename T, int NCorr, int NPol, typename Acc>
struct ChunkAccumulator {
  std::vector<std::vector<std::complex<Acc>>> num;  // [dir][ant*nsol*NPol]
  std::vector<std::vector<Acc>> den;                // [dir][ant*nsol*NPol]
};

template <typename T, int NCorr, int NPol, typename Acc>
void PerformChunk(const Problem& pr, size_t cb, size_t vis_begin,
                  size_t vis_end, const std::complex<double>* solutions,
                  ChunkAccumulator<T, NCorr, NPol, Acc>& acc) {
  const oracle_channel_block& c = pr.cbs[cb];
  const size_t n_vis = c.n_vis;
  acc.num.assign(pr.n_dir, {});
  acc.den.assign(pr.n_dir, {});
  for (size_t d = 0; d != pr.n_dir; ++d) {
    acc.num[d].assign(pr.n_ant * pr.n_sol_per_dir[d] * NPol,
                      std::complex<Acc>(0, 0));
    acc.den[d].assign(pr.n_ant * pr.n_sol_per_dir[d] * NPol, Acc(0));
  }
  if (vis_end <= vis_begin) return;
  const size_t n = vis_end - vis_begin;
  std::vector<Vis<T, NCorr>> residual(n);
  for (size_t i = 0; i != n; ++i)
    residual[i] = LoadVis<T, NCorr>(c.data + (vis_begin + i) * NCorr * 2);

  auto gain_diag = [&](uint32_t ant, uint32_t sol) {
    return LoadDiagGain<T>(&solutions[(ant * pr.n_sub + sol) * 2]);
  };
  auto gain_scalar = [&](uint32_t ant, uint32_t sol) {
    return std::complex<T>(solutions[ant * pr.n_sub + sol]);
  };

  // Subtract all directions (SolveData.h:204-244 with Add = false, and
  // IterativeScalarSolver.cc:197-229).
  for (size_t d = 0; d != pr.n_dir; ++d) {
    const float* model = c.model + d * n_vis * NCorr * 2;
    const uint32_t* solmap = c.solution_map + d * n_vis;
    for (size_t i = 0; i != n; ++i) {
      const size_t vis = vis_begin + i;
      const uint32_t a1 = c.antenna_pairs[2 * vis];
      const uint32_t a2 = c.antenna_pairs[2 * vis + 1];
      const uint32_t s = solmap[vis];
      const Vis<T, NCorr> m = LoadVis<T, NCorr>(model + vis * NCorr * 2);
      if constexpr (NPol == 2) {
        const Vis<T, NCorr> contrib =
            DiagContribution(gain_diag(a1, s), m, gain_diag(a2, s));
        for (int k = 0; k < NCorr; ++k) residual[i].v[k] -= contrib.v[k];
      } else {
        const std::complex<T> g1 = gain_scalar(a1, s);
        const std::complex<T> g2c = std::conj(gain_scalar(a2, s));
        for (int k = 0; k < NCorr; ++k)
          residual[i].v[k] -= (m.v[k] * g1) * g2c;
      }
    }
  }

  // Per direction: residual + this direction (v_residual = v_copy; Add),
  // then accumulate.
  for (size_t d = 0; d != pr.n_dir; ++d) {
    const float* model = c.model + d * n_vis * NCorr * 2;
    const uint32_t* solmap = c.solution_map + d * n_vis;
    const uint32_t sol0 = solmap[0];  // SolutionIndex(direction, 0)
    const uint32_t n_dir_sol = pr.n_sol_per_dir[d];
    std::complex<Acc>* num = acc.num[d].data();
    Acc* den = acc.den[d].data();
    for (size_t i = 0; i != n; ++i) {
      const size_t vis = vis_begin + i;
      const uint32_t a1 = c.antenna_pairs[2 * vis];
      const uint32_t a2 = c.antenna_pairs[2 * vis + 1];
      const uint32_t s = solmap[vis];
      const uint32_t rel = s - sol0;
      const Vis<T, NCorr> m = LoadVis<T, NCorr>(model + vis * NCorr * 2);
      Vis<T, NCorr> rd = residual[i];
      const size_t i1 = (a1 * n_dir_sol + rel) * NPol;
      const size_t i2 = (a2 * n_dir_sol + rel) * NPol;
      if constexpr (NPol == 2) {
        const DiagGain<T> ga = gain_diag(a1, s);
        const DiagGain<T> gb = gain_diag(a2, s);
        const Vis<T, NCorr> contrib = DiagContribution(ga, m, gb);
        for (int k = 0; k < NCorr; ++k) rd.v[k] += contrib.v[k];
        if constexpr (NCorr == 2 || NCorr == 4) {
          DiagSolveContribution<T, Acc>(rd, m, ga, gb, num + i1, den + i1,
                                        num + i2, den + i2);
        }
      } else {
        const std::complex<T> g1 = gain_scalar(a1, s);
        const std::complex<T> g2 = gain_scalar(a2, s);
        const std::complex<T> g2c = std::conj(g2);
        for (int k = 0; k < NCorr; ++k) rd.v[k] += (m.v[k] * g1) * g2c;
        ScalarSolveContribution<T, NCorr, Acc>(rd, m, g1, g2, num[i1], den[i1],
                                               num[i2], den[i2]);
      }
    }
  }
}

// Runs PerformIteration on all channel blocks. Tasks are (channel block,
// sub-chunk) with NSubThreads() = max(1, n_threads / n_cb) chunks per block
// (SolverBase.cc:416-420); chunk partials are merged in chunk order
// (the reference merges them under a mutex, IterativeDiagonalSolver.cc:199-203).
// Output: next[cb][ant][sub][pol] = num / den in FP64, NaN where den == 0
// (IterativeDiagonalSolver.cc:206-221, IterativeScalarSolver.cc:184-194).
template <typename T, int NCorr, int NPol, typename Acc>
void PerformIterationAll(const Problem& pr, size_t n_threads,
                         const std::vector<std::complex<double>>& solutions,
                         std::vector<std::complex<double>>& next) {
  const size_t per_cb = pr.n_ant * pr.n_sub * NPol;
  const size_t n_chunks = std::max<size_t>(1, n_threads / pr.n_cb);
  std::vector<ChunkAccumulator<T, NCorr, NPol, Acc>> accs(pr.n_cb * n_chunks);
  ParallelTasks(pr.n_cb * n_chunks, n_threads, [&](size_t task) {
    const size_t cb = task / n_chunks;
    const size_t chunk = task % n_chunks;
    const size_t n_vis = pr.cbs[cb].n_vis;
    PerformChunk<T, NCorr, NPol, Acc>(
        pr, cb, n_vis * chunk / n_chunks, n_vis * (chunk + 1) / n_chunks,
        solutions.data() + cb * per_cb, accs[task]);
  });
  std::vector<size_t> sol_start(pr.n_dir, 0);
  for (size_t d = 1; d != pr.n_dir; ++d)
    sol_start[d] = sol_start[d - 1] + pr.n_sol_per_dir[d - 1];
  for (size_t cb = 0; cb != pr.n_cb; ++cb) {
    for (size_t d = 0; d != pr.n_dir; ++d) {
      const size_t nds = pr.n_sol_per_dir[d];
      std::vector<std::complex<Acc>> num(pr.n_ant * nds * NPol,
                                         std::complex<Acc>(0, 0));
      std::vector<Acc> den(pr.n_ant * nds * NPol, Acc(0));
      for (size_t chunk = 0; chunk != n_chunks; ++chunk) {
        const auto& a = accs[cb * n_chunks + chunk];
        for (size_t i = 0; i != num.size(); ++i) num[i] += a.num[d][i];
        for (size_t i = 0; i != den.size(); ++i) den[i] += a.den[d][i];
      }
      // The reference uses SolutionIndex(direction, 0) as the first solution
      // of the direction; for regular data this equals the start index.
      const uint32_t sol0 =
          pr.cbs[cb].n_vis ? pr.cbs[cb].solution_map[d * pr.cbs[cb].n_vis]
                           : uint32_t(sol_start[d]);
      for (size_t ant = 0; ant != pr.n_ant; ++ant) {
        for (size_t rel = 0; rel != nds; ++rel) {
          const size_t sol = rel + sol0;
          for (size_t p = 0; p != NPol; ++p) {
            const size_t idx = (ant * nds + rel) * NPol + p;
            std::complex<double>& dst =
                next[cb * per_cb + (ant * pr.n_sub + sol) * NPol + p];
            if (den[idx] == Acc(0))
              dst = std::numeric_limits<double>::quiet_NaN();
            else
              dst = std::complex<double>(num[idx]) / double(den[idx]);
          }
        }
      }
    }
  }
}

bool IsFinite(const std::complex<double>& v) {
  return std::isfinite(v.real()) && std::isfinite(v.imag());
}

// SolverBase::MakeSolutionsFinite1Pol / 2Pol (SolverBase.cc:316-371),
// including the 2-pol quirk that averages |pol 0| for both polarizations.
void MakeSolutionsFinite(std::vector<std::complex<double>>& sols, size_t n_cb,
                         size_t per_cb, size_t n_pol) {
  for (size_t cb = 0; cb != n_cb; ++cb) {
    std::complex<double>* s = sols.data() + cb * per_cb;
    if (n_pol == 1) {
      size_t count = 0;
      double average = 0.0;
      for (size_t i = 0; i != per_cb; ++i)
        if (IsFinite(s[i])) {
          average += std::abs(s[i]);
          ++count;
        }
      average = count == 0 ? 1.0 : average / count;
      for (size_t i = 0; i != per_cb; ++i)
        if (!IsFinite(s[i])) s[i] = average;
    } else {
      size_t count = 0;
      double average[2] = {0.0, 0.0};
      for (size_t i = 0; i < per_cb; i += 2)
        if (IsFinite(s[i]) && IsFinite(s[i + 1])) {
          for (size_t p = 0; p != 2; ++p) average[p] += std::abs(s[i]);
          ++count;
        }
      if (count == 0) {
        average[0] = average[1] = 1.0;
      } else {
        for (size_t p = 0; p != 2; ++p) average[p] /= count;
      }
      for (size_t i = 0; i < per_cb; i += 2)
        if (!IsFinite(s[i]) || !IsFinite(s[i + 1]))
          for (size_t p = 0; p != 2; ++p) s[i + p] = average[p];
    }
  }
}

// SolverBase::Step (SolverBase.cc:88-158).
void Step(const std::vector<std::complex<double>>& sols,
          std::vector<std::complex<double>>& next, double step_size,
          bool phase_only) {
  for (size_t i = 0; i != next.size(); ++i) {
    if (!phase_only) {
      next[i] = sols[i] * (1.0 - step_size) + next[i] * step_size;
    } else {
      const double phase_from = std::arg(sols[i]);
      double distance = std::arg(next[i]) - phase_from;
      if (distance > M_PI)
        distance -= 2.0 * M_PI;
      else if (distance < -M_PI)
        distance += 2.0 * M_PI;
      next[i] = std::polar(1.0, phase_from + step_size * distance);
    }
  }
}

// SolverBase::AssignSolutions (SolverBase.cc:215-306) for 1 and 2 pols.
bool AssignSolutions(std::vector<std::complex<double>>& sols,
                     const std::vector<std::complex<double>>& next,
                     size_t n_pol, double step_size, double accuracy,
                     double constraint_accuracy, bool use_constraint_accuracy,
                     std::vector<double>& step_magnitudes) {
  double avg_abs_diff = 0.0;
  size_t n = 0;
  for (size_t i = 0; i < sols.size(); i += n_pol) {
    if (n_pol == 1) {
      if (sols[i] != 0.0) {
        const double a = std::abs((next[i] - sols[i]) / sols[i]);
        if (std::isfinite(a)) {
          avg_abs_diff += a;
          ++n;
        }
      }
    } else {
      const std::complex<double> s[2] = {sols[i], sols[i + 1]};
      const std::complex<double> s_inv[2] = {1.0 / s[0], 1.0 / s[1]};
      if (IsFinite(s_inv[0]) && IsFinite(s_inv[1])) {
        std::complex<double> ns[2] = {next[i], next[i + 1]};
        ns[0] = (ns[0] - s[0]) * s_inv[0];
        ns[1] = (ns[1] - s[1]) * s_inv[1];
        const double sumabs = std::abs(ns[0]) + std::abs(ns[1]);
        if (std::isfinite(sumabs)) {
          avg_abs_diff += sumabs;
          n += 2;
        }
      }
    }
  }
  std::copy(next.begin(), next.end(), sols.begin());
  const double step_magnitude = n == 0 ? 0 : avg_abs_diff / step_size / n;
  step_magnitudes.push_back(step_magnitude);
  return step_magnitude <=
         (use_constraint_accuracy ? constraint_accuracy : accuracy);
}

// SolverBase::DetectStall (SolverBase.cc:63-86).
struct StallState {
  size_t n_var_count = 0;
  double mean = 0, var = 0;
};
bool DetectStall(StallState& st, size_t iteration,
                 const std::vector<double>& mags, double sigma) {
  if (iteration == 1) {
    st.n_var_count = 1;
    st.mean = mags[iteration - 1];
    st.var = 0.0;
  } else {
    st.n_var_count += 1;
    const double delta_1 = mags[iteration - 1] - st.mean;
    st.mean += delta_1 / double(st.n_var_count);
    const double delta_2 = mags[iteration - 1] - st.mean;
    st.var += delta_1 * delta_2;
  }
  if (iteration < 30) return false;
  return st.mean < sigma * std::sqrt(st.var / double(st.n_var_count));
}

// IterativeDiagonalSolver::Solve (IterativeDiagonalSolver.cc:38-97) /
// IterativeScalarSolver::Solve (IterativeScalarSolver.cc:30-89), without
// constraints (ApplyConstraints then returns true, SolverBase.cc:174-190).
template <typename T, int NCorr, int NPol, typename Acc>
void SolveLoop(const Problem& pr, const oracle_settings& st, size_t n_threads,
               std::vector<std::complex<double>>& sols,
               std::vector<double>& step_magnitudes, oracle_result& res) {
  const size_t per_cb = pr.n_ant * pr.n_sub * NPol;
  std::vector<std::complex<double>> next(sols.size());
  size_t iteration = 0;
  bool has_converged = false, has_stalled = false;
  const bool constraints_satisfied = true;
  StallState stall;
  step_magnitudes.clear();
  do {
    MakeSolutionsFinite(sols, pr.n_cb, per_cb, NPol);
    PerformIterationAll<T, NCorr, NPol, Acc>(pr, n_threads, sols, next);
    Step(sols, next, st.step_size, st.phase_only != 0);
    has_converged = AssignSolutions(sols, next, NPol, st.step_size,
                                    st.accuracy, st.constraint_accuracy,
                                    !constraints_satisfied, step_magnitudes);
    ++iteration;
    // ReachedStoppingCriterion (SolverBase.h:274-285)
    has_stalled = false;
    if (st.detect_stalling && constraints_satisfied)
      has_stalled =
          DetectStall(stall, iteration, step_magnitudes, st.step_diff_sigma);
    const bool is_ready = iteration >= st.max_iterations ||
                          (has_converged && constraints_satisfied) ||
                          has_stalled;
    if (iteration >= st.min_iterations && is_ready) break;
  } while (true);
  // MakeResult (SolverBase.cc:192-213)
  res.iterations = uint32_t(has_converged && constraints_satisfied
                                ? iteration
                                : iteration + 1);
  res.constraint_iterations = constraints_satisfied ? 0 : uint32_t(iteration + 1);
  res.has_converged = has_converged;
  res.has_stalled = has_stalled;
}

template <typename Fn>
int Dispatch(const Problem& pr, int precision, Fn&& fn) {
#define DDO_CASE(NC, NP)                                        \
  if (pr.n_corr == NC && pr.n_pol == NP) {                      \
    if (precision == 64) {                                      \
      fn.template operator()<double, NC, NP, double>();         \
    } else if (NP == 2) {                                       \
      fn.template operator()<float, NC, NP, float>();           \
    } else {                                                    \
      fn.template operator()<float, NC, NP, double>();          \
    }                                                           \
    return 0;                                                   \
  }
  DDO_CASE(2, 2)
  DDO_CASE(4, 2)
  DDO_CASE(1, 1)
  DDO_CASE(2, 1)
  DDO_CASE(4, 1)
#undef DDO_CASE
  return 1;
}

}  // namespace

extern "C" int oracle_perform_iteration(const oracle_dims* dims,
                                        const oracle_channel_block* cbs,
                                        int precision, int n_threads,
                                        const double* solutions,
                                        double* next_solutions) {
  const Problem pr = MakeProblem(dims, cbs);
  const size_t total = pr.n_cb * pr.n_ant * pr.n_sub * pr.n_pol;
  std::vector<std::complex<double>> sols(
      reinterpret_cast<const std::complex<double>*>(solutions),
      reinterpret_cast<const std::complex<double>*>(solutions) + total);
  std::vector<std::complex<double>> next(total);
  const int rc = Dispatch(pr, precision, [&]<typename T, int NC, int NP,
                                             typename Acc>() {
    PerformIterationAll<T, NC, NP, Acc>(pr, std::max(1, n_threads), sols, next);
  });
  if (rc == 0)
    std::memcpy(next_solutions, next.data(), total * sizeof(std::complex<double>));
  return rc;
}

extern "C" int oracle_solve(const oracle_dims* dims,
                            const oracle_settings* settings,
                            const oracle_channel_block* cbs, int precision,
                            int n_threads, double* solutions,
                            double* step_magnitudes, oracle_result* result) {
  const Problem pr = MakeProblem(dims, cbs);
  const size_t total = pr.n_cb * pr.n_ant * pr.n_sub * pr.n_pol;
  std::complex<double>* sol_ptr =
      reinterpret_cast<std::complex<double>*>(solutions);
  std::vector<std::complex<double>> sols(sol_ptr, sol_ptr + total);
  std::vector<double> mags;
  oracle_result res{};
  const int rc = Dispatch(pr, precision, [&]<typename T, int NC, int NP,
                                             typename Acc>() {
    SolveLoop<T, NC, NP, Acc>(pr, *settings, std::max(1, n_threads), sols, mags,
                              res);
  });
  if (rc != 0) return rc;
  std::copy(sols.begin(), sols.end(), sol_ptr);
  if (step_magnitudes)
    std::copy(mags.begin(), mags.end(), step_magnitudes);
  if (result) *result = res;
  return 0;
}

// ---------------------------------------------------------------------------
// SolverTester restated (ddecal/test/unit/SolverTester.{h,cc}).
// ---------------------------------------------------------------------------
namespace {
constexpr size_t kNAntennas = 50;
constexpr size_t kNDirections = 3;
constexpr size_t kNChannels = 16;
constexpr size_t kNChannelBlocks = 4;
constexpr size_t kNRegularTimes = 50;
constexpr size_t kNBaselines = kNAntennas * (kNAntennas - 1) / 2;
constexpr size_t kDDSolutionsPerDirection[kNDirections] = {1, 2, 5};
}  // namespace

extern "C" int oracle_solver_tester_fill(int diagonal, int dd_intervals,
                                         uint32_t n_correlations, float** data,
                                         float** model,
                                         uint32_t** antenna_pairs,
                                         uint32_t** solution_map,
                                         double* input_solutions_out) {
  if (n_correlations != 1 && n_correlations != 2 && n_correlations != 4)
    return 1;
  // InitializeNSolutions (SolverTester.cc:313-323)
  std::vector<size_t> n_sol_per_dir(kNDirections, 1);
  if (dd_intervals)
    n_sol_per_dir.assign(std::begin(kDDSolutionsPerDirection),
                         std::end(kDDSolutionsPerDirection));
  const size_t n_solutions =
      std::accumulate(n_sol_per_dir.begin(), n_sol_per_dir.end(), size_t(0));

  // SetScalarSolutions / SetDiagonalSolutions (SolverTester.cc:331-363)
  std::vector<std::complex<float>> input_solutions(kNAntennas * n_solutions * 2);
  {
    std::mt19937 mt;
    std::uniform_real_distribution<float> uniform_sols(1.0, 2.0);
    if (diagonal) {
      for (size_t ant = 0; ant != kNAntennas; ++ant)
        for (size_t pol = 0; pol != 2; ++pol)
          for (size_t s = 0; s != n_solutions; ++s) {
            const size_t index = (ant * n_solutions + s) * 2 + pol;
            input_solutions[index] = {uniform_sols(mt), uniform_sols(mt)};
            if (s != 0) input_solutions[index] *= 0.5f;
          }
    } else {
      for (size_t ant = 0; ant != kNAntennas; ++ant)
        for (size_t s = 0; s != n_solutions; ++s) {
          const size_t index = (ant * n_solutions + s) * 2;
          input_solutions[index] = {uniform_sols(mt), uniform_sols(mt)};
          if (s != 0) input_solutions[index] *= 0.5f;
          input_solutions[index + 1] = input_solutions[index];
        }
    }
  }
  for (size_t i = 0; i != input_solutions.size(); ++i) {
    input_solutions_out[2 * i] = input_solutions[i].real();
    input_solutions_out[2 * i + 1] = input_solutions[i].imag();
  }

  // FillDdIntervalData (SolverTester.cc:95-202), non-leakage branch.
  std::uniform_real_distribution<float> uniform_data(-1.0, 1.0);
  std::mt19937 mt(0);
  std::vector<std::vector<size_t>> solution_indices(kNDirections);
  size_t first_solution_index = 0;
  for (size_t d = 0; d != kNDirections; ++d) {
    solution_indices[d].resize(kNRegularTimes);
    for (size_t t = 0; t != kNRegularTimes; ++t)
      solution_indices[d][t] =
          first_solution_index + t * n_sol_per_dir[d] / kNRegularTimes;
    first_solution_index += n_sol_per_dir[d];
  }

  // Channel split of the regular SolveData constructor (SolveData.cc:112-113)
  std::vector<size_t> channel_begin(kNChannelBlocks + 1, 0);
  for (size_t cb = 0; cb != kNChannelBlocks; ++cb)
    channel_begin[cb + 1] = (cb + 1) * kNChannels / kNChannelBlocks;

  std::vector<std::complex<float>> dir_data(kNDirections * kNBaselines *
                                            kNChannels * 4);
  std::vector<std::complex<float>> time_data(kNBaselines * kNChannels * 4);
  std::vector<size_t> vis_index(kNChannelBlocks, 0);
  std::vector<size_t> n_vis_cb(kNChannelBlocks);
  for (size_t cb = 0; cb != kNChannelBlocks; ++cb)
    n_vis_cb[cb] =
        kNRegularTimes * kNBaselines * (channel_begin[cb + 1] - channel_begin[cb]);

  auto to_specific = [&](const std::complex<float>* m, float* out) {
    // ToSpecificMatrix (SolveData.cc:18-31)
    if (n_correlations == 4) {
      for (int i = 0; i < 4; ++i) {
        out[2 * i] = m[i].real();
        out[2 * i + 1] = m[i].imag();
      }
    } else if (n_correlations == 2) {
      out[0] = m[0].real();
      out[1] = m[0].imag();
      out[2] = m[3].real();
      out[3] = m[3].imag();
    } else {
      const std::complex<float> v = 0.5f * (m[0] + m[3]);
      out[0] = v.real();
      out[1] = v.imag();
    }
  };

  for (size_t timestep = 0; timestep != kNRegularTimes; ++timestep) {
    for (size_t d = 0; d != kNDirections; ++d) {
      std::complex<float>* this_direction =
          &dir_data[d * kNBaselines * kNChannels * 4];
      for (size_t bl = 0; bl != kNBaselines; ++bl) {
        for (size_t ch = 0; ch != kNChannels; ++ch) {
          const size_t matrix_index = (bl * kNChannels + ch) * 4;
          this_direction[matrix_index + 0] =
              std::complex<float>(uniform_data(mt), uniform_data(mt));
          this_direction[matrix_index + 1] =
              std::complex<float>(uniform_data(mt), uniform_data(mt)) * 0.1f;
          this_direction[matrix_index + 2] =
              std::complex<float>(uniform_data(mt), uniform_data(mt)) * 0.1f;
          this_direction[matrix_index + 3] =
              std::complex<float>(uniform_data(mt), uniform_data(mt)) * 1.5f;
        }
      }
    }
    size_t baseline_index = 0;
    for (size_t a1 = 0; a1 != kNAntennas; ++a1) {
      for (size_t a2 = a1 + 1; a2 != kNAntennas; ++a2) {
        for (size_t ch = 0; ch != kNChannels; ++ch) {
          // perturbed_model = sum_d diag(g_a1) * M * diag(g_a2)^H, in FP64
          // (aocommon::MC2x2 / MC2x2Diag are double precision).
          std::complex<double> pm[4] = {0, 0, 0, 0};
          for (size_t d = 0; d != kNDirections; ++d) {
            const size_t s = solution_indices[d][timestep];
            const std::complex<float>* v =
                &dir_data[(d * kNBaselines + baseline_index) * kNChannels * 4 +
                          ch * 4];
            const std::complex<double> l0 =
                input_solutions[(a1 * n_solutions + s) * 2 + 0];
            const std::complex<double> l1 =
                input_solutions[(a1 * n_solutions + s) * 2 + 1];
            const std::complex<double> r0 =
                input_solutions[(a2 * n_solutions + s) * 2 + 0];
            const std::complex<double> r1 =
                input_solutions[(a2 * n_solutions + s) * 2 + 1];
            // val.MultiplyHerm(right) = val * right^H, right = diag(r0, r1)
            const std::complex<double> vh[4] = {
                std::complex<double>(v[0]) * std::conj(r0),
                std::complex<double>(v[1]) * std::conj(r1),
                std::complex<double>(v[2]) * std::conj(r0),
                std::complex<double>(v[3]) * std::conj(r1)};
            pm[0] += l0 * vh[0];
            pm[1] += l0 * vh[1];
            pm[2] += l1 * vh[2];
            pm[3] += l1 * vh[3];
          }
          for (size_t p = 0; p != 4; ++p)
            time_data[(baseline_index * kNChannels + ch) * 4 + p] =
                std::complex<float>(pm[p]);
        }
        ++baseline_index;
      }
    }
    // AssignAndWeight with unit weights and no flags multiplies by sqrt(1)
    // (SolverTools.cc:81-167): the identity. Then the regular SolveData
    // constructor (SolveData.cc:129-185) packs time -> baseline -> channel.
    for (size_t bl = 0; bl != kNBaselines; ++bl) {
      // Antenna numbering of the SolverTester (SolverTester.cc:75-80)
      size_t a1 = 0, rem = bl;
      while (rem >= kNAntennas - 1 - a1) {
        rem -= kNAntennas - 1 - a1;
        ++a1;
      }
      const size_t a2 = a1 + 1 + rem;
      for (size_t cb = 0; cb != kNChannelBlocks; ++cb) {
        size_t& vi = vis_index[cb];
        const size_t first = channel_begin[cb];
        const size_t size = channel_begin[cb + 1] - first;
        for (size_t i = 0; i != size; ++i) {
          to_specific(&time_data[(bl * kNChannels + first + i) * 4],
                      data[cb] + (vi + i) * n_correlations * 2);
          antenna_pairs[cb][2 * (vi + i)] = uint32_t(a1);
          antenna_pairs[cb][2 * (vi + i) + 1] = uint32_t(a2);
        }
        size_t start = 0;
        for (size_t d = 0; d != kNDirections; ++d) {
          const size_t sol_index = timestep * n_sol_per_dir[d] / kNRegularTimes + start;
          start += n_sol_per_dir[d];
          for (size_t i = 0; i != size; ++i) {
            to_specific(&dir_data[(d * kNBaselines + bl) * kNChannels * 4 +
                                  (first + i) * 4],
                        model[cb] + (d * n_vis_cb[cb] + vi + i) * n_correlations * 2);
            solution_map[cb][d * n_vis_cb[cb] + vi + i] = uint32_t(sol_index);
          }
        }
        vi += size;
      }
    }
  }
  return 0;
}
