// One regular solution interval handed to DP3's own solver code: the C
// structs of the reference-code oracle's entry points and the two steps that
// every caller of DP3's solvers takes -- packing the interval into DPBuffers
// and through the reference's regular SolveData constructor
// (ddecal/gain_solvers/SolveData.cc:77-188), and configuring a SolverBase the
// way DDECal's SolverFactory does (SolverFactory.cc:49-146, 276-290:
// Initialize, the setters, AddConstraint + Constraint::Initialize).
//
// TEST INFRASTRUCTURE ONLY: shared by the reference-code oracle
// (oracle/ref_harness.cc) and the test harness of the DP3 adapter
// (tests/adapter/adapter_harness.cc). Compiled against DP3's sources.
#ifndef DP3B200_ORACLE_REF_PROBLEM_H
#define DP3B200_ORACLE_REF_PROBLEM_H

#include <algorithm>
#include <complex>
#include <cstdint>
#include <memory>
#include <numeric>
#include <set>
#include <string>
#include <vector>

#include "ddecal/constraints/AntennaConstraint.h"
#include "ddecal/constraints/SmoothnessConstraint.h"
#include "ddecal/gain_solvers/SolveData.h"
#include "ddecal/gain_solvers/SolverBase.h"

extern "C" {

enum {
  REF_DIAGONAL_DUO = 0,   // IterativeDiagonalSolver<MC2x2FDiag>
  REF_DIAGONAL_FULL = 1,  // IterativeDiagonalSolver<MC2x2F>
  REF_SCALAR_UNI = 2,     // IterativeScalarSolver<std::complex<float>>
  REF_SCALAR_DUO = 3,     // IterativeScalarSolver<MC2x2FDiag>
  REF_SCALAR_FULL = 4,    // IterativeScalarSolver<MC2x2F>
  REF_FULL_JONES = 5,     // IterativeFullJonesSolver (MC2x2F data, 2x2 gains)
};

typedef struct {
  uint32_t n_antennas, n_times, n_baselines, n_channels, n_channel_blocks, n_directions;
  uint32_t n_correlations_in;                 // 1, 2 (XX, YY) or 4 per input visibility
  const uint32_t* n_solutions_per_direction;  // [n_directions]
  const int32_t* antenna1;                    // [n_baselines]
  const int32_t* antenna2;
  // Per channel block cb (channels [cb n_ch / n_cb, (cb + 1) n_ch / n_cb)):
  //   data[cb]  float [n_times][n_baselines][n_ch_cb][n_correlations_in][2]
  //   model[cb] float [n_directions][n_times][n_baselines][n_ch_cb][n_corr_in][2]
  const float* const* data;
  const float* const* model;
} ref_problem;

typedef struct {
  uint32_t max_iterations;
  uint32_t min_iterations;
  double accuracy;
  double constraint_accuracy;
  double step_size;
  int32_t detect_stalling;
  double step_diff_sigma;
  int32_t phase_only;
} ref_settings;

typedef struct {
  // AntennaConstraint: n_antenna_sets sets, set k has antenna_set_sizes[k]
  // members, listed consecutively in antenna_set_members.
  uint32_t n_antenna_sets;
  const uint32_t* antenna_set_sizes;
  const uint32_t* antenna_set_members;
  // SmoothnessConstraint (when smoothness != 0).
  int32_t smoothness;
  double bandwidth_hz;
  double bandwidth_ref_frequency_hz;
  double spectral_exponent;
  int32_t kernel_truncation;
  const double* smoothness_weights;  // [n_antennas * n_channel_blocks] or NULL (all 1)
  // Mean frequency of each channel block (Constraint::Initialize).
  const double* channel_block_frequencies;  // [n_channel_blocks]
  // SmoothnessConstraint::SetAntennaFactors [n_antennas] or NULL (all 1),
  // SetDdSmoothingFactors [n_sub_solutions] or NULL (none), and
  // SetSubSolutionWeights [n_sub_solutions][n_antennas * n_channel_blocks]
  // or NULL (none).
  const double* antenna_factors;
  const double* dd_factors;
  const double* sub_solution_weights;
  // Appends a constraint whose Apply is Constraint::ApplyReferenceAntenna
  // (the phase referencing of DP3's TEC constraints).
  int32_t reference_antenna;
} ref_constraints;

typedef struct {
  uint32_t iterations;
  uint32_t constraint_iterations;
  double seconds_packing;  // DPBuffers -> SolveData (the reference constructor)
  double seconds_solve;    // Solve()
} ref_result;

}  // extern "C"

namespace dp3b200_ref {

// DPBuffers of the interval -> SolveData<V> through the reference's regular
// constructor.
template <typename V>
dp3::ddecal::SolveData<V> Pack(const ref_problem& p) {
  using dp3::base::DPBuffer;
  const size_t n_corr = p.n_correlations_in;
  std::vector<std::string> names;
  for (uint32_t d = 0; d < p.n_directions; ++d) names.push_back("direction" + std::to_string(d));
  std::vector<DPBuffer> buffers(p.n_times);
  for (uint32_t t = 0; t < p.n_times; ++t) {
    DPBuffer& b = buffers[t];
    auto fill = [&](DPBuffer::DataType& cube, const float* const* src, size_t dir) {
      for (uint32_t cb = 0; cb < p.n_channel_blocks; ++cb) {
        const size_t c0 = size_t(cb) * p.n_channels / p.n_channel_blocks;
        const size_t c1 = size_t(cb + 1) * p.n_channels / p.n_channel_blocks;
        const size_t L = c1 - c0;
        const float* s = src[cb] + (dir * p.n_times + t) * p.n_baselines * L * n_corr * 2;
        for (uint32_t bl = 0; bl < p.n_baselines; ++bl)
          for (size_t c = 0; c < L; ++c) {
            const float* v = s + (size_t(bl) * L + c) * n_corr * 2;
            std::complex<float>* out = &cube(bl, c0 + c, 0);
            if (n_corr == 4) {
              for (int k = 0; k < 4; ++k) out[k] = {v[2 * k], v[2 * k + 1]};
            } else if (n_corr == 2) {
              out[0] = {v[0], v[1]};
              out[1] = out[2] = 0.f;
              out[3] = {v[2], v[3]};
            } else {
              out[0] = out[3] = {v[0], v[1]};
              out[1] = out[2] = 0.f;
            }
          }
      }
    };
    fill(b.AddData("", p.n_baselines, p.n_channels, 4), p.data, 0);
    for (uint32_t d = 0; d < p.n_directions; ++d)
      fill(b.AddData(names[d], p.n_baselines, p.n_channels, 4), p.model, d);
  }
  const std::vector<size_t> nspd(p.n_solutions_per_direction,
                                 p.n_solutions_per_direction + p.n_directions);
  const std::vector<int> a1(p.antenna1, p.antenna1 + p.n_baselines);
  const std::vector<int> a2(p.antenna2, p.antenna2 + p.n_baselines);
  return dp3::ddecal::SolveData<V>(std::move(buffers), names, p.n_channel_blocks, p.n_antennas,
                                   nspd, a1, a2);
}

// A constraint that only phase-references the solutions
// (Constraint::ApplyReferenceAntenna, Constraint.cc:7-37), as DP3's TEC
// constraints do when phase referencing is on.
class ReferenceAntennaConstraint final : public dp3::ddecal::Constraint {
 public:
  void Apply(dp3::ddecal::SolutionSpan& solutions, double) override {
    ApplyReferenceAntenna(solutions);
  }
};

// Initialize, setters and constraints, as SolverFactory does. Smoothness: the
// smoothness constraint class (DP3's, or one with the same constructor and
// setters).
template <typename Smoothness = dp3::ddecal::SmoothnessConstraint>
inline void Configure(dp3::ddecal::SolverBase& solver, const ref_problem& p,
                      const ref_settings& s, const ref_constraints* c) {
  std::vector<size_t> nspd(p.n_solutions_per_direction,
                           p.n_solutions_per_direction + p.n_directions);
  solver.Initialize(p.n_antennas, nspd, p.n_channel_blocks);
  solver.SetMaxIterations(s.max_iterations);
  solver.SetMinIterations(s.min_iterations);
  solver.SetAccuracy(s.accuracy);
  solver.SetConstraintAccuracy(s.constraint_accuracy);
  solver.SetStepSize(s.step_size);
  solver.SetDetectStalling(s.detect_stalling != 0, s.step_diff_sigma);
  solver.SetPhaseOnly(s.phase_only != 0);
  if (!c) return;
  std::vector<uint32_t> spd(p.n_solutions_per_direction,
                            p.n_solutions_per_direction + p.n_directions);
  std::vector<double> freqs(c->channel_block_frequencies,
                            c->channel_block_frequencies + p.n_channel_blocks);
  if (c->n_antenna_sets) {
    auto ac = std::make_unique<dp3::ddecal::AntennaConstraint>();
    std::vector<std::set<size_t>> sets(c->n_antenna_sets);
    size_t k = 0;
    for (uint32_t i = 0; i < c->n_antenna_sets; ++i)
      for (uint32_t j = 0; j < c->antenna_set_sizes[i]; ++j)
        sets[i].insert(c->antenna_set_members[k++]);
    ac->SetAntennaSets(std::move(sets));
    ac->Initialize(p.n_antennas, spd, freqs);
    solver.AddConstraint(std::move(ac));
  }
  if (c->smoothness) {
    auto sc = std::make_unique<Smoothness>(
        c->bandwidth_hz, c->bandwidth_ref_frequency_hz, c->spectral_exponent,
        c->kernel_truncation != 0);
    sc->Initialize(p.n_antennas, spd, freqs);
    std::vector<double> w(size_t(p.n_antennas) * p.n_channel_blocks, 1.0);
    if (c->smoothness_weights) std::copy_n(c->smoothness_weights, w.size(), w.begin());
    sc->SetWeights(w);
    std::vector<double> af(p.n_antennas, 1.0);
    if (c->antenna_factors) std::copy_n(c->antenna_factors, af.size(), af.begin());
    sc->SetAntennaFactors(std::move(af));
    size_t n_sub = 0;
    for (uint32_t d = 0; d < p.n_directions; ++d) n_sub += p.n_solutions_per_direction[d];
    if (c->dd_factors)
      sc->SetDdSmoothingFactors(std::vector<double>(c->dd_factors, c->dd_factors + n_sub));
    if (c->sub_solution_weights) {
      std::vector<std::vector<double>> sw(n_sub);
      for (size_t s = 0; s < n_sub; ++s)
        sw[s].assign(c->sub_solution_weights + s * w.size(),
                     c->sub_solution_weights + (s + 1) * w.size());
      sc->SetSubSolutionWeights(sw);
    }
    solver.AddConstraint(std::move(sc));
  }
  if (c->reference_antenna) {
    auto rc = std::make_unique<ReferenceAntennaConstraint>();
    rc->Initialize(p.n_antennas, spd, freqs);
    solver.AddConstraint(std::move(rc));
  }
}

// Copies between the flat [cb][ant][sub][pol] complex128 array and the
// solver's std::vector<std::vector<std::complex<double>>>.
inline std::vector<std::vector<std::complex<double>>> ToVectors(const double* flat, size_t n_cb,
                                                               size_t per_cb) {
  std::vector<std::vector<std::complex<double>>> v(n_cb);
  for (size_t cb = 0; cb < n_cb; ++cb) {
    v[cb].resize(per_cb);
    std::copy_n(reinterpret_cast<const std::complex<double>*>(flat) + cb * per_cb, per_cb,
                v[cb].begin());
  }
  return v;
}

inline void FromVectors(const std::vector<std::vector<std::complex<double>>>& v, double* flat) {
  size_t off = 0;
  for (const auto& cb : v) {
    std::copy(cb.begin(), cb.end(), reinterpret_cast<std::complex<double>*>(flat) + off);
    off += cb.size();
  }
}

}  // namespace dp3b200_ref

#endif
