// IterativeSolverB200 -- DP3's direction-iterative diagonal / scalar gain
// solvers on a B200, behind DP3's own dp3::ddecal::SolverBase.
//
// Drop-in for IterativeDiagonalSolver<V> (NPol = 2,
// ddecal/gain_solvers/IterativeDiagonalSolver.h:13-41) and
// IterativeScalarSolver<V> (NPol = 1, IterativeScalarSolver.h:15-49):
// the same virtual surface (SolverBase.h:76-78, 205-227), so that DDECal's
// SolverFactory (ddecal/SolverFactory.cc:49-146) can return it and
// DDECal::doSolve (steps/DDECal.cc:655-699) calls it unchanged. The work goes
// through the C ABI of libddsolve_b200.so (include/ddsolve_b200.h); no
// exception crosses that ABI, failures come back as status codes and are
// rethrown here as std::runtime_error, as the reference throws.
//
// Solve without constraints: the whole iterate-until-converged loop runs on
// the device (ddsolve_solve). DP3's SolverBase keeps the stall-detection
// sigma private without a getter (SolverBase.h:160-164), so the device loop
// runs without stall detection and this class evaluates DP3's own stopping
// rule (SolverBase::ReachedStoppingCriterion -> DetectStall) on the host over
// the per-iteration step magnitudes the device returns; where DP3 would have
// stopped earlier on a stall, the device solve is repeated from the same
// initial solutions with the iteration cap at that iteration, which gives
// the solutions and the result of the stalled solve.
//
// Solve with constraints that all have a device form (DP3's AntennaConstraint
// and SmoothnessConstraintB200 below): they become device constraints
// (ddsolve_add_*_constraint) and the whole constrained loop runs on the
// device as above. Otherwise DP3's own loop (IterativeDiagonalSolver.cc:
// 38-97) on the host -- MakeSolutionsFinite, Step, ApplyConstraints,
// AssignSolutions and ReachedStoppingCriterion are SolverBase's own -- with
// PerformIteration replaced by one device pass (ddsolve_perform_iteration).
//
// The Solve(data, solutions, time, stat_stream) overload writes one line
// "iteration step_magnitude" per iteration to stat_stream (cf. the
// statistics stream of IterativeDiagonalSolverCuda.h:23-25).
#ifndef DP3B200_ITERATIVE_SOLVER_B200_H
#define DP3B200_ITERATIVE_SOLVER_B200_H

#include <algorithm>
#include <complex>
#include <cstring>
#include <ostream>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include <aocommon/matrix2x2.h>
#include <aocommon/matrix2x2diag.h>

#include "ddsolve_b200.h"
#include "ddecal/constraints/AntennaConstraint.h"
#include "ddecal/constraints/SmoothnessConstraint.h"
#include "ddecal/gain_solvers/SolveData.h"
#include "ddecal/gain_solvers/SolverBase.h"

// Progress hook (a no-op unless the includer defines it, e.g. a test
// harness that logs where a solve is).
#ifndef DP3B200_ADAPTER_TRACE
#define DP3B200_ADAPTER_TRACE(what) ((void)0)
#endif

namespace dp3::ddecal {

// DP3's SmoothnessConstraint with a device form. The same constructor and
// setters (SmoothnessConstraint.h:18-75); Apply runs DP3's own
// SmoothnessConstraint on the host (the host loop of IterativeSolverB200),
// and IterativeSolverB200 hands the same settings to the device
// (ddsolve_add_smoothness_constraint) when every constraint of a solve has a
// device form, so that the constrained loop stays on the GPU. DP3's class is
// final and keeps its settings private, hence a wrapper: SolverFactory
// creates it in place of SmoothnessConstraint together with the B200 solver.
class SmoothnessConstraintB200 final : public Constraint {
 public:
  SmoothnessConstraintB200(double bandwidth_hz, double bandwidth_ref_frequency_hz,
                           double spectral_exponent, bool kernel_truncation)
      : host_(bandwidth_hz, bandwidth_ref_frequency_hz, spectral_exponent, kernel_truncation),
        bandwidth_hz_(bandwidth_hz),
        bandwidth_ref_frequency_hz_(bandwidth_ref_frequency_hz),
        spectral_exponent_(spectral_exponent),
        kernel_truncation_(kernel_truncation) {}

  void Initialize(size_t n_antennas, const std::vector<uint32_t>& solutions_per_direction,
                  const std::vector<double>& frequencies) override {
    Constraint::Initialize(n_antennas, solutions_per_direction, frequencies);
    host_.Initialize(n_antennas, solutions_per_direction, frequencies);
    frequencies_ = frequencies;
  }
  void SetWeights(const std::vector<double>& weights) override {
    host_.SetWeights(weights);
    weights_ = weights;
  }
  void SetSubSolutionWeights(const std::vector<std::vector<double>>& weights) override {
    host_.SetSubSolutionWeights(weights);
    sub_solution_weights_ = weights;
  }
  void SetAntennaFactors(std::vector<double>&& antenna_factors) {
    antenna_factors_ = antenna_factors;
    host_.SetAntennaFactors(std::move(antenna_factors));
  }
  const std::vector<double>& GetAntennaFactors() const { return antenna_factors_; }
  void SetDdSmoothingFactors(std::vector<double> dd_smoothing_factors) {
    host_.SetDdSmoothingFactors(dd_smoothing_factors);  // checks the size
    dd_factors_ = std::move(dd_smoothing_factors);
  }
  const std::vector<double>& GetDdSmoothingFactors() const { return dd_factors_; }

  void Apply(SolutionSpan& solutions, double time) override { host_.Apply(solutions, time); }

  // Adds the device form to a context (status of the C ABI call).
  int AddTo(ddsolve_ctx* ctx) const {
    std::vector<double> flat_sub;
    for (const std::vector<double>& w : sub_solution_weights_)
      flat_sub.insert(flat_sub.end(), w.begin(), w.end());
    ddsolve_smoothness s{};
    s.frequencies = frequencies_.data();
    s.bandwidth_hz = bandwidth_hz_;
    s.bandwidth_ref_frequency_hz = bandwidth_ref_frequency_hz_;
    s.spectral_exponent = spectral_exponent_;
    s.kernel_truncation = kernel_truncation_ ? 1 : 0;
    s.weights = weights_.empty() ? nullptr : weights_.data();
    s.sub_solution_weights = flat_sub.empty() ? nullptr : flat_sub.data();
    s.antenna_factors = antenna_factors_.empty() ? nullptr : antenna_factors_.data();
    s.dd_factors = dd_factors_.empty() ? nullptr : dd_factors_.data();
    return ddsolve_add_smoothness_constraint(ctx, &s);
  }

 private:
  SmoothnessConstraint host_;
  double bandwidth_hz_, bandwidth_ref_frequency_hz_, spectral_exponent_;
  bool kernel_truncation_;
  std::vector<double> frequencies_, weights_, antenna_factors_, dd_factors_;
  std::vector<std::vector<double>> sub_solution_weights_;
};

template <typename VisMatrix, size_t NPol>
class IterativeSolverB200 final : public SolverBase {
  static_assert(NPol == 1 || NPol == 2 || NPol == 4,
                "scalar (1), diagonal (2) or full-Jones (4) solutions");
  static_assert(NPol == 1 || !std::is_same_v<VisMatrix, std::complex<float>>,
                "the diagonal solver needs 2 or 4 correlations");
  static_assert(NPol != 4 || std::is_same_v<VisMatrix, aocommon::MC2x2F>,
                "the full-Jones solver needs 4 correlations");

 public:
  explicit IterativeSolverB200(int device = 0) : device_(device) {}
  ~IterativeSolverB200() override { ddsolve_destroy(ctx_); }
  IterativeSolverB200(const IterativeSolverB200&) = delete;
  IterativeSolverB200& operator=(const IterativeSolverB200&) = delete;

  void Initialize(size_t n_antennas, const std::vector<size_t>& n_solutions_per_direction,
                  size_t n_channel_blocks) override {
    SolverBase::Initialize(n_antennas, n_solutions_per_direction, n_channel_blocks);
    n_solutions_per_direction_.assign(n_solutions_per_direction.begin(),
                                      n_solutions_per_direction.end());
    ddsolve_destroy(ctx_);  // dimensions changed: a new context on the next Solve
    ctx_ = nullptr;
  }

  size_t NSolutionPolarizations() const override { return NPol; }
  bool SupportsDdSolutionIntervals() const override { return true; }

  SolveResult Solve(const SolveData<VisMatrix>& data,
                    std::vector<std::vector<DComplex>>& solutions, double time) override {
    return Solve(data, solutions, time, nullptr);
  }

  SolveResult Solve(const SolveData<VisMatrix>& data,
                    std::vector<std::vector<DComplex>>& solutions, double time,
                    std::ostream* stat_stream) {
    Upload(data);
    // (the full-Jones device path has no device constraints)
    const bool device_loop = NPol == 4 ? GetConstraints().empty() : UploadDeviceConstraints();
    if (device_loop) return SolveOnDevice(solutions, stat_stream);
    return SolveWithHostConstraints(solutions, time, stat_stream);
  }

  /// The step after the solve on the GPU, for one time step of an interval:
  /// DDECal::CorrectAndSubtractModels (steps/DDECal.cc:1081-1125) with
  /// ApplySolutionAndSubtract (:1031-1079) through
  /// ddsolve_correct_and_subtract. data: the step's DPBuffer data
  /// [baseline][channel][4]; models: every direction's model buffer of that
  /// step (DPBuffer::GetData(direction name)), same shape; antenna1 /
  /// antenna2: DDECal's antennas per baseline (autocorrelations included).
  /// With subtract, data -= the sum of the corrected models; with
  /// keep_model_data, each model buffer is replaced by its corrected model.
  /// Throws as the reference does for direction-dependent intervals.
  void CorrectAndSubtract(const std::vector<std::vector<DComplex>>& solutions,
                          size_t n_baselines, size_t n_channels,
                          const std::vector<uint32_t>& antenna1,
                          const std::vector<uint32_t>& antenna2, std::complex<float>* data,
                          const std::vector<std::complex<float>*>& models, bool subtract,
                          bool keep_model_data) {
    if (models.size() != n_solutions_per_direction_.size() ||
        antenna1.size() != n_baselines || antenna2.size() != n_baselines)
      throw std::runtime_error("B200 solver: CorrectAndSubtract arguments do not match");
    EnsureContext();
    const std::vector<double> flat = Flatten(solutions);
    std::vector<const float*> in(models.size());
    std::vector<float*> out(models.size());
    for (size_t d = 0; d != models.size(); ++d) {
      in[d] = reinterpret_cast<const float*>(models[d]);
      out[d] = reinterpret_cast<float*>(models[d]);
    }
    ddsolve_subtract_buffers b{};
    b.n_times = 1;
    b.n_baselines = uint32_t(n_baselines);
    b.n_channels = uint32_t(n_channels);
    b.antenna1 = antenna1.data();
    b.antenna2 = antenna2.data();
    b.data = reinterpret_cast<const float*>(data);
    b.models = in.data();
    Check(ddsolve_correct_and_subtract(ctx_, &b, flat.data(),
                                       subtract ? reinterpret_cast<float*>(data) : nullptr,
                                       keep_model_data ? out.data() : nullptr));
  }

 private:
  static constexpr uint32_t kNCorrelations =
      std::is_same_v<VisMatrix, aocommon::MC2x2F>       ? 4
      : std::is_same_v<VisMatrix, aocommon::MC2x2FDiag> ? 2
                                                         : 1;
  static_assert(sizeof(VisMatrix) == kNCorrelations * sizeof(std::complex<float>),
                "visibilities must be packed complex<float> values");

  void Check(int rc) const {
    if (rc != DDSOLVE_OK)
      throw std::runtime_error(std::string("B200 solver: ") + ddsolve_last_error(ctx_));
  }

  void EnsureContext() {
    if (ctx_) return;
    const ddsolve_dims dims{uint32_t(NAntennas()),
                            uint32_t(n_solutions_per_direction_.size()),
                            uint32_t(NChannelBlocks()),
                            kNCorrelations,
                            uint32_t(NPol),
                            n_solutions_per_direction_.data()};
    Check(ddsolve_create(&dims, device_, &ctx_));
    DP3B200_ADAPTER_TRACE("context created");
  }

  void Upload(const SolveData<VisMatrix>& data) {
    if (data.NChannelBlocks() != NChannelBlocks())
      throw std::runtime_error("B200 solver: SolveData has another channel-block count");
    EnsureContext();
    std::vector<uint32_t> pairs;
    for (size_t cb = 0; cb != data.NChannelBlocks(); ++cb) {
      const typename SolveData<VisMatrix>::ChannelBlockData& block = data.ChannelBlock(cb);
      const size_t n = block.NVisibilities();
      pairs.resize(2 * n);
      for (size_t v = 0; v != n; ++v) {
        pairs[2 * v] = block.Antenna1Index(v);
        pairs[2 * v + 1] = block.Antenna2Index(v);
      }
      const float* vis = n ? reinterpret_cast<const float*>(&*block.DataBegin()) : nullptr;
      const float* model =
          n ? reinterpret_cast<const float*>(&block.ModelVisibility(0, 0)) : nullptr;
      Check(ddsolve_set_channel_block(ctx_, uint32_t(cb), n, vis, model, pairs.data(),
                                      block.SolutionMapData()));
      DP3B200_ADAPTER_TRACE("channel block uploaded");
    }
  }

  // The solver's constraints as device constraints, when every one has a
  // device form (DP3's AntennaConstraint, SmoothnessConstraintB200); these
  // are always satisfied (Constraint::Satisfied), so the device loop's
  // stopping rule is DP3's. Returns false (device constraints cleared) when
  // some constraint runs on the host only.
  bool UploadDeviceConstraints() {
    Check(ddsolve_clear_constraints(ctx_));
    for (const std::unique_ptr<Constraint>& c : GetConstraints()) {
      if (const auto* a = dynamic_cast<const AntennaConstraint*>(c.get())) {
        std::vector<uint32_t> offsets{0}, antennas;
        for (const std::set<size_t>& set : a->GetAntennaSets()) {
          for (size_t ant : set) antennas.push_back(uint32_t(ant));
          offsets.push_back(uint32_t(antennas.size()));
        }
        Check(ddsolve_add_antenna_constraint(ctx_, uint32_t(offsets.size() - 1),
                                             offsets.data(), antennas.data()));
      } else if (const auto* s = dynamic_cast<const SmoothnessConstraintB200*>(c.get())) {
        Check(s->AddTo(ctx_));
      } else {
        Check(ddsolve_clear_constraints(ctx_));
        return false;
      }
    }
    return true;
  }

  ddsolve_settings DeviceSettings(uint32_t max_iterations) const {
    ddsolve_settings s;
    ddsolve_default_settings(&s);
    s.max_iterations = max_iterations;
    s.min_iterations = uint32_t(GetMinIterations());
    s.accuracy = GetAccuracy();
    s.constraint_accuracy = GetConstraintAccuracy();
    s.step_size = GetStepSize();
    s.detect_stalling = 0;  // evaluated on the host with DP3's own DetectStall
    s.phase_only = GetPhaseOnly() ? 1 : 0;
    return s;
  }

  std::vector<double> Flatten(const std::vector<std::vector<DComplex>>& solutions) const {
    const size_t per_cb = NAntennas() * NSubSolutions() * NPol;
    std::vector<double> flat(2 * per_cb * solutions.size());
    for (size_t cb = 0; cb != solutions.size(); ++cb) {
      if (solutions[cb].size() != per_cb)
        throw std::runtime_error("B200 solver: solutions have the wrong size");
      std::memcpy(flat.data() + 2 * cb * per_cb, solutions[cb].data(), per_cb * sizeof(DComplex));
    }
    return flat;
  }

  void Unflatten(const std::vector<double>& flat,
                 std::vector<std::vector<DComplex>>& solutions) const {
    const size_t per_cb = NAntennas() * NSubSolutions() * NPol;
    for (size_t cb = 0; cb != solutions.size(); ++cb)
      std::memcpy(solutions[cb].data(), flat.data() + 2 * cb * per_cb, per_cb * sizeof(DComplex));
  }

  SolveResult SolveOnDevice(std::vector<std::vector<DComplex>>& solutions,
                            std::ostream* stat_stream) {
    const std::vector<double> start = Flatten(solutions);
    const uint32_t max_it = uint32_t(GetMaxIterations());
    std::vector<double> flat = start;
    std::vector<double> mags(std::max<size_t>({GetMaxIterations(), GetMinIterations(), 1}));
    ddsolve_settings s = DeviceSettings(max_it);
    Check(ddsolve_set_settings(ctx_, &s));
    ddsolve_result r;
    DP3B200_ADAPTER_TRACE("device solve");
    Check(ddsolve_solve(ctx_, flat.data(), &r, mags.data()));
    DP3B200_ADAPTER_TRACE("device solve done");
    size_t iteration = std::min<size_t>(r.has_converged ? r.iterations : r.iterations - 1,
                                        mags.size());
    bool has_converged = r.has_converged != 0;
    if (GetDetectStalling()) {
      // DP3's stopping rule over the device's step magnitudes: the first
      // iteration at which it stops (ReachedStoppingCriterion also runs
      // DetectStall, with DP3's own sigma).
      std::vector<double> prefix;
      prefix.reserve(iteration);
      for (size_t it = 1; it <= iteration; ++it) {
        prefix.push_back(mags[it - 1]);
        const bool converged_here = mags[it - 1] <= GetAccuracy();
        if (ReachedStoppingCriterion(it, converged_here, true, prefix)) {
          if (it < iteration) {  // stalled before the device loop stopped
            flat = start;
            s = DeviceSettings(uint32_t(it));
            Check(ddsolve_set_settings(ctx_, &s));
            Check(ddsolve_solve(ctx_, flat.data(), &r, mags.data()));
            iteration = it;
            has_converged = r.has_converged != 0;
          }
          break;
        }
      }
    }
    Unflatten(flat, solutions);
    if (stat_stream)
      for (size_t i = 0; i < iteration; ++i) *stat_stream << i + 1 << ' ' << mags[i] << '\n';
    return MakeResult(iteration, has_converged, true);
  }

  SolveResult SolveWithHostConstraints(std::vector<std::vector<DComplex>>& solutions,
                                       double time, std::ostream* stat_stream) {
    PrepareConstraints();
    SolutionTensor next_solutions(
        {NChannelBlocks(), NAntennas(), NSubSolutions(), NSolutionPolarizations()});
    size_t iteration = 0;
    bool has_converged = false;
    bool has_previously_converged = false;
    bool constraints_satisfied = false;
    std::vector<double> step_magnitudes;
    step_magnitudes.reserve(GetMaxIterations());
    do {
      if constexpr (NPol == 4)
        MakeSolutionsFinite4Pol(solutions);
      else if constexpr (NPol == 2)
        MakeSolutionsFinite2Pol(solutions);
      else
        MakeSolutionsFinite1Pol(solutions);
      const std::vector<double> flat = Flatten(solutions);
      Check(ddsolve_perform_iteration(ctx_, flat.data(),
                                      reinterpret_cast<double*>(next_solutions.data())));
      Step(solutions, next_solutions);
      constraints_satisfied =
          ApplyConstraints(iteration, time, has_previously_converged, next_solutions);
      double avg_squared_diff;
      has_converged = AssignSolutions(solutions, next_solutions, !constraints_satisfied,
                                      avg_squared_diff, step_magnitudes);
      ++iteration;
      has_previously_converged = has_converged || has_previously_converged;
    } while (!ReachedStoppingCriterion(iteration, has_converged, constraints_satisfied,
                                       step_magnitudes));
    if (stat_stream)
      for (size_t i = 0; i < step_magnitudes.size(); ++i)
        *stat_stream << i + 1 << ' ' << step_magnitudes[i] << '\n';
    return MakeResult(iteration, has_converged, constraints_satisfied);
  }

  int device_;
  ddsolve_ctx* ctx_ = nullptr;
  std::vector<uint32_t> n_solutions_per_direction_;
};

template <typename VisMatrix>
using IterativeDiagonalSolverB200 = IterativeSolverB200<VisMatrix, 2>;
template <typename VisMatrix>
using IterativeScalarSolverB200 = IterativeSolverB200<VisMatrix, 1>;
// Drop-in for IterativeFullJonesSolver (IterativeFullJonesSolver.h:15-47).
using IterativeFullJonesSolverB200 = IterativeSolverB200<aocommon::MC2x2F, 4>;

}  // namespace dp3::ddecal

#endif
