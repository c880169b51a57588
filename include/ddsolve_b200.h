/*
 * ddsolve_b200 -- C ABI of the B200 direction-iterative gain solver.
 *
 * This is the drop-in boundary for DP3's DDECal direction-iterative solvers.
 * A DP3-side adapter class derived from dp3::ddecal::SolverBase
 * (dp3_b200/dp3/IterativeSolverB200.h) binds these entry points; every entry
 * point below names the reference interface it replaces.
 *
 * Conventions
 *  - Plain pointers and sizes only. No exception crosses the ABI: every
 *    function returns 0 on success or a nonzero DDSOLVE_E_* code, and
 *    ddsolve_last_error() gives the message (thread-local for failures that
 *    have no context yet).
 *  - Visibility layout per channel block is the reference SolveData layout
 *    (ddecal/gain_solvers/SolveData.h:28-194):
 *      data          float32 [n_vis][n_correlations][re,im]
 *      model         float32 [n_directions][n_vis][n_correlations][re,im]
 *      antenna_pairs uint32  [n_vis][2]
 *      solution_map  uint32  [n_directions][n_vis]  (absolute sub-solution)
 *    n_correlations: 1 = complex<float> (UniSolveData), 2 = XX/YY
 *    (aocommon::MC2x2FDiag, DuoSolveData), 4 = full 2x2 row-major
 *    (aocommon::MC2x2F, FullSolveData).
 *  - Solutions: float64 complex [n_channel_blocks][n_antennas][n_sub][n_pol]
 *    ([re,im] interleaved), i.e. the concatenation of the reference's
 *    std::vector<std::vector<std::complex<double>>> solutions
 *    (ddecal/gain_solvers/SolverBase.h:205-227).
 *  - One context = one CUDA stream on one device. Contexts are not re-entrant;
 *    distinct contexts may be used from distinct threads.
 *  - The library never falls back to the CPU: without a usable sm_100 device
 *    ddsolve_create() fails with DDSOLVE_E_CUDA.
 */
#ifndef DDSOLVE_B200_H
#define DDSOLVE_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DDSOLVE_API __attribute__((visibility("default")))
#else
#define DDSOLVE_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define DDSOLVE_OK 0
#define DDSOLVE_E_INVALID 1     /* bad argument / dimension */
#define DDSOLVE_E_CUDA 2        /* CUDA runtime error */
#define DDSOLVE_E_STATE 3       /* call out of order (e.g. solve before data) */
#define DDSOLVE_E_UNSUPPORTED 4 /* valid but not supported combination */
#define DDSOLVE_E_TIMEOUT 5     /* a device-side bounded wait gave up */

typedef struct ddsolve_ctx ddsolve_ctx;

/* Dimensions; replaces SolverBase::Initialize(n_antennas,
 * n_solutions_per_direction, n_channel_blocks)
 * (ddecal/gain_solvers/SolverBase.h:76-78, SolverBase.cc:41-61) plus the
 * solver choice made by SolverFactory::CreateDiagonalSolver /
 * CreateScalarSolver (ddecal/SolverFactory.cc:49-146). */
typedef struct {
  uint32_t n_antennas;
  uint32_t n_directions;
  uint32_t n_channel_blocks;
  uint32_t n_correlations;           /* 1, 2 or 4, see above */
  uint32_t n_solution_polarizations; /* 2 = IterativeDiagonalSolver,
                                        1 = IterativeScalarSolver,
                                        4 = IterativeFullJonesSolver
                                        (IterativeFullJonesSolver.cc:17-228;
                                        4 correlations, single
                                        intervals, no device
                                        constraints; solutions
                                        [.., 4] = J_00 J_01 J_10 J_11) */
  const uint32_t* n_solutions_per_direction; /* [n_directions], >= 1 */
} ddsolve_dims;

/* Solver settings; replaces the SolverBase setters SetMaxIterations,
 * SetMinIterations, SetAccuracy, SetConstraintAccuracy, SetStepSize,
 * SetDetectStalling and SetPhaseOnly (ddecal/gain_solvers/SolverBase.h:89-177)
 * with the defaults of SolverBase::SolverBase (SolverBase.cc:27-39). */
typedef struct {
  uint32_t max_iterations;
  uint32_t min_iterations;
  double accuracy;
  double constraint_accuracy;
  double step_size;
  int32_t detect_stalling;
  double step_diff_sigma;
  int32_t phase_only;
} ddsolve_settings;

/* Replaces SolverBase::SolveResult (ddecal/gain_solvers/SolverBase.h:61-65):
 * iterations follows SolverBase::MakeResult (SolverBase.cc:192-213). */
typedef struct {
  uint32_t iterations;
  uint32_t constraint_iterations;
  int32_t has_converged;
  int32_t has_stalled;
} ddsolve_result;

/* Creates a solver on CUDA device `device` (ordinal). Replaces constructing
 * IterativeDiagonalSolver<V> / IterativeScalarSolver<V> and calling
 * SolverBase::Initialize (ddecal/gain_solvers/SolverBase.cc:41-61): the same
 * dimension checks apply. */
DDSOLVE_API int ddsolve_create(const ddsolve_dims* dims, int device, ddsolve_ctx** out);

/* Frees all device memory of the context. NULL is accepted. */
DDSOLVE_API int ddsolve_destroy(ddsolve_ctx* ctx);

/* Message of the last failure on this context (or of the last failed create
 * on this thread when ctx == NULL). Never NULL. */
DDSOLVE_API const char* ddsolve_last_error(const ddsolve_ctx* ctx);

/* Default settings of SolverBase::SolverBase (SolverBase.cc:27-39). */
DDSOLVE_API void ddsolve_default_settings(ddsolve_settings* settings);

/* Replaces the SolverBase setters (SolverBase.h:89-177). */
DDSOLVE_API int ddsolve_set_settings(ddsolve_ctx* ctx, const ddsolve_settings* settings);

/* Uploads one channel block of a SolveData, in the reference layout above
 * (replaces reading SolveData<V>::ChannelBlockData, SolveData.h:31-133, inside
 * IterativeDiagonalSolver::Solve). Any visibility order and antenna/solution
 * assignment is accepted (regular and BDA data); consecutive visibilities
 * that share antennas and solution indices are solved together. data and
 * model may be host memory (pinned memory makes the copy asynchronous) or
 * device memory of the context's device; antenna_pairs and solution_map are
 * host memory. Replaces any previous data of that channel block. */
DDSOLVE_API int ddsolve_set_channel_block(ddsolve_ctx* ctx, uint32_t channel_block,
                              uint64_t n_vis, const float* data,
                              const float* model,
                              const uint32_t* antenna_pairs,
                              const uint32_t* solution_map);

/* Same as ddsolve_set_channel_block for data packed by the regular SolveData
 * constructor (ddecal/gain_solvers/SolveData.cc:77-188): visibility index
 * ((t * n_baselines) + b) * n_channels + c, baseline b between antenna1[b] and
 * antenna2[b] (autocorrelations already removed), solution index of direction
 * d at time t = t * min(n_sol[d], n_times) / n_times + first solution of d.
 * No per-visibility antenna / solution arrays are read. data and model as in
 * ddsolve_set_channel_block (host or device memory); antenna1 / antenna2 are
 * host memory. */
DDSOLVE_API int ddsolve_set_channel_block_regular(ddsolve_ctx* ctx, uint32_t channel_block,
                                      uint32_t n_times, uint32_t n_baselines,
                                      uint32_t n_channels, const float* data,
                                      const float* model,
                                      const uint32_t* antenna1,
                                      const uint32_t* antenna2);

/* Point sources of one direction: DP3's PointSource (base/PointSource.h)
 * with a flat spectrum (Stokes I, Q, U, V independent of frequency). */
typedef struct {
  uint32_t n_sources;
  const double* lmn;    /* [n_sources][3]: l, m, n of each source relative to
                           the phase centre (as DP3's radec2lmn gives them) */
  const double* stokes; /* [n_sources][4]: I, Q, U, V in Jy */
} ddsolve_sky_direction;

/* ddsolve_set_channel_block_regular with the model visibilities predicted
 * on the GPU instead of uploaded: replaces DDECal's per-direction predict of
 * point sources (steps/OnePredict.cc -> base/Simulator.cc:112-245
 * visit(PointSource), station phases :477-520, spectrum :522-547) together
 * with the model's SolveData packing. Per source, phi_p = 2 pi / c (u_p l +
 * v_p m + w_p (n - 1)) and V_pq(nu) = sum S exp(i (phi_q - phi_p) nu) with
 * S = I + Q, U + iV, U - iV, I - Q for XX, XY, YX, YY (XX and YY for 2
 * correlations, I for 1), in FP64, stored complex64; no time or frequency
 * smearing and no beam. Only `data` crosses PCIe (host or device memory);
 * frequencies [n_channels] (Hz) are this block's channels, station_uvw
 * [n_times][n_antennas][3] (m) the station UVW per time step, sky one entry
 * per direction. Limit: at most 3200 sources in one direction
 * (DDSOLVE_E_UNSUPPORTED beyond). */
DDSOLVE_API int ddsolve_set_channel_block_regular_sky(
    ddsolve_ctx* ctx, uint32_t channel_block, uint32_t n_times, uint32_t n_baselines,
    uint32_t n_channels, const float* data, const double* frequencies,
    const double* station_uvw, const uint32_t* antenna1, const uint32_t* antenna2,
    const ddsolve_sky_direction* sky);

/* The same prediction alone: model [n_directions][n_times * n_baselines *
 * n_channels][n_correlations][2] float32, in host memory or device memory of
 * the context's device; returns after the model is written.
 * Autocorrelation baselines (antenna1 == antenna2) get a zero model, as the
 * reference's Simulator skips them (Simulator.cc:162-163). */
DDSOLVE_API int ddsolve_predict_regular(ddsolve_ctx* ctx, uint32_t n_times,
                                        uint32_t n_baselines, uint32_t n_channels,
                                        const double* frequencies, const double* station_uvw,
                                        const uint32_t* antenna1, const uint32_t* antenna2,
                                        const ddsolve_sky_direction* sky, float* model);

/* One solution interval in DP3's buffer layout (the DPBuffers DDECal holds
 * per interval: [time][baseline][channel][XX XY YX YY], autocorrelations
 * included). */
typedef struct {
  uint32_t n_times;
  uint32_t n_baselines; /* all baselines of the buffers */
  uint32_t n_channels;  /* all channels; channel block cb of the context gets
                           channels [cb n_ch / n_cb, (cb + 1) n_ch / n_cb) */
  const uint32_t* antenna1; /* [n_baselines] */
  const uint32_t* antenna2;
  const float* data;    /* [n_times][n_baselines][n_channels][4][2] unweighted */
  const float* weights; /* [n_times][n_baselines][n_channels][4] */
  const uint8_t* flags; /* [n_times][n_baselines][n_channels][4], nonzero =
                           flagged; NULL = nothing flagged */
  const float* model;   /* [n_directions][n_times][n_baselines][n_channels][4][2]
                           unweighted model, or NULL: predicted from `sky` */
  const double* frequencies;        /* [n_channels] Hz (with sky) */
  const double* station_uvw;        /* [n_times][n_antennas][3] m (with sky) */
  const ddsolve_sky_direction* sky; /* [n_directions] (with sky) */
  int32_t linear_weighting; /* 1: weight by w, 0: by sqrt(w) */
} ddsolve_interval_buffers;

/* Uploads one solution interval from DP3's raw buffers and does on the GPU
 * what DDECal does on the host before a solve: AssignAndWeight
 * (ddecal/gain_solvers/SolverTools.cc:81-167: a visibility is flagged when
 * any correlation of the data or of any direction's model is flagged or
 * non-finite; data and models are weighted by sqrt(w) per correlation, or
 * by w in linear_weighting mode; flagged visibilities become zero) and the
 * regular SolveData constructor (SolveData.cc:77-188: even channel-block
 * split, autocorrelations dropped, XX / YY or (XX + YY) / 2 per the
 * context's correlations, direction-dependent solution indices), for every
 * channel block of the context. With model == NULL the unweighted model is
 * predicted on the GPU first (as ddsolve_set_channel_block_regular_sky).
 * data, weights, flags and model may be host memory or device memory of the
 * context's device; the call returns when the interval is in place. */
DDSOLVE_API int ddsolve_set_interval_buffers(ddsolve_ctx* ctx,
                                             const ddsolve_interval_buffers* buffers);

/* One interval as DDECal holds it for the step after the solve: data
 * [n_times][n_baselines][n_channels][XX XY YX YY] and one model buffer per
 * direction (DPBuffer::GetData(direction name) per time step; one call per
 * time step passes n_times = 1 and that step's buffers). */
typedef struct {
  uint32_t n_times;
  uint32_t n_baselines;     /* all baselines, autocorrelations included */
  uint32_t n_channels;      /* channel block cb of the context gets channels
                               [cb n_ch / n_cb, (cb + 1) n_ch / n_cb) */
  const uint32_t* antenna1; /* [n_baselines], host memory */
  const uint32_t* antenna2;
  const float* data;            /* [n_times][n_baselines][n_channels][4][2] */
  const float* const* models;   /* [n_directions] host array of pointers, each
                                   [n_times][n_baselines][n_channels][4][2]; or
                                   NULL: predicted from `sky` */
  const double* frequencies;        /* [n_channels] Hz (with sky) */
  const double* station_uvw;        /* [n_times][n_antennas][3] m (with sky) */
  const ddsolve_sky_direction* sky; /* [n_directions] (with sky) */
} ddsolve_subtract_buffers;

/* The step after the solve: applies the solutions to every direction's model
 * and subtracts the corrected models from the data. Replaces
 * DDECal::CorrectAndSubtractModels (steps/DDECal.cc:1081-1125) with
 * ApplySolutionAndSubtract and its ApplyFullJones/Diagonal/ScalarSolution
 * helpers (:1004-1079). Per visibility (autocorrelations included) and
 * direction the corrected model is G_1 M G_2^H in FP64, as the reference's
 * complex<double> arithmetic (products and sums rounded separately); the sum
 * over directions is subtracted as float(double(data) - sum). With models ==
 * NULL the unweighted model of every baseline (autocorrelations zero) is
 * predicted from sky / frequencies / station_uvw first, as
 * ddsolve_predict_regular. The reference leaves weights and flags alone, and
 * so does this call.
 *   solutions:  complex float64 [n_channel_blocks][n_antennas][n_directions]
 *               [n_pol] (DDECal's solutions_ of the interval); the context
 *               must have one solution per direction (otherwise
 *               DDSOLVE_E_UNSUPPORTED, as the reference throws).
 *   data_out:   [n_times][n_baselines][n_channels][4][2]: data - the sum over
 *               directions of the corrected models ("subtract"); may equal
 *               buffers->data; NULL = no subtraction.
 *   models_out: [n_directions] host array of pointers, each like a model
 *               buffer: the corrected models ("keepmodel"); each may equal
 *               its buffers->models[d]; NULL = not kept.
 * Data, models, solutions and outputs may be host or device memory of the
 * context's device. The call returns when the outputs are written. It does
 * not use the context's uploaded visibilities or solutions. */
DDSOLVE_API int ddsolve_correct_and_subtract(ddsolve_ctx* ctx,
                                             const ddsolve_subtract_buffers* buffers,
                                             const double* solutions, float* data_out,
                                             float* const* models_out);

/* Full iterate-until-converged solve on the device with no host constraints:
 * replaces IterativeDiagonalSolver<V>::Solve
 * (ddecal/gain_solvers/IterativeDiagonalSolver.cc:38-97) and
 * IterativeScalarSolver<V>::Solve (IterativeScalarSolver.cc:30-89) for a
 * solver without constraints. `solutions` holds the initial values on entry
 * and the result on return, like the reference's in/out argument; it may be a
 * host array or, with unified addressing, device memory of the context's
 * device (as may the solution arrays of ddsolve_perform_iteration[s]).
 * step_magnitudes (optional, host, [max_iterations]) receives the step
 * magnitude of every iteration (the statistics stream of the reference's
 * stat_stream overload). */
DDSOLVE_API int ddsolve_solve(ddsolve_ctx* ctx, double* solutions, ddsolve_result* result,
                  double* step_magnitudes);

/* Several independent solution intervals in one context (no counterpart in
 * the reference, which solves one interval per Solve call): channel blocks
 * [first_channel_block[g], first_channel_block[g + 1]) form interval g, for
 * g < n_intervals (first_channel_block[0] = 0, first_channel_block[n] =
 * n_channel_blocks; NULL with n_intervals = 1 restores one interval). Every
 * interval has its own iteration count, convergence, stall detection and
 * stopping, exactly as if solved alone; one streaming pass per iteration
 * covers all intervals still iterating (the data of intervals that have
 * stopped is skipped on the pipelined path), and an interval that has stopped
 * keeps its solutions. */
DDSOLVE_API int ddsolve_set_intervals(ddsolve_ctx* ctx, uint32_t n_intervals,
                                      const uint32_t* first_channel_block);

/* ddsolve_solve for every interval of the context: results[g] per interval,
 * step_magnitudes (optional) [n_intervals][max(max_iterations,
 * min_iterations, 1)]. ddsolve_solve refuses a context with several
 * intervals. */
DDSOLVE_API int ddsolve_solve_batch(ddsolve_ctx* ctx, double* solutions, ddsolve_result* results,
                                    double* step_magnitudes);

/* Device-side constraints. SolverBase::ApplyConstraints (SolverBase.cc:
 * 174-190) runs a solver's constraints on the host between SolverBase::Step
 * and AssignSolutions (IterativeDiagonalSolver.cc:77-83); the constraints
 * added here run on the device at that point of every iteration of
 * ddsolve_solve, in the order they were added, so that a constrained solve
 * stays in the device loop (one CUDA graph) instead of returning to the host
 * once per iteration. All three are satisfied from the start
 * (Constraint::Satisfied), so the stopping rule is the unconstrained one.
 * The arithmetic is the reference's, in FP64, in its order of operations.
 * Single-interval contexts only (DDSOLVE_E_UNSUPPORTED from
 * ddsolve_solve_batch). Adding or clearing a constraint rebuilds the
 * context's graph at the next solve. */
#define DDSOLVE_CONSTRAINT_SMOOTHNESS 1
#define DDSOLVE_CONSTRAINT_ANTENNA 2
#define DDSOLVE_CONSTRAINT_REFERENCE_ANTENNA 3

/* SmoothnessConstraint (ddecal/constraints/SmoothnessConstraint.cc:11-97)
 * with its Gaussian KernelSmoother (KernelSmoother.h:69-160): every
 * (antenna, sub-solution, polarization) series over channel blocks is
 * replaced by its kernel-weighted mean; non-finite values get weight 0, and
 * a mean over zero weight is NaN. */
typedef struct {
  const double* frequencies;          /* [n_channel_blocks] Hz, ascending
                                         (Constraint::Initialize) */
  double bandwidth_hz;                /* constructor arguments */
  double bandwidth_ref_frequency_hz;
  double spectral_exponent;
  int32_t kernel_truncation;
  const double* weights;              /* [n_antennas * n_channel_blocks]
                                         (Constraint::SetWeights), or NULL
                                         when sub_solution_weights is given */
  const double* sub_solution_weights; /* NULL or [n_sub_solutions][n_antennas
                                         * n_channel_blocks] (SetSubSolutionWeights,
                                         used instead of weights) */
  const double* antenna_factors;      /* [n_antennas] (SetAntennaFactors) or
                                         NULL = all 1 */
  const double* dd_factors;           /* NULL or [n_sub_solutions]
                                         (SetDdSmoothingFactors) */
} ddsolve_smoothness;

DDSOLVE_API int ddsolve_add_smoothness_constraint(ddsolve_ctx* ctx,
                                                  const ddsolve_smoothness* s);

/* AntennaConstraint (ddecal/constraints/AntennaConstraint.h:29-82): set k
 * holds antennas[set_offsets[k] .. set_offsets[k + 1]) (a std::set: order
 * and repeats do not matter); per channel block, sub-solution and
 * polarization every member gets the mean of the set's finite solutions. */
DDSOLVE_API int ddsolve_add_antenna_constraint(ddsolve_ctx* ctx, uint32_t n_sets,
                                               const uint32_t* set_offsets,
                                               const uint32_t* antennas);

/* Constraint::ApplyReferenceAntenna (ddecal/constraints/Constraint.cc:7-37),
 * the phase referencing of DP3's TEC constraints: per polarization, every
 * antenna's solutions divided by those of the first antenna whose
 * sub-solution-0 solutions are finite in more than 20% of the channel
 * blocks, which become 1. */
DDSOLVE_API int ddsolve_add_reference_antenna_constraint(ddsolve_ctx* ctx);

/* Removes every device constraint. */
DDSOLVE_API int ddsolve_clear_constraints(ddsolve_ctx* ctx);

/* One direction-iterative pass over every channel block:
 * next_solutions = sum(num) / sum(den) per antenna, sub-solution and
 * polarization, NaN where the denominator is zero -- exactly the
 * next_solutions tensor that IterativeDiagonalSolver::PerformIteration
 * (IterativeDiagonalSolver.cc:100-222) / IterativeScalarSolver
 * (IterativeScalarSolver.cc:91-195) fill before SolverBase::Step. Use it to
 * run the iteration loop on the host when host constraints
 * (SolverBase::ApplyConstraints, SolverBase.cc:166-190) are present. Host
 * pointers, layout as `solutions`. */
DDSOLVE_API int ddsolve_perform_iteration(ddsolve_ctx* ctx, const double* solutions,
                              double* next_solutions);

/* n_passes consecutive PerformIteration passes (IterativeDiagonalSolver.cc:
 * 100-127), each pass starting from the previous pass's next_solutions, with
 * no host round trip in between: outputs[k] ([n_passes][same layout as
 * `solutions`]) = PerformIteration(outputs[k - 1]), outputs[-1] = start. Each
 * pass costs one streaming pass over the data. Replaces a host loop of
 * ddsolve_perform_iteration calls; the learned warm start
 * (include/ddwarm_b200.h) uses these undamped passes as residual statistics
 * of the current interval. With `outputs` in device memory the call only
 * enqueues the passes on the context's stream (ddsolve_stream) and returns; a
 * bounded-wait failure then surfaces at the next call that waits. Device
 * arrays on the context's GPU are used in place (the first pass reads `start`,
 * every pass writes its slice of `outputs`, no staging copies) unless the two
 * overlap; they must stay allocated and unmodified until the passes have run
 * in stream order. Non-finite input solutions are used as given (no
 * MakeSolutionsFinite, as in PerformIteration). */
DDSOLVE_API int ddsolve_perform_iterations(ddsolve_ctx* ctx, const double* start,
                                           uint32_t n_passes, double* outputs);

/* The CUDA stream of the context (a cudaStream_t), so that callers can order
 * their own work or CUDA events against the solver. */
DDSOLVE_API void* ddsolve_stream(ddsolve_ctx* ctx);

/* Tuning of the streaming kernel: directions per thread group (0 = auto) and
 * the maximum number of time steps folded into one slab (0 = all). Replaces
 * nothing in the reference (its thread count is SolverBase::NSubThreads). */
DDSOLVE_API int ddsolve_set_tuning(ddsolve_ctx* ctx, uint32_t direction_groups,
                       uint32_t max_slab_times);

/* Plan variants of the streaming pass (no reference counterpart: DP3's only
 * knob is its thread count, SolverBase::NSubThreads). Negative / zero fields
 * mean "automatic". */
typedef struct {
  int32_t use_pipe;          /* -1 auto, 0 stream_kernel + finalize_kernel, 1 pipe_kernel */
  uint32_t direction_groups; /* stream_kernel: lanes per run, 0 auto, power of 2 <= 32 */
  uint32_t stages;           /* pipe_kernel: bulk-copy ring stages, 0 = as many as fit, >= 2 */
  int32_t model_powers;      /* pipe_kernel: -1 auto, 0 summed in the row loop, 1 precomputed */
  uint32_t gain_buffers;     /* pipe_kernel: gain-table buffers, 0 auto, 1 or 2 */
} ddsolve_tuning;

DDSOLVE_API int ddsolve_get_tuning(const ddsolve_ctx* ctx, ddsolve_tuning* tuning);
DDSOLVE_API int ddsolve_set_plan_tuning(ddsolve_ctx* ctx, const ddsolve_tuning* tuning);

/* Autotuner: on the uploaded data, times every applicable plan variant
 * (pipe_kernel with model powers on / off, one or two gain-table buffers,
 * all or three ring stages; stream_kernel with 1..32 lanes per run) over
 * `launches` iterations in next-solutions mode, keeps the fastest (time per
 * iteration, the once-per-solve model powers spread over max_iterations) and
 * caches the choice per process, keyed on stations, directions,
 * correlations, polarizations, the per-block visibilities, channels and slabs
 * and the solutions per direction: a later context of the same shape takes
 * the cached choice without timing. The solutions held by the context are
 * overwritten. */
DDSOLVE_API int ddsolve_autotune(ddsolve_ctx* ctx, uint32_t launches, ddsolve_tuning* chosen,
                                 float* iteration_ms);

/* Device time of the streaming kernel: launches it n_launches times on the
 * context stream with the current solutions and returns the mean duration in
 * milliseconds, measured with CUDA events. Solutions are not modified. With
 * four solution polarizations this times the full-Jones pass together with
 * its finalisation (two launches per pass). */
DDSOLVE_API int ddsolve_time_stream_kernel(ddsolve_ctx* ctx, uint32_t n_launches,
                               float* mean_ms);

/* Allocation-free direction-iterative pass (no counterpart in the reference:
 * DP3's solvers always own their buffers).
 *
 * Some callers cannot let a library allocate device memory: frameworks that
 * serve all device memory from their own pool or arena (an allocation behind
 * the pool's back escapes its accounting and can fail once the pool holds
 * the device), and processes whose device memory is budgeted in advance.
 * This entry point computes the same next_solutions as
 * ddsolve_perform_iteration without a context and without calling
 * cudaMalloc, cudaFree or any allocating library routine. Its per-antenna
 * accumulators live in one fixed 4 MiB array compiled into this library;
 * every GPU that loads the library holds that array until the process exits.
 * They are summed with FP32 global atomics, without compensation, so the
 * summation order (and the last bits of the result) can differ between
 * calls; the context entry points use fixed-order compensated merges.
 *
 * Inputs and outputs are DEVICE pointers the caller owns, for regular data
 * in the layout of ddsolve_set_channel_block_regular, with the channel blocks
 * concatenated: data = cb 0's [n_times*n_baselines*cb_channels[0]][n_corr][2]
 * floats, then cb 1's, ...; model = cb 0's [n_dir][n_vis_cb0][n_corr][2],
 * then cb 1's, ...; antenna1 / antenna2 [n_baselines]; solutions and
 * next_solutions [n_cb][n_ant][n_sub][n_pol] complex double. dims and
 * cb_channels are host pointers. Baselines with an antenna index
 * >= n_antennas are skipped, and so are autocorrelations (antenna1 ==
 * antenna2), which the reference's SolveData drops (SolveData.cc:100,137).
 *
 * Limits (DDSOLVE_E_UNSUPPORTED with a message beyond them): at most 256
 * channel blocks, 64 directions, 16 channels per block and 65535 time steps,
 * and n_cb * n_ant * n_sub * n_pol * 3 <= 1048576 accumulators.
 *
 * Work is queued on `stream` (a cudaStream_t; NULL = the legacy default
 * stream) and the call returns without waiting. The first call on a device
 * looks up the array's device address with that device current and caches
 * it for the rest of the process; cudaDeviceReset invalidates that cached
 * address, so do not call this entry point after resetting the device.
 * Every call reuses the same array and
 * clears the part it needs at its start, so calls that overlap on the GPU
 * (different streams or devices sharing a context) race: order them on one
 * stream or synchronise between them. */
DDSOLVE_API int ddsolve_perform_iteration_noalloc(
    const ddsolve_dims* dims, uint32_t n_times, uint32_t n_baselines,
    const uint32_t* cb_channels, const float* data, const float* model,
    const uint32_t* antenna1, const uint32_t* antenna2,
    const double* solutions, double* next_solutions, void* stream);

/* Number of kernel launches issued by the last ddsolve_solve call. */
DDSOLVE_API uint64_t ddsolve_last_launch_count(const ddsolve_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif
