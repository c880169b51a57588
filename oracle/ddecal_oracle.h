/*
 * CPU oracle for the DDECal direction-iterative gain solve.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker for the CUDA solver
 * in dp3_b200: only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * --impl reference legs of bench.py may load it. The product never links it.
 *
 * It is a plain C++ restatement of the reference algorithm:
 *   IterativeDiagonalSolver  ddecal/gain_solvers/IterativeDiagonalSolver.cc:38-222
 *   IterativeScalarSolver    ddecal/gain_solvers/IterativeScalarSolver.cc:30-229
 *   SolverBase bookkeeping   ddecal/gain_solvers/SolverBase.cc:63-371,
 *                            ddecal/gain_solvers/SolverBase.h:274-285
 *   add/subtract direction   ddecal/gain_solvers/SolveData.h:204-244
 *   SolverTester fixture     ddecal/test/unit/SolverTester.cc:95-202,331-363
 *   regular SolveData pack   ddecal/gain_solvers/SolveData.cc:77-188
 *
 * Memory layout of one channel block (identical to the reference SolveData):
 *   data          float32 [n_vis][n_correlations][re,im]
 *   model         float32 [n_directions][n_vis][n_correlations][re,im]
 *   antenna_pairs uint32  [n_vis][2]
 *   solution_map  uint32  [n_directions][n_vis]   (absolute sub-solution index)
 * Solutions: float64 [n_channel_blocks][n_antennas][n_sub_solutions][n_pol][re,im]
 */
#ifndef DDECAL_ORACLE_H
#define DDECAL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  uint32_t n_antennas;
  uint32_t n_directions;
  uint32_t n_channel_blocks;
  uint32_t n_correlations;           /* 1, 2 (XX/YY) or 4 (full 2x2) */
  uint32_t n_solution_polarizations; /* 1 = scalar solver, 2 = diagonal */
  const uint32_t* n_solutions_per_direction; /* [n_directions] */
} oracle_dims;

typedef struct {
  uint32_t max_iterations;
  uint32_t min_iterations;
  double accuracy;
  double constraint_accuracy;
  double step_size;
  int32_t detect_stalling;
  double step_diff_sigma;
  int32_t phase_only;
} oracle_settings;

typedef struct {
  uint64_t n_vis;
  const float* data;
  const float* model;
  const uint32_t* antenna_pairs;
  const uint32_t* solution_map;
} oracle_channel_block;

typedef struct {
  uint32_t iterations;
  uint32_t constraint_iterations;
  int32_t has_converged;
  int32_t has_stalled;
} oracle_result;

/* precision: 32 = reference arithmetic (FP32 per visibility, FP32 accumulators
 * for the diagonal solver, FP64 accumulators for the scalar solver, FP64
 * division), 64 = everything in FP64 (the "FP64 oracle").
 * n_threads: thread-pool size, split over channel blocks and then over
 * visibility chunks exactly like SolverBase::NSubThreads().
 * step_magnitudes: optional output [max_iterations]. */
int oracle_solve(const oracle_dims* dims, const oracle_settings* settings,
                 const oracle_channel_block* cbs, int precision, int n_threads,
                 double* solutions, double* step_magnitudes,
                 oracle_result* result);

/* One PerformIteration over every channel block: next_solutions = num/den
 * (no step, no constraints). */
int oracle_perform_iteration(const oracle_dims* dims,
                             const oracle_channel_block* cbs, int precision,
                             int n_threads, const double* solutions,
                             double* next_solutions);

/* SolverTester fixture restated (FillDdIntervalData + SolveData regular
 * constructor + Set{Scalar,Diagonal}Solutions).
 * Sizes: 50 antennas, 1225 baselines, 3 directions, 16 channels in 4 channel
 * blocks, 50 time steps. n_vis per channel block = 50*1225*4.
 * diagonal: 1 = SetDiagonalSolutions, 0 = SetScalarSolutions.
 * dd_intervals: 1 = {1,2,5} solutions per direction, 0 = {1,1,1}.
 * n_correlations: data written as 1, 2 or 4 correlations (Uni/Duo/Full).
 * Output buffers are caller-allocated per the layout above; input_solutions
 * gets [50][n_sub][2] complex float64 (the true gains). */
int oracle_solver_tester_fill(int diagonal, int dd_intervals,
                              uint32_t n_correlations, float** data,
                              float** model, uint32_t** antenna_pairs,
                              uint32_t** solution_map,
                              double* input_solutions);

#ifdef __cplusplus
}
#endif

#endif
