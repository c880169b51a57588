/*
 * ddwarm_b200 — learned warm start for the direction-iterative gain solver.
 *
 * A three-layer perceptron (n_in -> n_hidden -> n_hidden -> n_out, ReLU)
 * whose forward and training passes run on the B200's 5th-generation tensor
 * cores (tcgen05.mma, BF16 operands, FP32 accumulation in tensor memory). In
 * the solver it maps, per (antenna, direction), the last solutions and the
 * current interval's one-pass residual statistics to the initial gains of the
 * new interval; the solver then iterates to the same tolerance as without it,
 * so only the iteration count changes.
 *
 * The reference (DP3 DDECal) has no learned component: none of these entry
 * points replaces a reference interface. Its nearest counterpart is the
 * solution propagation of DDECal (steps/DDECal.cc, `propagatesolutions`),
 * which starts an interval from the previous interval's solutions; this
 * network is an alternative source of those initial solutions, passed to
 * ddsolve_solve (include/ddsolve_b200.h) exactly as propagated ones are.
 *
 * Parameters are FP32 masters (Adam state in FP32) with BF16 copies used by
 * the tensor cores. Packed parameter order (FP32, logical shapes, row-major):
 *   W1 [n_hidden][n_in], b1 [n_hidden], W2 [n_hidden][n_hidden],
 *   b2 [n_hidden], W3 [n_out][n_hidden], b3 [n_out].
 * Loss: mean over rows and outputs of (y - target)^2.
 *
 * Status codes as in ddsolve_b200.h (0 ok, 1 invalid, 2 CUDA, 4 unsupported,
 * 5 a bounded device wait ran out).
 */
#ifndef DDWARM_B200_H
#define DDWARM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef DDSOLVE_API
#define DDSOLVE_API __attribute__((visibility("default")))
#endif

typedef struct ddwarm_ctx ddwarm_ctx;

/* n_in in [1, 1024], n_out in [1, 256]; n_hidden a multiple of 64 in [64, 256].
 * Weights: He-uniform from std::mt19937_64(seed), biases zero. */
DDSOLVE_API int ddwarm_create(uint32_t n_in, uint32_t n_hidden, uint32_t n_out,
                              uint64_t seed, int device, ddwarm_ctx** out);
DDSOLVE_API void ddwarm_destroy(ddwarm_ctx* ctx);
DDSOLVE_API const char* ddwarm_last_error(const ddwarm_ctx* ctx);

/* Number of packed FP32 parameters. */
DDSOLVE_API uint64_t ddwarm_param_count(const ddwarm_ctx* ctx);
DDSOLVE_API int ddwarm_get_params(ddwarm_ctx* ctx, float* params);
DDSOLVE_API int ddwarm_set_params(ddwarm_ctx* ctx, const float* params);

/* Forward pass: x [n][n_in] -> y [n][n_out], host FP32 buffers. */
DDSOLVE_API int ddwarm_predict(ddwarm_ctx* ctx, uint32_t n, const float* x, float* y);

/* Loss and its gradient for one batch (no update): grads packed as the
 * parameters. For checking the training kernels. */
DDSOLVE_API int ddwarm_gradients(ddwarm_ctx* ctx, uint32_t n, const float* x,
                                 const float* target, float* grads, float* loss);

/* Intermediate values of one pass, so that each tensor-core product can be
 * checked on its own against an oracle fed the GPU's own inputs of that
 * layer. Every pointer may be NULL (not returned). Host FP32 arrays, BF16
 * quantities as their exact FP32 values:
 *   xb [n][n_in]       the input rounded to BF16 (the first product's A)
 *   h1, h2 [n][n_hidden]  BF16 hidden activations relu(z + b)
 *   y [n][n_out]       FP32 output
 * With a target [n][n_out] (else these stay untouched):
 *   dy [n][n_out]      BF16 dL/dY = 2 (y - t) / (n n_out)
 *   dz2, dz1 [n][n_hidden]  BF16 dL/dZ after the ReLU masks
 *   grads              packed as the parameters (as ddwarm_gradients)
 *   loss               mean (y - t)^2 (one float)
 * No counterpart in the reference (DP3 has no learned component). */
typedef struct {
  float* xb;
  float* h1;
  float* h2;
  float* y;
  float* dy;
  float* dz2;
  float* dz1;
  float* grads;
  float* loss;
} ddwarm_trace_out;
DDSOLVE_API int ddwarm_trace(ddwarm_ctx* ctx, uint32_t n, const float* x, const float* target,
                             const ddwarm_trace_out* out);

/* Trains on the data set x [n][n_in], target [n][n_out] (host FP32, uploaded
 * once): `epochs` passes of shuffled mini-batches of `batch` rows (the order
 * from std::mt19937_64(seed)), Adam (beta 0.9 / 0.999, eps 1e-8) at learning
 * rate `lr`. epoch_loss[e] (optional, `epochs` entries) receives the mean
 * batch loss of epoch e. */
DDSOLVE_API int ddwarm_train(ddwarm_ctx* ctx, uint32_t n, const float* x,
                             const float* target, uint32_t epochs, uint32_t batch,
                             float lr, uint64_t seed, float* epoch_loss);

/* Solver-side layout of the warm start: solutions are [n_channel_blocks]
 * [n_antennas][n_sub][n_pol] complex128, as in ddsolve_solve. */
typedef struct {
  uint32_t n_channel_blocks;
  uint32_t n_antennas;
  uint32_t n_sub;  /* sum of the solutions per direction */
  uint32_t n_pol;
  double scale;    /* feature / output scale */
} ddwarm_layout;

/* Network samples from solution sets (each in the layout above): sets[0] is
 * the base, sets[1..n_sets-1] the others. One row per (antenna,
 * sub-solution), row = antenna * n_sub + sub; with W = n_channel_blocks *
 * n_pol values per row and set (index channel_block * n_pol + pol), set k >= 1
 * fills columns [(k - 1) 2W, (k - 1) 2W + W) with scale * Re log(set_k /
 * base) and the next W with scale * Im log(set_k / base); non-finite values
 * give 0. x: [n_antennas * n_sub][2 W (n_sets - 1)] float32 (host). Computed
 * on the GPU (used for training data and targets). 2 <= n_sets <= 16. */
DDSOLVE_API int ddwarm_features(ddwarm_ctx* ctx, const ddwarm_layout* layout, uint32_t n_sets,
                                const double* const* sets, float* x);

/* Initial solutions for the solver: start = base * exp((y_re + i y_im) /
 * scale), y = the network's output for ddwarm_features(sets) (the network
 * must have n_in = 2 W (n_sets - 1) and n_out = 2 W); entries whose result is
 * not finite take the base value. Features, forward pass and the update run
 * on the GPU. `sets` and `start` may be host arrays or, with unified
 * addressing, device memory of the context's device (for example the outputs
 * of ddsolve_perform_iterations kept on the device), which is read in place.
 * With `start` in device memory the call only enqueues the work on the
 * context's stream and returns; a bounded-wait failure then surfaces at the
 * context's next call that waits (a host `start`, ddwarm_features, ...). */
DDSOLVE_API int ddwarm_predict_start(ddwarm_ctx* ctx, const ddwarm_layout* layout,
                                     uint32_t n_sets, const double* const* sets, double* start);

/* Runs the context's work on `stream` (a cudaStream_t of the same device,
 * e.g. ddsolve_stream() of the solver, so that the warm start and the solve
 * are ordered without host waits); NULL restores the context's own stream.
 * Waits for the work already enqueued. */
DDSOLVE_API int ddwarm_set_stream(ddwarm_ctx* ctx, void* stream);

#ifdef __cplusplus
}
#endif

#endif
