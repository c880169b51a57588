// B200 direction-iterative gain solver: kernels, host driver and C ABI.
//
// Algorithm: DP3 DDECal's IterativeDiagonalSolver / IterativeScalarSolver
// (ddecal/gain_solvers/IterativeDiagonalSolver.cc:38-222,
// IterativeScalarSolver.cc:30-229), restated for one streaming pass per
// iteration:
//
//   The reference subtracts every direction from the data, then for each
//   direction d adds d back and accumulates, per antenna a and polarization,
//     num_a(d) = sum_b  R_d,ab g_b conj(M_d,ab)   den_a(d) = sum_b |g_b M_d,ab|^2
//   with R_d = R + g_a M_d g_b^H.  Since g is constant over the visibilities
//   of one baseline within one solution slot,
//     num_a(d) = g_a den_a(d) + sum_b g_b P_ab(d),  P_ab(d) = sum_vis R conj(M_d)
//     den_a(d) = sum_b |g_b|^2 Q_ab(d),            Q_ab(d) = sum_vis |M_d|^2
//   so one pass that reads the data and each model direction once per
//   visibility gives every direction's normal equations (the add-back term
//   g_a den_a is applied in the finalisation), and the per-antenna reduction
//   runs once per baseline slot instead of once per visibility.
//
// Device layout: every channel block is repacked once per upload into slabs.
// A slab is a set of "runs" (baselines, or generic groups of visibilities that
// share both antennas and every direction's solution index) x T time steps x
// L channels, stored [T][L][R] (runs fastest) for the data and [dir][T][L][R]
// for the model, so that a warp's 32 runs are 32 consecutive 16-byte
// visibilities: each model element is read from HBM exactly once per
// iteration with full coalescing.
//
// Kernels per iteration (all on one stream, captured in one CUDA graph whose
// while-node runs the whole iterate-until-converged loop):
//   make_finite_kernel  SolverBase::MakeSolutionsFinite{1,2}Pol (only acts on
//                       channel blocks flagged non-finite)
//   stream_kernel       persistent: residual, per-direction P/Q sums, per-CTA
//                       shared-memory antenna accumulators, one partial slot
//                       per (CTA, slab) visit -- no global atomics
//   finalize_kernel     fixed-order compensated merge of the partial slots,
//                       FP64 num/den + add-back, SolverBase::Step,
//                       AssignSolutions norm, DetectStall and the stopping
//                       rule (last block), which sets the graph's loop
//                       condition.
#include "ddsolve_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <type_traits>
#include <vector>

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kInvalidKey = 0xFFFFFFFFu;
constexpr uint32_t kMaxAntennas = 65535;

// ---------------------------------------------------------------------------
// Device-side plan structures
// ---------------------------------------------------------------------------
struct SlabDesc {
  const void* data;         // [T][L][R] elements
  const void* model;        // [n_dir][T][L][R] elements
  const uint32_t* run_ant;  // [R] antenna1 | antenna2 << 16
  uint32_t cb, T, L, R;
  uint32_t sol_off;  // first of n_dir entries in slab_sol
  uint32_t pad;
};

struct Visit {
  uint32_t slab, run_lo, run_hi, pad;
};

struct DevSettings {
  uint32_t max_iterations;
  uint32_t min_iterations;
  double accuracy;
  double constraint_accuracy;
  double step_size;
  int32_t detect_stalling;
  int32_t phase_only;
  double step_diff_sigma;
  uint32_t hard_cap;
  uint32_t pad;
};

struct LoopState {
  uint32_t iteration;
  int32_t done;
  int32_t has_converged;
  int32_t has_stalled;
  uint32_t n_var_count;
  uint32_t blocks_done;
  double step_mean;
  double step_var;
};

struct StreamParams {
  const SlabDesc* slabs;
  const Visit* visits;
  const uint32_t* cta_visit_off;
  const uint32_t* slab_sol;
  const double2* solutions;
  float* partials;
  uint32_t n_ant, n_dir, n_sub, ng;
};

struct FinParams {
  const float* partials;
  const uint32_t* fin_off;     // [n_cb * n_sub + 1]
  const uint32_t* fin_visits;  // visit indices
  const uint32_t* dir_of_sub;  // [n_sub]
  double2* solutions;          // [n_cb][n_ant][n_sub][NPOL]
  double2* next_out;           // host mode output
  uint32_t n_cb, n_ant, n_dir, n_sub;
  int32_t host_mode;
  const DevSettings* settings;
  double* block_sum;
  uint32_t* block_cnt;
  LoopState* state;
  uint32_t* nonfinite;  // [n_cb]
  double* step_magnitudes;
  cudaGraphConditionalHandle handle;
  int32_t use_handle;
};

// ---------------------------------------------------------------------------
// Complex helpers (float2 / double2)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cmul_conj(float2 a, float2 b) {  // a*conj(b)
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cconj(float2 a) {
  return make_float2(a.x, -a.y);
}
__device__ __forceinline__ float cnorm(float2 a) {
  return fmaf(a.x, a.x, a.y * a.y);
}

// Polarization of the row (left gain) and column (right gain) of correlation
// c. NCORR = 4 is the row-major 2x2 [XX XY; YX YY]; NCORR = 2 is XX/YY; a
// scalar solution (NPOL = 1) applies one gain to every correlation.
template <int NCORR, int NPOL>
__device__ __forceinline__ constexpr int RowPol(int c) {
  return NPOL == 1 ? 0 : (NCORR == 4 ? (c >> 1) : c);
}
template <int NCORR, int NPOL>
__device__ __forceinline__ constexpr int ColPol(int c) {
  return NPOL == 1 ? 0 : (NCORR == 4 ? (c & 1) : c);
}

template <int NCORR>
__device__ __forceinline__ void LoadVis(const void* base, size_t idx,
                                        float2 (&v)[NCORR]) {
  if constexpr (NCORR == 1) {
    v[0] = __ldg(reinterpret_cast<const float2*>(base) + idx);
  } else if constexpr (NCORR == 2) {
    const float4 x = __ldg(reinterpret_cast<const float4*>(base) + idx);
    v[0] = make_float2(x.x, x.y);
    v[1] = make_float2(x.z, x.w);
  } else {
    const float4* p = reinterpret_cast<const float4*>(base) + 2 * idx;
    const float4 x = __ldg(p);
    const float4 y = __ldg(p + 1);
    v[0] = make_float2(x.x, x.y);
    v[1] = make_float2(x.z, x.w);
    v[2] = make_float2(y.x, y.y);
    v[3] = make_float2(y.z, y.w);
  }
}

// ---------------------------------------------------------------------------
// Pack kernel: reference SolveData layout -> slab layout.
// dst element (t, ch, r) of a slab <- source visibility
//   src_base + t * tstride + run_src[r] + ch   (zero if ch >= run_len[r])
// ---------------------------------------------------------------------------
struct PackSlab {
  uint64_t dst_elem_off;  // into the cb's packed data buffer
  uint64_t src_base;
  uint64_t tstride;
  uint32_t T, L, R, run_off;
};

template <int E>  // element size in bytes (8, 16, 32)
__global__ void pack_kernel(const PackSlab* __restrict__ slabs, uint32_t slab,
                            const uint32_t* __restrict__ run_src,
                            const uint32_t* __restrict__ run_len,
                            const char* __restrict__ src_data,
                            const char* __restrict__ src_model, uint64_t n_vis,
                            uint32_t n_dir, uint64_t n_elems_cb,
                            char* __restrict__ dst_data,
                            char* __restrict__ dst_model) {
  const PackSlab s = slabs[slab];
  const uint64_t tlr = uint64_t(s.T) * s.L * s.R;
  using Word = typename std::conditional<E == 8, float2, float4>::type;
  constexpr int kWords = E / int(sizeof(Word));
  for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e < tlr;
       e += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t r = uint32_t(e % s.R);
    const uint64_t tl = e / s.R;
    const uint32_t ch = uint32_t(tl % s.L);
    const uint32_t t = uint32_t(tl / s.L);
    const bool valid = ch < run_len[s.run_off + r];
    const uint64_t v = s.src_base + t * s.tstride + run_src[s.run_off + r] + ch;
    const uint64_t dst = s.dst_elem_off + e;
    Word zero;
    memset(&zero, 0, sizeof(zero));
    for (int w = 0; w < kWords; ++w) {
      reinterpret_cast<Word*>(dst_data)[dst * kWords + w] =
          valid ? reinterpret_cast<const Word*>(src_data)[v * kWords + w] : zero;
    }
    // model block of the slab: [n_dir][T][L][R] starting at n_dir * dst_elem_off
    for (uint32_t d = 0; d < n_dir; ++d) {
      const uint64_t md = uint64_t(n_dir) * s.dst_elem_off + d * tlr + e;
      const uint64_t ms = d * n_vis + v;
      for (int w = 0; w < kWords; ++w) {
        reinterpret_cast<Word*>(dst_model)[md * kWords + w] =
            valid ? reinterpret_cast<const Word*>(src_model)[ms * kWords + w]
                  : zero;
      }
    }
  }
  (void)n_elems_cb;
}

// ---------------------------------------------------------------------------
// make_finite_kernel: SolverBase::MakeSolutionsFinite1Pol / 2Pol
// (ddecal/gain_solvers/SolverBase.cc:316-371), one block per channel block.
// The 2-pol version averages |pol 0| for both polarizations, as the
// reference does (SolverBase.cc:354). It only runs on blocks flagged
// non-finite by the previous finalisation (or by a new upload).
// Block 0 also resets the graph loop condition to "stop"; the finalisation
// sets it back to "continue", so a loop whose control step did not run ends.
// ---------------------------------------------------------------------------
template <int NPOL>
__global__ void __launch_bounds__(kThreads)
    make_finite_kernel(double2* __restrict__ sols, uint32_t* nonfinite,
                       uint32_t per_cb, cudaGraphConditionalHandle handle,
                       int use_handle) {
  if (use_handle && blockIdx.x == 0 && threadIdx.x == 0)
    cudaGraphSetConditional(handle, 0);
  const uint32_t cb = blockIdx.x;
  if (nonfinite[cb] == 0) return;
  double2* s = sols + size_t(cb) * per_cb;
  __shared__ double red_sum[kThreads];
  __shared__ uint32_t red_cnt[kThreads];
  double sum = 0.0;
  uint32_t cnt = 0;
  auto finite = [](double2 v) { return isfinite(v.x) && isfinite(v.y); };
  for (uint32_t i = threadIdx.x * NPOL; i < per_cb; i += blockDim.x * NPOL) {
    bool ok = finite(s[i]);
    if (NPOL == 2) ok = ok && finite(s[i + 1]);
    if (ok) {
      sum += hypot(s[i].x, s[i].y);
      ++cnt;
    }
  }
  red_sum[threadIdx.x] = sum;
  red_cnt[threadIdx.x] = cnt;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      red_sum[threadIdx.x] += red_sum[threadIdx.x + w];
      red_cnt[threadIdx.x] += red_cnt[threadIdx.x + w];
    }
    __syncthreads();
  }
  const double average =
      red_cnt[0] == 0 ? 1.0 : red_sum[0] / double(red_cnt[0]);
  for (uint32_t i = threadIdx.x * NPOL; i < per_cb; i += blockDim.x * NPOL) {
    bool ok = finite(s[i]);
    if (NPOL == 2) ok = ok && finite(s[i + 1]);
    if (!ok)
      for (int p = 0; p < NPOL; ++p) s[i + p] = make_double2(average, 0.0);
  }
  __syncthreads();
  if (threadIdx.x == 0) nonfinite[cb] = 0;
}

// ---------------------------------------------------------------------------
// stream_kernel: the hot loop. Persistent CTAs walk their list of (slab, run
// range) visits; each group of `ng` lanes owns one run and ceil(n_dir/ng)
// directions (direction d = g + k*ng for lane g of the group).
//
// Per visibility:  R = D - sum_d G_d (.) M_d     (G_d = g_a1 conj(g_a2))
//                  P_d += R conj(M_d),  Q_d += |M_d|^2
// Per run (after T*L visibilities), per direction and solution polarization:
//   antenna 1: num += g_a2 P,        den += |g_a2|^2 Q  (segmented warp sum)
//   antenna 2: num += g_a1 conj(P),  den += |g_a1|^2 Q  (shared atomics)
// Accumulators: shared float [n_ant][n_dir][NPOL][3]; flushed per visit.
// ---------------------------------------------------------------------------
template <int NCORR, int NPOL, int DMAX>
__global__ void __launch_bounds__(kThreads)
    stream_kernel(const StreamParams p) {
  extern __shared__ float4 smem4[];
  float* acc = reinterpret_cast<float*>(smem4);
  const uint32_t acc_n = p.n_ant * p.n_dir * NPOL * 3;
  float2* gtab = reinterpret_cast<float2*>(acc + ((acc_n + 3u) & ~3u));
  const uint32_t gtab_n = p.n_ant * p.n_dir * NPOL;

  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int ng = int(p.ng);
  const int g = tid & (ng - 1);
  const int slot = tid / ng;
  const int wslot = lane / ng;
  const int nslots = 32 / ng;
  const int runs_per_block = blockDim.x / ng;
  const int nd_max = int((p.n_dir + ng - 1) / ng);
  const int nd = int(p.n_dir) > g ? (int(p.n_dir) - g + ng - 1) / ng : 0;
  const uint32_t n_dir = p.n_dir;

  const uint32_t v_begin = p.cta_visit_off[blockIdx.x];
  const uint32_t v_end = p.cta_visit_off[blockIdx.x + 1];
  for (uint32_t vi = v_begin; vi < v_end; ++vi) {
    const Visit vis = p.visits[vi];
    const SlabDesc sl = p.slabs[vis.slab];
    for (uint32_t i = tid; i < acc_n; i += blockDim.x) acc[i] = 0.f;
    for (uint32_t i = tid; i < gtab_n; i += blockDim.x) {
      const uint32_t ant = i / (n_dir * NPOL);
      const uint32_t rem = i - ant * n_dir * NPOL;
      const uint32_t d = rem / NPOL;
      const uint32_t pol = rem - d * NPOL;
      const uint32_t s = p.slab_sol[sl.sol_off + d];
      const double2 gv =
          p.solutions[(size_t(sl.cb * p.n_ant + ant) * p.n_sub + s) * NPOL +
                      pol];
      gtab[i] = make_float2(float(gv.x), float(gv.y));
    }
    __syncthreads();
    const size_t tlr = size_t(sl.T) * sl.L * sl.R;

    for (uint32_t run0 = vis.run_lo; run0 < vis.run_hi; run0 += runs_per_block) {
      const uint32_t run = run0 + slot;
      const bool active = run < vis.run_hi;
      uint32_t a1 = 0, a2 = 0;
      if (active) {
        const uint32_t ap = sl.run_ant[run];
        a1 = ap & 0xFFFFu;
        a2 = ap >> 16;
      }
      // Gains of the two antennas of this run, per direction handled here.
      float2 G[DMAX][NCORR];
#pragma unroll
      for (int k = 0; k < DMAX; ++k) {
        float2 ga[NPOL], gb[NPOL];
#pragma unroll
        for (int q = 0; q < NPOL; ++q) {
          ga[q] = make_float2(0.f, 0.f);
          gb[q] = make_float2(0.f, 0.f);
        }
        if (active && k < nd) {
          const uint32_t d = g + k * ng;
#pragma unroll
          for (int q = 0; q < NPOL; ++q) {
            ga[q] = gtab[(a1 * n_dir + d) * NPOL + q];
            gb[q] = gtab[(a2 * n_dir + d) * NPOL + q];
          }
        }
#pragma unroll
        for (int c = 0; c < NCORR; ++c)
          G[k][c] = cmul_conj(ga[RowPol<NCORR, NPOL>(c)],
                              gb[ColPol<NCORR, NPOL>(c)]);
      }
      float2 P[DMAX][NCORR];
      float Q[DMAX][NCORR];
#pragma unroll
      for (int k = 0; k < DMAX; ++k)
#pragma unroll
        for (int c = 0; c < NCORR; ++c) {
          P[k][c] = make_float2(0.f, 0.f);
          Q[k][c] = 0.f;
        }

      for (uint32_t t = 0; t < sl.T; ++t) {
        for (uint32_t ch = 0; ch < sl.L; ++ch) {
          const size_t e = (size_t(t) * sl.L + ch) * sl.R + run;
          float2 Rv[NCORR];
#pragma unroll
          for (int c = 0; c < NCORR; ++c) Rv[c] = make_float2(0.f, 0.f);
          if (active && g == 0) LoadVis<NCORR>(sl.data, e, Rv);
          float2 M[DMAX][NCORR];
#pragma unroll
          for (int k = 0; k < DMAX; ++k) {
            if (active && k < nd) {
              LoadVis<NCORR>(sl.model, size_t(g + k * ng) * tlr + e, M[k]);
            } else {
#pragma unroll
              for (int c = 0; c < NCORR; ++c) M[k][c] = make_float2(0.f, 0.f);
            }
          }
#pragma unroll
          for (int k = 0; k < DMAX; ++k)
#pragma unroll
            for (int c = 0; c < NCORR; ++c) {
              const float2 gm = cmul(G[k][c], M[k][c]);
              Rv[c].x -= gm.x;
              Rv[c].y -= gm.y;
            }
          for (int m = 1; m < ng; m <<= 1) {
#pragma unroll
            for (int c = 0; c < NCORR; ++c) {
              Rv[c].x += __shfl_xor_sync(0xFFFFFFFFu, Rv[c].x, m);
              Rv[c].y += __shfl_xor_sync(0xFFFFFFFFu, Rv[c].y, m);
            }
          }
#pragma unroll
          for (int k = 0; k < DMAX; ++k)
#pragma unroll
            for (int c = 0; c < NCORR; ++c) {
              const float2 rm = cmul_conj(Rv[c], M[k][c]);
              P[k][c].x += rm.x;
              P[k][c].y += rm.y;
              Q[k][c] += cnorm(M[k][c]);
            }
        }
      }

      // Segmented reduction over runs of the warp that share antenna 1.
      const uint32_t key = active ? a1 : kInvalidKey;
      const uint32_t next_key = __shfl_down_sync(0xFFFFFFFFu, key, ng);
      const uint32_t prev_key = __shfl_up_sync(0xFFFFFFFFu, key, ng);
      const bool tail = (wslot == nslots - 1) || (next_key != key);
      const bool head = (wslot == 0) || (prev_key != key);
      const uint32_t tail_mask = __ballot_sync(0xFFFFFFFFu, tail);
      const int base = wslot * ng;
      const int seg_end = base + (__ffs(tail_mask >> base) - 1) + g;

#pragma unroll
      for (int k = 0; k < DMAX; ++k) {
        if (k >= nd_max) break;
        const bool mine = active && k < nd;
        const uint32_t d = g + k * ng;
        float2 ga[NPOL], gb[NPOL];
#pragma unroll
        for (int q = 0; q < NPOL; ++q) {
          ga[q] = mine ? gtab[(a1 * n_dir + d) * NPOL + q] : make_float2(0.f, 0.f);
          gb[q] = mine ? gtab[(a2 * n_dir + d) * NPOL + q] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int q = 0; q < NPOL; ++q) {
          float2 n1 = make_float2(0.f, 0.f), n2 = make_float2(0.f, 0.f);
          float d1 = 0.f, d2 = 0.f;
#pragma unroll
          for (int c = 0; c < NCORR; ++c) {
            const int rp = RowPol<NCORR, NPOL>(c);
            const int cp = ColPol<NCORR, NPOL>(c);
            if (rp == q) {
              const float2 t1 = cmul(gb[cp], P[k][c]);
              n1.x += t1.x;
              n1.y += t1.y;
              d1 += cnorm(gb[cp]) * Q[k][c];
            }
            if (cp == q) {
              const float2 t2 = cmul(ga[rp], cconj(P[k][c]));
              n2.x += t2.x;
              n2.y += t2.y;
              d2 += cnorm(ga[rp]) * Q[k][c];
            }
          }
          if (mine) {
            float* a = acc + ((a2 * n_dir + d) * NPOL + q) * 3;
            atomicAdd(a + 0, n2.x);
            atomicAdd(a + 1, n2.y);
            atomicAdd(a + 2, d2);
          }
          for (int off = ng; off < 32; off <<= 1) {
            const float ox = __shfl_down_sync(0xFFFFFFFFu, n1.x, off);
            const float oy = __shfl_down_sync(0xFFFFFFFFu, n1.y, off);
            const float od = __shfl_down_sync(0xFFFFFFFFu, d1, off);
            if (lane + off <= seg_end) {
              n1.x += ox;
              n1.y += oy;
              d1 += od;
            }
          }
          if (head && mine) {
            float* a = acc + ((a1 * n_dir + d) * NPOL + q) * 3;
            atomicAdd(a + 0, n1.x);
            atomicAdd(a + 1, n1.y);
            atomicAdd(a + 2, d1);
          }
        }
      }
    }
    __syncthreads();
    float* out = p.partials + size_t(vi) * acc_n;
    for (uint32_t i = tid; i < acc_n; i += blockDim.x) out[i] = acc[i];
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// finalize_kernel: one thread per (channel block, antenna, sub-solution).
// ---------------------------------------------------------------------------
struct NeumaierSum {  // compensated FP32 summation (two-sum)
  float s = 0.f, c = 0.f;
  __device__ __forceinline__ void Add(float x) {
    const float t = s + x;
    if (fabsf(s) >= fabsf(x))
      c += (s - t) + x;
    else
      c += (x - t) + s;
    s = t;
  }
  __device__ __forceinline__ float Value() const { return s + c; }
};

__device__ __forceinline__ double2 dmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ bool dfinite(double2 a) {
  return isfinite(a.x) && isfinite(a.y);
}
// 1 / s (Smith's algorithm), as std::complex<double> division does for
// finite operands.
__device__ __forceinline__ double2 dinv(double2 s) {
  if (fabs(s.x) >= fabs(s.y)) {
    const double r = s.y / s.x;
    const double den = s.x + s.y * r;
    return make_double2(1.0 / den, -r / den);
  } else {
    const double r = s.x / s.y;
    const double den = s.x * r + s.y;
    return make_double2(r / den, -1.0 / den);
  }
}

template <int NPOL>
__global__ void __launch_bounds__(kThreads) finalize_kernel(const FinParams p) {
  const uint32_t n_items = p.n_cb * p.n_ant * p.n_sub;
  const uint32_t item = blockIdx.x * blockDim.x + threadIdx.x;
  double norm_sum = 0.0;
  uint32_t norm_cnt = 0;
  const DevSettings st = *p.settings;
  if (item < n_items) {
    const uint32_t cb = item / (p.n_ant * p.n_sub);
    const uint32_t rem = item - cb * p.n_ant * p.n_sub;
    const uint32_t ant = rem / p.n_sub;
    const uint32_t s = rem - ant * p.n_sub;
    const uint32_t d = p.dir_of_sub[s];
    const uint32_t acc_n = p.n_ant * p.n_dir * NPOL * 3;
    NeumaierSum nr[NPOL], ni[NPOL], dn[NPOL];
    const uint32_t j0 = p.fin_off[cb * p.n_sub + s];
    const uint32_t j1 = p.fin_off[cb * p.n_sub + s + 1];
    for (uint32_t j = j0; j < j1; ++j) {
      const float* a = p.partials + size_t(p.fin_visits[j]) * acc_n +
                       ((ant * p.n_dir + d) * NPOL) * 3;
#pragma unroll
      for (int q = 0; q < NPOL; ++q) {
        nr[q].Add(a[q * 3 + 0]);
        ni[q].Add(a[q * 3 + 1]);
        dn[q].Add(a[q * 3 + 2]);
      }
    }
    double2* sol = p.solutions + (size_t(cb) * p.n_ant * p.n_sub +
                                  size_t(ant) * p.n_sub + s) * NPOL;
    double2 old[NPOL], nxt[NPOL];
#pragma unroll
    for (int q = 0; q < NPOL; ++q) {
      old[q] = sol[q];
      const float den = dn[q].Value();
      if (den == 0.f) {
        // IterativeDiagonalSolver.cc:212-214 / IterativeScalarSolver.cc:189-190
        nxt[q] = make_double2(nan(""), 0.0);
      } else {
        // num = g_a den + sum_b g_b P  =>  num / den = g_a + (sum_b g_b P)/den,
        // with g_a the single-precision gain the reference uses for add-back.
        const double ga_r = double(float(old[q].x));
        const double ga_i = double(float(old[q].y));
        nxt[q] = make_double2(ga_r + double(nr[q].Value()) / double(den),
                              ga_i + double(ni[q].Value()) / double(den));
      }
    }
    if (p.host_mode) {
      double2* out = p.next_out + (size_t(cb) * p.n_ant * p.n_sub +
                                   size_t(ant) * p.n_sub + s) * NPOL;
#pragma unroll
      for (int q = 0; q < NPOL; ++q) out[q] = nxt[q];
    } else {
      // SolverBase::Step (SolverBase.cc:88-158)
#pragma unroll
      for (int q = 0; q < NPOL; ++q) {
        if (!st.phase_only) {
          nxt[q] = make_double2(old[q].x * (1.0 - st.step_size) + nxt[q].x * st.step_size,
                                old[q].y * (1.0 - st.step_size) + nxt[q].y * st.step_size);
        } else {
          const double from = atan2(old[q].y, old[q].x);
          double dist = atan2(nxt[q].y, nxt[q].x) - from;
          if (dist > M_PI)
            dist -= 2.0 * M_PI;
          else if (dist < -M_PI)
            dist += 2.0 * M_PI;
          double sn, cs;
          sincos(from + st.step_size * dist, &sn, &cs);
          nxt[q] = make_double2(cs, sn);
        }
      }
      // SolverBase::AssignSolutions norm (SolverBase.cc:234-285)
      if (NPOL == 1) {
        if (old[0].x != 0.0 || old[0].y != 0.0) {
          const double2 inv = dinv(old[0]);
          const double2 diff = dmul(make_double2(nxt[0].x - old[0].x,
                                                 nxt[0].y - old[0].y),
                                    inv);
          const double a = hypot(diff.x, diff.y);
          if (isfinite(a)) {
            norm_sum += a;
            norm_cnt += 1;
          }
        }
      } else {
        const double2 inv0 = dinv(old[0]);
        const double2 inv1 = dinv(old[NPOL - 1]);
        if (dfinite(inv0) && dfinite(inv1)) {
          const double2 d0 = dmul(make_double2(nxt[0].x - old[0].x,
                                               nxt[0].y - old[0].y), inv0);
          const double2 d1 = dmul(make_double2(nxt[NPOL - 1].x - old[NPOL - 1].x,
                                               nxt[NPOL - 1].y - old[NPOL - 1].y),
                                  inv1);
          const double sumabs = hypot(d0.x, d0.y) + hypot(d1.x, d1.y);
          if (isfinite(sumabs)) {
            norm_sum += sumabs;
            norm_cnt += 2;
          }
        }
      }
      bool all_finite = true;
#pragma unroll
      for (int q = 0; q < NPOL; ++q) {
        sol[q] = nxt[q];
        all_finite = all_finite && dfinite(nxt[q]);
      }
      if (!all_finite) p.nonfinite[cb] = 1u;
    }
  }
  if (p.host_mode) return;

  // Block reduction of the norm, then the last block finishes the iteration.
  __shared__ double s_sum[kThreads];
  __shared__ uint32_t s_cnt[kThreads];
  __shared__ bool s_last;
  s_sum[threadIdx.x] = norm_sum;
  s_cnt[threadIdx.x] = norm_cnt;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s_sum[threadIdx.x] += s_sum[threadIdx.x + w];
      s_cnt[threadIdx.x] += s_cnt[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    p.block_sum[blockIdx.x] = s_sum[0];
    p.block_cnt[blockIdx.x] = s_cnt[0];
    __threadfence();
    const uint32_t prev = atomicAdd(&p.state->blocks_done, 1u);
    s_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  double sum = 0.0;
  uint64_t cnt = 0;
  for (uint32_t b = 0; b < gridDim.x; ++b) {
    sum += reinterpret_cast<volatile double*>(p.block_sum)[b];
    cnt += reinterpret_cast<volatile uint32_t*>(p.block_cnt)[b];
  }
  LoopState& ls = *p.state;
  ls.blocks_done = 0;
  // AssignSolutions (SolverBase.cc:297-306), no constraints: accuracy.
  const double mag = cnt == 0 ? 0.0 : sum / st.step_size / double(cnt);
  const uint32_t it = ls.iteration + 1;
  ls.iteration = it;
  if (it <= st.hard_cap) p.step_magnitudes[it - 1] = mag;
  const bool converged = mag <= st.accuracy;
  // ReachedStoppingCriterion / DetectStall (SolverBase.h:274-285,
  // SolverBase.cc:63-86)
  bool stalled = false;
  if (st.detect_stalling) {
    if (it == 1) {
      ls.n_var_count = 1;
      ls.step_mean = mag;
      ls.step_var = 0.0;
    } else {
      ls.n_var_count += 1;
      const double delta_1 = mag - ls.step_mean;
      ls.step_mean += delta_1 / double(ls.n_var_count);
      const double delta_2 = mag - ls.step_mean;
      ls.step_var += delta_1 * delta_2;
    }
    if (it >= 30)
      stalled = ls.step_mean <
                st.step_diff_sigma * sqrt(ls.step_var / double(ls.n_var_count));
  }
  const bool ready = it >= st.max_iterations || converged || stalled;
  const bool stop = (it >= st.min_iterations && ready) || it >= st.hard_cap;
  ls.has_converged = converged;
  ls.has_stalled = stalled;
  ls.done = stop;
  if (p.use_handle) cudaGraphSetConditional(p.handle, stop ? 0u : 1u);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
thread_local std::string g_last_error = "no error";

#define DDS_CHECK_CUDA(ctx, call)                                         \
  do {                                                                    \
    const cudaError_t err_ = (call);                                      \
    if (err_ != cudaSuccess) {                                            \
      return (ctx)->Fail(DDSOLVE_E_CUDA, std::string(#call) + ": " +      \
                                             cudaGetErrorString(err_));   \
    }                                                                     \
  } while (0)

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept
      : ptr(o.ptr), bytes(o.bytes), realloc_flag(o.realloc_flag) {
    o.ptr = nullptr;
    o.bytes = 0;
  }
  ~DevBuf() {
    if (ptr) cudaFree(ptr);
  }
  bool realloc_flag = false;  // set when Reserve() moved the buffer
  cudaError_t Reserve(size_t n) {
    if (n <= bytes && ptr) return cudaSuccess;
    realloc_flag = true;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
    const cudaError_t e = cudaMalloc(&ptr, std::max<size_t>(n, 256));
    if (e == cudaSuccess) bytes = std::max<size_t>(n, 256);
    return e;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(ptr);
  }
};

struct HostSlab {
  uint32_t T, L, R;
  uint64_t elem_off;  // within the channel block's packed buffer
  uint64_t src_base, tstride;
  uint32_t run_off;
  std::vector<uint32_t> sol;  // [n_dir]
};

bool SameLayout(const std::vector<HostSlab>& a, const std::vector<HostSlab>& b) {
  if (a.size() != b.size()) return false;
  for (size_t i = 0; i < a.size(); ++i)
    if (a[i].T != b[i].T || a[i].L != b[i].L || a[i].R != b[i].R ||
        a[i].elem_off != b[i].elem_off || a[i].run_off != b[i].run_off ||
        a[i].sol != b[i].sol)
      return false;
  return true;
}

struct ChannelBlockStore {
  bool set = false;
  uint64_t n_vis = 0;
  uint64_t n_elems = 0;
  std::vector<HostSlab> slabs;
  std::vector<uint32_t> run_ant, run_src, run_len;
  DevBuf data, model, run_ant_dev;
  // Layout of the previous upload; an upload with the same layout into the
  // same buffers keeps the streaming plan (and its CUDA graph) valid.
  std::vector<HostSlab> prev_slabs;
  std::vector<uint32_t> prev_run_ant;
};

using StreamFn = void (*)(StreamParams);

}  // namespace

struct ddsolve_ctx {
  // dimensions
  uint32_t n_ant = 0, n_dir = 0, n_cb = 0, n_corr = 0, n_pol = 0, n_sub = 0;
  std::vector<uint32_t> n_sol_per_dir, sol_start, dir_of_sub;
  size_t elem_bytes = 0;
  int device = 0;
  int n_sm = 0;
  cudaStream_t stream = nullptr;
  std::string err = "no error";
  ddsolve_settings settings{};
  uint32_t tune_ng = 0, tune_max_times = 0;

  std::vector<ChannelBlockStore> cbs;
  DevBuf staging, pack_desc, run_src_dev, run_len_dev;

  // plan
  bool plan_dirty = true;
  uint32_t ng = 1, dmax = 1;
  StreamFn stream_fn = nullptr;
  size_t stream_smem = 0;
  uint32_t n_ctas = 0, n_visits = 0, fin_blocks = 0;
  DevBuf d_slabs, d_visits, d_cta_off, d_slab_sol, d_partials, d_fin_off,
      d_fin_visits, d_dir_of_sub, d_block_sum, d_block_cnt;
  // solver state
  DevBuf d_sol, d_next, d_state, d_nonfinite, d_mags, d_settings;
  // graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraphConditionalHandle handle = 0;
  bool graph_ok = false;
  uint64_t last_launches = 0;

  int Fail(int code, const std::string& msg) {
    err = msg;
    return code;
  }
  ~ddsolve_ctx() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    if (stream) cudaStreamDestroy(stream);
  }
  void DestroyGraph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
    graph_ok = false;
  }
};

namespace {

// Registry of streaming-kernel instantiations keyed by (ncorr, npol, dmax).
struct KernelEntry {
  int ncorr, npol, dmax;
  const void* fn;
};

template <int NC, int NP, int DM>
constexpr KernelEntry Entry() {
  return KernelEntry{NC, NP, DM,
                     reinterpret_cast<const void*>(&stream_kernel<NC, NP, DM>)};
}

const std::vector<KernelEntry>& Kernels() {
  static const std::vector<KernelEntry> k = {
      Entry<2, 2, 1>(), Entry<2, 2, 2>(), Entry<2, 2, 3>(), Entry<2, 2, 4>(),
      Entry<2, 2, 5>(), Entry<2, 2, 6>(), Entry<2, 2, 8>(),
      Entry<4, 2, 1>(), Entry<4, 2, 2>(), Entry<4, 2, 4>(),
      Entry<1, 1, 1>(), Entry<1, 1, 2>(), Entry<1, 1, 4>(), Entry<1, 1, 8>(),
      Entry<2, 1, 1>(), Entry<2, 1, 2>(), Entry<2, 1, 4>(), Entry<2, 1, 8>(),
      Entry<4, 1, 1>(), Entry<4, 1, 2>(), Entry<4, 1, 4>(),
  };
  return k;
}

// Smallest instantiated dmax >= need for this (ncorr, npol); 0 if none.
const KernelEntry* FindKernel(int ncorr, int npol, int need) {
  const KernelEntry* best = nullptr;
  for (const KernelEntry& e : Kernels())
    if (e.ncorr == ncorr && e.npol == npol && e.dmax >= need &&
        (!best || e.dmax < best->dmax))
      best = &e;
  return best;
}

int PreferredDirsPerLane(int ncorr) { return ncorr == 4 ? 2 : (ncorr == 2 ? 5 : 8); }

size_t ElemBytes(uint32_t ncorr) { return size_t(ncorr) * 8; }

int CheckDims(const ddsolve_dims* dims) {
  if (!dims) return DDSOLVE_E_INVALID;
  if (dims->n_antennas < 2 || dims->n_antennas > kMaxAntennas)
    return DDSOLVE_E_INVALID;
  if (dims->n_directions == 0 || dims->n_channel_blocks == 0)
    return DDSOLVE_E_INVALID;
  if (!dims->n_solutions_per_direction) return DDSOLVE_E_INVALID;
  const uint32_t nc = dims->n_correlations, np = dims->n_solution_polarizations;
  if (!((nc == 2 && np == 2) || (nc == 4 && np == 2) || (nc == 1 && np == 1) ||
        (nc == 2 && np == 1) || (nc == 4 && np == 1)))
    return DDSOLVE_E_UNSUPPORTED;
  for (uint32_t d = 0; d < dims->n_directions; ++d)
    if (dims->n_solutions_per_direction[d] == 0) return DDSOLVE_E_INVALID;
  return DDSOLVE_OK;
}

// Uploads the staged reference-layout block and packs it into slabs.
int UploadAndPack(ddsolve_ctx* ctx, ChannelBlockStore& cb, const float* data,
                  const float* model) {
  const size_t E = ctx->elem_bytes;
  const size_t src_bytes = size_t(cb.n_vis) * E * (1 + ctx->n_dir);
  DDS_CHECK_CUDA(ctx, ctx->staging.Reserve(src_bytes));
  cb.data.realloc_flag = cb.model.realloc_flag = cb.run_ant_dev.realloc_flag = false;
  DDS_CHECK_CUDA(ctx, cb.data.Reserve(cb.n_elems * E));
  DDS_CHECK_CUDA(ctx, cb.model.Reserve(cb.n_elems * E * ctx->n_dir));
  DDS_CHECK_CUDA(ctx, cb.run_ant_dev.Reserve(cb.run_ant.size() * 4));
  DDS_CHECK_CUDA(ctx, ctx->run_src_dev.Reserve(cb.run_src.size() * 4));
  DDS_CHECK_CUDA(ctx, ctx->run_len_dev.Reserve(cb.run_len.size() * 4));
  std::vector<PackSlab> ps(cb.slabs.size());
  for (size_t i = 0; i < cb.slabs.size(); ++i) {
    const HostSlab& s = cb.slabs[i];
    ps[i] = PackSlab{s.elem_off, s.src_base, s.tstride, s.T, s.L, s.R, s.run_off};
  }
  DDS_CHECK_CUDA(ctx, ctx->pack_desc.Reserve(ps.size() * sizeof(PackSlab)));
  char* st = ctx->staging.as<char>();
  if (cb.n_vis) {
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(st, data, size_t(cb.n_vis) * E,
                                        cudaMemcpyHostToDevice, ctx->stream));
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(st + size_t(cb.n_vis) * E, model,
                                        size_t(cb.n_vis) * E * ctx->n_dir,
                                        cudaMemcpyHostToDevice, ctx->stream));
  }
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(cb.run_ant_dev.ptr, cb.run_ant.data(),
                                      cb.run_ant.size() * 4,
                                      cudaMemcpyHostToDevice, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->run_src_dev.ptr, cb.run_src.data(),
                                      cb.run_src.size() * 4,
                                      cudaMemcpyHostToDevice, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->run_len_dev.ptr, cb.run_len.data(),
                                      cb.run_len.size() * 4,
                                      cudaMemcpyHostToDevice, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->pack_desc.ptr, ps.data(),
                                      ps.size() * sizeof(PackSlab),
                                      cudaMemcpyHostToDevice, ctx->stream));
  for (size_t i = 0; i < cb.slabs.size(); ++i) {
    const uint64_t tlr = uint64_t(cb.slabs[i].T) * cb.slabs[i].L * cb.slabs[i].R;
    if (tlr == 0) continue;
    const uint32_t blocks =
        uint32_t(std::min<uint64_t>((tlr + 255) / 256, uint64_t(ctx->n_sm) * 8));
    if (E == 8)
      pack_kernel<8><<<blocks, 256, 0, ctx->stream>>>(
          ctx->pack_desc.as<PackSlab>(), uint32_t(i), ctx->run_src_dev.as<uint32_t>(),
          ctx->run_len_dev.as<uint32_t>(), st, st + size_t(cb.n_vis) * E, cb.n_vis,
          ctx->n_dir, cb.n_elems, cb.data.as<char>(), cb.model.as<char>());
    else if (E == 16)
      pack_kernel<16><<<blocks, 256, 0, ctx->stream>>>(
          ctx->pack_desc.as<PackSlab>(), uint32_t(i), ctx->run_src_dev.as<uint32_t>(),
          ctx->run_len_dev.as<uint32_t>(), st, st + size_t(cb.n_vis) * E, cb.n_vis,
          ctx->n_dir, cb.n_elems, cb.data.as<char>(), cb.model.as<char>());
    else
      pack_kernel<32><<<blocks, 256, 0, ctx->stream>>>(
          ctx->pack_desc.as<PackSlab>(), uint32_t(i), ctx->run_src_dev.as<uint32_t>(),
          ctx->run_len_dev.as<uint32_t>(), st, st + size_t(cb.n_vis) * E, cb.n_vis,
          ctx->n_dir, cb.n_elems, cb.data.as<char>(), cb.model.as<char>());
    DDS_CHECK_CUDA(ctx, cudaGetLastError());
  }
  // The staging and run arrays are reused by the next upload: keep the
  // stream order (a later upload's copies follow these kernels).
  const bool moved =
      cb.data.realloc_flag || cb.model.realloc_flag || cb.run_ant_dev.realloc_flag;
  if (!cb.set || moved || !SameLayout(cb.slabs, cb.prev_slabs) ||
      cb.run_ant != cb.prev_run_ant) {
    ctx->plan_dirty = true;
    cb.prev_slabs = cb.slabs;
    cb.prev_run_ant = cb.run_ant;
  }
  cb.set = true;
  return DDSOLVE_OK;
}

// Builds the streaming plan: kernel choice, CTA work split, partial slots and
// the finalisation lists.
int BuildPlan(ddsolve_ctx* ctx) {
  for (uint32_t c = 0; c < ctx->n_cb; ++c)
    if (!ctx->cbs[c].set)
      return ctx->Fail(DDSOLVE_E_STATE,
                       "channel block " + std::to_string(c) + " has no data");
  // Kernel choice: ng lanes per run so that each lane handles at most the
  // preferred number of directions.
  uint32_t ng = ctx->tune_ng;
  if (ng == 0) {
    ng = 1;
    while (ng < 32 && (ctx->n_dir + ng - 1) / ng >
                          uint32_t(PreferredDirsPerLane(int(ctx->n_corr))))
      ng <<= 1;
  }
  if (ng == 0 || ng > 32 || (ng & (ng - 1)))
    return ctx->Fail(DDSOLVE_E_INVALID, "direction groups must be a power of 2 <= 32");
  const int need = int((ctx->n_dir + ng - 1) / ng);
  const KernelEntry* ke = FindKernel(int(ctx->n_corr), int(ctx->n_pol), need);
  while (!ke && ng < 32) {
    ng <<= 1;
    ke = FindKernel(int(ctx->n_corr), int(ctx->n_pol),
                    int((ctx->n_dir + ng - 1) / ng));
  }
  if (!ke)
    return ctx->Fail(DDSOLVE_E_UNSUPPORTED, "too many directions for the kernel set");
  ctx->ng = ng;
  ctx->dmax = uint32_t(ke->dmax);
  ctx->stream_fn = reinterpret_cast<StreamFn>(const_cast<void*>(ke->fn));

  const size_t acc_n = size_t(ctx->n_ant) * ctx->n_dir * ctx->n_pol * 3;
  const size_t smem = ((acc_n + 3) & ~size_t(3)) * 4 +
                      size_t(ctx->n_ant) * ctx->n_dir * ctx->n_pol * 8;
  int max_optin = 0;
  DDS_CHECK_CUDA(ctx, cudaDeviceGetAttribute(
                          &max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                          ctx->device));
  if (smem > size_t(max_optin))
    return ctx->Fail(DDSOLVE_E_UNSUPPORTED,
                     "antenna x direction accumulators exceed shared memory");
  DDS_CHECK_CUDA(ctx, cudaFuncSetAttribute(ke->fn,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(smem)));
  int occ = 0;
  DDS_CHECK_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                          &occ, ke->fn, kThreads, smem));
  if (occ < 1) return ctx->Fail(DDSOLVE_E_UNSUPPORTED, "stream kernel cannot launch");
  ctx->stream_smem = smem;

  // Global slab list and steps.
  struct GSlab {
    uint32_t cb, idx;
  };
  std::vector<GSlab> gslabs;
  std::vector<SlabDesc> descs;
  std::vector<uint32_t> slab_sol;
  const uint32_t runs_per_block = kThreads / ng;
  struct Step {
    uint32_t slab, run_lo, run_hi;
    double w;
  };
  std::vector<Step> steps;
  for (uint32_t c = 0; c < ctx->n_cb; ++c) {
    ChannelBlockStore& cb = ctx->cbs[c];
    for (uint32_t i = 0; i < cb.slabs.size(); ++i) {
      const HostSlab& s = cb.slabs[i];
      SlabDesc sd{};
      sd.data = cb.data.as<char>() + s.elem_off * ctx->elem_bytes;
      sd.model = cb.model.as<char>() + s.elem_off * ctx->n_dir * ctx->elem_bytes;
      sd.run_ant = cb.run_ant_dev.as<uint32_t>() + s.run_off;
      sd.cb = c;
      sd.T = s.T;
      sd.L = s.L;
      sd.R = s.R;
      sd.sol_off = uint32_t(slab_sol.size());
      slab_sol.insert(slab_sol.end(), s.sol.begin(), s.sol.end());
      const uint32_t gi = uint32_t(descs.size());
      descs.push_back(sd);
      gslabs.push_back({c, i});
      for (uint32_t r = 0; r < s.R; r += runs_per_block) {
        const uint32_t hi = std::min(s.R, r + runs_per_block);
        steps.push_back({gi, r, hi, double(hi - r) * s.T * s.L + 64.0});
      }
    }
  }
  const uint32_t max_ctas = uint32_t(ctx->n_sm) * uint32_t(occ);
  uint32_t n_ctas = std::max<uint32_t>(1, std::min<uint32_t>(max_ctas, uint32_t(steps.size())));
  double total_w = 0;
  for (const Step& s : steps) total_w += s.w;
  // Contiguous step ranges per CTA, balanced by weight.
  std::vector<uint32_t> cta_step_begin(n_ctas + 1, uint32_t(steps.size()));
  {
    double cum = 0;
    uint32_t c = 0;
    cta_step_begin[0] = 0;
    for (uint32_t i = 0; i < steps.size(); ++i) {
      const double mid = cum + 0.5 * steps[i].w;
      while (c + 1 < n_ctas && mid >= total_w * double(c + 1) / n_ctas) {
        ++c;
        cta_step_begin[c] = i;
      }
      cum += steps[i].w;
    }
    for (uint32_t k = c + 1; k <= n_ctas; ++k) cta_step_begin[k] = uint32_t(steps.size());
  }
  std::vector<Visit> visits;
  std::vector<uint32_t> cta_off(n_ctas + 1, 0);
  for (uint32_t c = 0; c < n_ctas; ++c) {
    cta_off[c] = uint32_t(visits.size());
    for (uint32_t i = cta_step_begin[c]; i < cta_step_begin[c + 1]; ++i) {
      const Step& s = steps[i];
      if (!visits.empty() && uint32_t(visits.size()) > cta_off[c] &&
          visits.back().slab == s.slab && visits.back().run_hi == s.run_lo) {
        visits.back().run_hi = s.run_hi;
      } else {
        visits.push_back({s.slab, s.run_lo, s.run_hi, 0});
      }
    }
  }
  cta_off[n_ctas] = uint32_t(visits.size());
  // Drop trailing CTAs without work (keeps the kernel grid dense).
  while (n_ctas > 1 && cta_off[n_ctas - 1] == cta_off[n_ctas]) {
    --n_ctas;
    cta_off.pop_back();
  }
  ctx->n_ctas = n_ctas;
  ctx->n_visits = uint32_t(visits.size());

  // Finalisation lists: for (cb, s), the visits whose slab has cb and uses s.
  std::vector<std::vector<uint32_t>> lists(size_t(ctx->n_cb) * ctx->n_sub);
  for (uint32_t v = 0; v < visits.size(); ++v) {
    const SlabDesc& sd = descs[visits[v].slab];
    for (uint32_t d = 0; d < ctx->n_dir; ++d) {
      const uint32_t s = slab_sol[sd.sol_off + d];
      if (s < ctx->n_sub) lists[size_t(sd.cb) * ctx->n_sub + s].push_back(v);
    }
  }
  std::vector<uint32_t> fin_off(lists.size() + 1, 0), fin_visits;
  for (size_t i = 0; i < lists.size(); ++i) {
    fin_off[i] = uint32_t(fin_visits.size());
    fin_visits.insert(fin_visits.end(), lists[i].begin(), lists[i].end());
  }
  fin_off[lists.size()] = uint32_t(fin_visits.size());

  const uint32_t n_items = ctx->n_cb * ctx->n_ant * ctx->n_sub;
  ctx->fin_blocks = (n_items + kThreads - 1) / kThreads;

  auto upload = [&](DevBuf& b, const void* src, size_t bytes) -> int {
    DDS_CHECK_CUDA(ctx, b.Reserve(bytes));
    if (bytes)
      DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(b.ptr, src, bytes, cudaMemcpyHostToDevice,
                                          ctx->stream));
    return DDSOLVE_OK;
  };
  int rc;
  if ((rc = upload(ctx->d_slabs, descs.data(), descs.size() * sizeof(SlabDesc)))) return rc;
  if ((rc = upload(ctx->d_visits, visits.data(), visits.size() * sizeof(Visit)))) return rc;
  if ((rc = upload(ctx->d_cta_off, cta_off.data(), cta_off.size() * 4))) return rc;
  if ((rc = upload(ctx->d_slab_sol, slab_sol.data(), slab_sol.size() * 4))) return rc;
  if ((rc = upload(ctx->d_fin_off, fin_off.data(), fin_off.size() * 4))) return rc;
  if ((rc = upload(ctx->d_fin_visits, fin_visits.data(), fin_visits.size() * 4))) return rc;
  if ((rc = upload(ctx->d_dir_of_sub, ctx->dir_of_sub.data(), ctx->dir_of_sub.size() * 4)))
    return rc;
  DDS_CHECK_CUDA(ctx, ctx->d_partials.Reserve(size_t(ctx->n_visits) * acc_n * 4));
  DDS_CHECK_CUDA(ctx, ctx->d_block_sum.Reserve(size_t(ctx->fin_blocks) * 8));
  DDS_CHECK_CUDA(ctx, ctx->d_block_cnt.Reserve(size_t(ctx->fin_blocks) * 4));
  // Plan arrays are small host vectors: wait so they can be released.
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->plan_dirty = false;
  ctx->DestroyGraph();
  return DDSOLVE_OK;
}

StreamParams MakeStreamParams(ddsolve_ctx* ctx) {
  StreamParams p;
  p.slabs = ctx->d_slabs.as<SlabDesc>();
  p.visits = ctx->d_visits.as<Visit>();
  p.cta_visit_off = ctx->d_cta_off.as<uint32_t>();
  p.slab_sol = ctx->d_slab_sol.as<uint32_t>();
  p.solutions = ctx->d_sol.as<double2>();
  p.partials = ctx->d_partials.as<float>();
  p.n_ant = ctx->n_ant;
  p.n_dir = ctx->n_dir;
  p.n_sub = ctx->n_sub;
  p.ng = ctx->ng;
  return p;
}

FinParams MakeFinParams(ddsolve_ctx* ctx, bool host_mode) {
  FinParams f;
  f.partials = ctx->d_partials.as<float>();
  f.fin_off = ctx->d_fin_off.as<uint32_t>();
  f.fin_visits = ctx->d_fin_visits.as<uint32_t>();
  f.dir_of_sub = ctx->d_dir_of_sub.as<uint32_t>();
  f.solutions = ctx->d_sol.as<double2>();
  f.next_out = ctx->d_next.as<double2>();
  f.n_cb = ctx->n_cb;
  f.n_ant = ctx->n_ant;
  f.n_dir = ctx->n_dir;
  f.n_sub = ctx->n_sub;
  f.host_mode = host_mode ? 1 : 0;
  f.settings = ctx->d_settings.as<DevSettings>();
  f.block_sum = ctx->d_block_sum.as<double>();
  f.block_cnt = ctx->d_block_cnt.as<uint32_t>();
  f.state = ctx->d_state.as<LoopState>();
  f.nonfinite = ctx->d_nonfinite.as<uint32_t>();
  f.step_magnitudes = ctx->d_mags.as<double>();
  f.handle = ctx->handle;
  f.use_handle = 0;
  return f;
}

// Launches one iteration's kernels on the context stream.
int LaunchIteration(ddsolve_ctx* ctx, bool host_mode, bool use_handle,
                    bool with_make_finite) {
  const uint32_t per_cb = ctx->n_ant * ctx->n_sub * ctx->n_pol;
  if (with_make_finite) {
    if (ctx->n_pol == 2)
      make_finite_kernel<2><<<ctx->n_cb, kThreads, 0, ctx->stream>>>(
          ctx->d_sol.as<double2>(), ctx->d_nonfinite.as<uint32_t>(), per_cb,
          ctx->handle, use_handle ? 1 : 0);
    else
      make_finite_kernel<1><<<ctx->n_cb, kThreads, 0, ctx->stream>>>(
          ctx->d_sol.as<double2>(), ctx->d_nonfinite.as<uint32_t>(), per_cb,
          ctx->handle, use_handle ? 1 : 0);
    DDS_CHECK_CUDA(ctx, cudaGetLastError());
  }
  const StreamParams sp = MakeStreamParams(ctx);
  ctx->stream_fn<<<ctx->n_ctas, kThreads, ctx->stream_smem, ctx->stream>>>(sp);
  DDS_CHECK_CUDA(ctx, cudaGetLastError());
  FinParams fp = MakeFinParams(ctx, host_mode);
  fp.use_handle = use_handle ? 1 : 0;
  if (ctx->n_pol == 2)
    finalize_kernel<2><<<ctx->fin_blocks, kThreads, 0, ctx->stream>>>(fp);
  else
    finalize_kernel<1><<<ctx->fin_blocks, kThreads, 0, ctx->stream>>>(fp);
  DDS_CHECK_CUDA(ctx, cudaGetLastError());
  return DDSOLVE_OK;
}

int BuildGraph(ddsolve_ctx* ctx) {
  ctx->DestroyGraph();
  cudaGraph_t graph = nullptr;
  DDS_CHECK_CUDA(ctx, cudaGraphCreate(&graph, 0));
  ctx->graph = graph;
  DDS_CHECK_CUDA(ctx, cudaGraphConditionalHandleCreate(&ctx->handle, graph, 1,
                                                        cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = ctx->handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  DDS_CHECK_CUDA(ctx, cudaGraphAddNode(&node, graph, nullptr, 0, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  DDS_CHECK_CUDA(ctx, cudaStreamBeginCaptureToGraph(ctx->stream, body, nullptr,
                                                     nullptr, 0,
                                                     cudaStreamCaptureModeThreadLocal));
  const int rc = LaunchIteration(ctx, false, true, true);
  cudaGraph_t captured = nullptr;
  const cudaError_t end = cudaStreamEndCapture(ctx->stream, &captured);
  if (rc != DDSOLVE_OK) return rc;
  DDS_CHECK_CUDA(ctx, end);
  DDS_CHECK_CUDA(ctx, cudaGraphInstantiate(&ctx->graph_exec, graph, 0));
  ctx->graph_ok = true;
  return DDSOLVE_OK;
}

int EnsureSolutionsBuffers(ddsolve_ctx* ctx) {
  const size_t n = size_t(ctx->n_cb) * ctx->n_ant * ctx->n_sub * ctx->n_pol;
  DDS_CHECK_CUDA(ctx, ctx->d_sol.Reserve(n * sizeof(double2)));
  DDS_CHECK_CUDA(ctx, ctx->d_next.Reserve(n * sizeof(double2)));
  return DDSOLVE_OK;
}

int UploadSettings(ddsolve_ctx* ctx) {
  DevSettings ds{};
  ds.max_iterations = ctx->settings.max_iterations;
  ds.min_iterations = ctx->settings.min_iterations;
  ds.accuracy = ctx->settings.accuracy;
  ds.constraint_accuracy = ctx->settings.constraint_accuracy;
  ds.step_size = ctx->settings.step_size;
  ds.detect_stalling = ctx->settings.detect_stalling;
  ds.phase_only = ctx->settings.phase_only;
  ds.step_diff_sigma = ctx->settings.step_diff_sigma;
  ds.hard_cap = std::max(std::max(ctx->settings.max_iterations,
                                  ctx->settings.min_iterations), 1u);
  DDS_CHECK_CUDA(ctx, ctx->d_settings.Reserve(sizeof(DevSettings)));
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->d_settings.ptr, &ds, sizeof(ds),
                                      cudaMemcpyHostToDevice, ctx->stream));
  DDS_CHECK_CUDA(ctx, ctx->d_mags.Reserve(size_t(ds.hard_cap) * 8));
  // keep `ds` alive until the copy has been issued from pageable memory
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return DDSOLVE_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

void ddsolve_default_settings(ddsolve_settings* s) {
  if (!s) return;
  // SolverBase::SolverBase (ddecal/gain_solvers/SolverBase.cc:27-39)
  s->max_iterations = 100;
  s->min_iterations = 0;
  s->accuracy = 1.0e-5;
  s->constraint_accuracy = 1.0e-4;
  s->step_size = 0.2;
  s->detect_stalling = 1;
  s->step_diff_sigma = 0.1;
  s->phase_only = 0;
}

int ddsolve_create(const ddsolve_dims* dims, int device, ddsolve_ctx** out) {
  if (!out) {
    g_last_error = "ddsolve_create: out is NULL";
    return DDSOLVE_E_INVALID;
  }
  *out = nullptr;
  const int dc = CheckDims(dims);
  if (dc != DDSOLVE_OK) {
    g_last_error = "ddsolve_create: invalid or unsupported dimensions";
    return dc;
  }
  int n_dev = 0;
  cudaError_t e = cudaGetDeviceCount(&n_dev);
  if (e != cudaSuccess || device < 0 || device >= n_dev) {
    g_last_error = std::string("ddsolve_create: no CUDA device: ") +
                   (e == cudaSuccess ? "bad ordinal" : cudaGetErrorString(e));
    return DDSOLVE_E_CUDA;
  }
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess || prop.major < 10) {
    g_last_error = "ddsolve_create: device is not sm_100 class";
    return DDSOLVE_E_CUDA;
  }
  e = cudaSetDevice(device);
  if (e != cudaSuccess) {
    g_last_error = std::string("ddsolve_create: ") + cudaGetErrorString(e);
    return DDSOLVE_E_CUDA;
  }
  std::unique_ptr<ddsolve_ctx> ctx(new ddsolve_ctx());
  ctx->device = device;
  ctx->n_sm = prop.multiProcessorCount;
  ctx->n_ant = dims->n_antennas;
  ctx->n_dir = dims->n_directions;
  ctx->n_cb = dims->n_channel_blocks;
  ctx->n_corr = dims->n_correlations;
  ctx->n_pol = dims->n_solution_polarizations;
  ctx->n_sol_per_dir.assign(dims->n_solutions_per_direction,
                            dims->n_solutions_per_direction + ctx->n_dir);
  ctx->sol_start.resize(ctx->n_dir);
  uint32_t acc = 0;
  for (uint32_t d = 0; d < ctx->n_dir; ++d) {
    ctx->sol_start[d] = acc;
    for (uint32_t k = 0; k < ctx->n_sol_per_dir[d]; ++k) ctx->dir_of_sub.push_back(d);
    acc += ctx->n_sol_per_dir[d];
  }
  ctx->n_sub = acc;
  ctx->elem_bytes = ElemBytes(ctx->n_corr);
  ctx->cbs.resize(ctx->n_cb);
  ddsolve_default_settings(&ctx->settings);
  e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    g_last_error = std::string("ddsolve_create: ") + cudaGetErrorString(e);
    return DDSOLVE_E_CUDA;
  }
  const int rc = EnsureSolutionsBuffers(ctx.get());
  if (rc != DDSOLVE_OK) {
    g_last_error = ctx->err;
    return rc;
  }
  if (ctx->d_state.Reserve(sizeof(LoopState)) != cudaSuccess ||
      ctx->d_nonfinite.Reserve(size_t(ctx->n_cb) * 4) != cudaSuccess) {
    g_last_error = "ddsolve_create: out of device memory";
    return DDSOLVE_E_CUDA;
  }
  if (UploadSettings(ctx.get()) != DDSOLVE_OK) {
    g_last_error = ctx->err;
    return DDSOLVE_E_CUDA;
  }
  *out = ctx.release();
  return DDSOLVE_OK;
}

int ddsolve_destroy(ddsolve_ctx* ctx) {
  if (!ctx) return DDSOLVE_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  delete ctx;
  return DDSOLVE_OK;
}

const char* ddsolve_last_error(const ddsolve_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_last_error.c_str();
}

int ddsolve_set_settings(ddsolve_ctx* ctx, const ddsolve_settings* s) {
  if (!ctx || !s) return DDSOLVE_E_INVALID;
  if (!(s->step_size > 0.0) || !std::isfinite(s->accuracy))
    return ctx->Fail(DDSOLVE_E_INVALID, "invalid settings");
  cudaSetDevice(ctx->device);
  ctx->settings = *s;
  return UploadSettings(ctx);
}

int ddsolve_set_tuning(ddsolve_ctx* ctx, uint32_t direction_groups,
                       uint32_t max_slab_times) {
  if (!ctx) return DDSOLVE_E_INVALID;
  if (direction_groups != 0 &&
      (direction_groups > 32 || (direction_groups & (direction_groups - 1))))
    return ctx->Fail(DDSOLVE_E_INVALID, "direction_groups must be 0 or a power of 2 <= 32");
  ctx->tune_ng = direction_groups;
  ctx->tune_max_times = max_slab_times;
  ctx->plan_dirty = true;
  return DDSOLVE_OK;
}

void* ddsolve_stream(ddsolve_ctx* ctx) { return ctx ? ctx->stream : nullptr; }

uint64_t ddsolve_last_launch_count(const ddsolve_ctx* ctx) {
  return ctx ? ctx->last_launches : 0;
}

int ddsolve_set_channel_block_regular(ddsolve_ctx* ctx, uint32_t cbi,
                                      uint32_t n_times, uint32_t n_baselines,
                                      uint32_t n_channels, const float* data,
                                      const float* model,
                                      const uint32_t* antenna1,
                                      const uint32_t* antenna2) {
  if (!ctx) return DDSOLVE_E_INVALID;
  if (cbi >= ctx->n_cb) return ctx->Fail(DDSOLVE_E_INVALID, "channel block out of range");
  if (n_times == 0 || n_baselines == 0 || n_channels == 0 || !data || !model ||
      !antenna1 || !antenna2)
    return ctx->Fail(DDSOLVE_E_INVALID, "empty channel block or NULL pointer");
  for (uint32_t b = 0; b < n_baselines; ++b)
    if (antenna1[b] >= ctx->n_ant || antenna2[b] >= ctx->n_ant ||
        antenna1[b] == antenna2[b])
      return ctx->Fail(DDSOLVE_E_INVALID, "bad antenna pair (or autocorrelation)");
  cudaSetDevice(ctx->device);
  ChannelBlockStore& cb = ctx->cbs[cbi];
  cb.n_vis = uint64_t(n_times) * n_baselines * n_channels;
  cb.slabs.clear();
  cb.run_ant.resize(n_baselines);
  cb.run_src.resize(n_baselines);
  cb.run_len.assign(n_baselines, n_channels);
  for (uint32_t b = 0; b < n_baselines; ++b) {
    cb.run_ant[b] = antenna1[b] | (antenna2[b] << 16);
    cb.run_src[b] = b * n_channels;
  }
  // Solution index per (direction, time), SolveData.cc:102-105,124-125,167.
  std::vector<uint32_t> nsol(ctx->n_dir), start(ctx->n_dir);
  uint32_t acc = 0;
  for (uint32_t d = 0; d < ctx->n_dir; ++d) {
    nsol[d] = std::min(ctx->n_sol_per_dir[d], n_times);
    start[d] = acc;
    acc += nsol[d];
  }
  auto sol_of = [&](uint32_t d, uint32_t t) {
    return uint32_t(uint64_t(t) * nsol[d] / n_times) + start[d];
  };
  const uint32_t max_t = ctx->tune_max_times ? ctx->tune_max_times : n_times;
  uint64_t off = 0;
  uint32_t t0 = 0;
  while (t0 < n_times) {
    uint32_t t1 = t0 + 1;
    while (t1 < n_times && t1 - t0 < max_t) {
      bool same = true;
      for (uint32_t d = 0; d < ctx->n_dir && same; ++d)
        same = sol_of(d, t1) == sol_of(d, t0);
      if (!same) break;
      ++t1;
    }
    HostSlab s;
    s.T = t1 - t0;
    s.L = n_channels;
    s.R = n_baselines;
    s.elem_off = off;
    s.src_base = uint64_t(t0) * n_baselines * n_channels;
    s.tstride = uint64_t(n_baselines) * n_channels;
    s.run_off = 0;
    s.sol.resize(ctx->n_dir);
    for (uint32_t d = 0; d < ctx->n_dir; ++d) s.sol[d] = sol_of(d, t0);
    off += uint64_t(s.T) * s.L * s.R;
    cb.slabs.push_back(std::move(s));
    t0 = t1;
  }
  cb.n_elems = off;
  return UploadAndPack(ctx, cb, data, model);
}

int ddsolve_set_channel_block(ddsolve_ctx* ctx, uint32_t cbi, uint64_t n_vis,
                              const float* data, const float* model,
                              const uint32_t* antenna_pairs,
                              const uint32_t* solution_map) {
  if (!ctx) return DDSOLVE_E_INVALID;
  if (cbi >= ctx->n_cb) return ctx->Fail(DDSOLVE_E_INVALID, "channel block out of range");
  if (n_vis > 0 && (!data || !model || !antenna_pairs || !solution_map))
    return ctx->Fail(DDSOLVE_E_INVALID, "NULL pointer");
  if (n_vis >= (uint64_t(1) << 32))
    return ctx->Fail(DDSOLVE_E_UNSUPPORTED, "more than 2^32 visibilities in a channel block");
  cudaSetDevice(ctx->device);
  ChannelBlockStore& cb = ctx->cbs[cbi];
  cb.n_vis = n_vis;
  cb.slabs.clear();
  // Runs: consecutive visibilities with equal antennas and solution indices.
  struct Run {
    uint32_t start, len, ant;
  };
  std::vector<Run> runs;
  for (uint64_t v = 0; v < n_vis;) {
    const uint32_t a1 = antenna_pairs[2 * v], a2 = antenna_pairs[2 * v + 1];
    if (a1 >= ctx->n_ant || a2 >= ctx->n_ant)
      return ctx->Fail(DDSOLVE_E_INVALID, "antenna index out of range");
    for (uint32_t d = 0; d < ctx->n_dir; ++d)
      if (solution_map[size_t(d) * n_vis + v] >= ctx->n_sub)
        return ctx->Fail(DDSOLVE_E_INVALID, "solution index out of range");
    uint64_t w = v + 1;
    while (w < n_vis && antenna_pairs[2 * w] == a1 && antenna_pairs[2 * w + 1] == a2) {
      bool same = true;
      for (uint32_t d = 0; d < ctx->n_dir && same; ++d)
        same = solution_map[size_t(d) * n_vis + w] == solution_map[size_t(d) * n_vis + v];
      if (!same) break;
      ++w;
    }
    runs.push_back({uint32_t(v), uint32_t(w - v), a1 | (a2 << 16)});
    v = w;
  }
  // Group runs into slabs by (length, solution indices). Runs of one slab are
  // ordered by antenna 1 so that the warp-level segmented reduction finds
  // long segments; the sum does not depend on the order.
  std::map<std::vector<uint32_t>, std::vector<uint32_t>> groups;
  for (uint32_t i = 0; i < runs.size(); ++i) {
    std::vector<uint32_t> key(ctx->n_dir + 1);
    key[0] = runs[i].len;
    for (uint32_t d = 0; d < ctx->n_dir; ++d)
      key[d + 1] = solution_map[size_t(d) * n_vis + runs[i].start];
    groups[key].push_back(i);
  }
  cb.run_ant.clear();
  cb.run_src.clear();
  cb.run_len.clear();
  uint64_t off = 0;
  for (auto& kv : groups) {
    std::vector<uint32_t>& members = kv.second;
    std::stable_sort(members.begin(), members.end(), [&](uint32_t x, uint32_t y) {
      return (runs[x].ant & 0xFFFFu) < (runs[y].ant & 0xFFFFu);
    });
    HostSlab s;
    s.T = 1;
    s.L = kv.first[0];
    s.R = uint32_t(members.size());
    s.elem_off = off;
    s.src_base = 0;
    s.tstride = 0;
    s.run_off = uint32_t(cb.run_ant.size());
    s.sol.assign(kv.first.begin() + 1, kv.first.end());
    for (uint32_t m : members) {
      cb.run_ant.push_back(runs[m].ant);
      cb.run_src.push_back(runs[m].start);
      cb.run_len.push_back(runs[m].len);
    }
    off += uint64_t(s.L) * s.R;
    cb.slabs.push_back(std::move(s));
  }
  cb.n_elems = off;
  if (cb.run_ant.empty()) {
    cb.run_ant.push_back(0);
    cb.run_src.push_back(0);
    cb.run_len.push_back(0);
  }
  return UploadAndPack(ctx, cb, data, model);
}

int ddsolve_solve(ddsolve_ctx* ctx, double* solutions, ddsolve_result* result,
                  double* step_magnitudes) {
  if (!ctx || !solutions) return DDSOLVE_E_INVALID;
  cudaSetDevice(ctx->device);
  int rc;
  if (ctx->plan_dirty && (rc = BuildPlan(ctx)) != DDSOLVE_OK) return rc;
  const size_t n_sol = size_t(ctx->n_cb) * ctx->n_ant * ctx->n_sub * ctx->n_pol;
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->d_sol.ptr, solutions, n_sol * sizeof(double2),
                                      cudaMemcpyHostToDevice, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_state.ptr, 0, sizeof(LoopState), ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_nonfinite.ptr, 1, size_t(ctx->n_cb) * 4,
                                      ctx->stream));
  if (!ctx->graph_ok) {
    rc = BuildGraph(ctx);
    if (rc != DDSOLVE_OK) {
      // Conditional graphs unavailable: fall back to host-driven launches.
      ctx->DestroyGraph();
      cudaGetLastError();
    }
  }
  LoopState ls{};
  if (ctx->graph_ok) {
    DDS_CHECK_CUDA(ctx, cudaGraphLaunch(ctx->graph_exec, ctx->stream));
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(&ls, ctx->d_state.ptr, sizeof(ls),
                                        cudaMemcpyDeviceToHost, ctx->stream));
  } else {
    const uint32_t cap = std::max(std::max(ctx->settings.max_iterations,
                                           ctx->settings.min_iterations), 1u);
    for (uint32_t it = 0; it < cap; ++it) {
      if ((rc = LaunchIteration(ctx, false, false, true)) != DDSOLVE_OK) return rc;
      DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(&ls, ctx->d_state.ptr, sizeof(ls),
                                          cudaMemcpyDeviceToHost, ctx->stream));
      DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      if (ls.done) break;
    }
  }
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(solutions, ctx->d_sol.ptr, n_sol * sizeof(double2),
                                      cudaMemcpyDeviceToHost, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (step_magnitudes && ls.iteration > 0) {
    DDS_CHECK_CUDA(ctx, cudaMemcpy(step_magnitudes, ctx->d_mags.ptr,
                                   size_t(ls.iteration) * 8, cudaMemcpyDeviceToHost));
  }
  ctx->last_launches = uint64_t(ls.iteration) * 3;
  if (result) {
    // SolverBase::MakeResult (SolverBase.cc:192-213), constraints satisfied.
    result->iterations = ls.has_converged ? ls.iteration : ls.iteration + 1;
    result->constraint_iterations = 0;
    result->has_converged = ls.has_converged;
    result->has_stalled = ls.has_stalled;
  }
  return DDSOLVE_OK;
}

int ddsolve_perform_iteration(ddsolve_ctx* ctx, const double* solutions,
                              double* next_solutions) {
  if (!ctx || !solutions || !next_solutions) return DDSOLVE_E_INVALID;
  cudaSetDevice(ctx->device);
  int rc;
  if (ctx->plan_dirty && (rc = BuildPlan(ctx)) != DDSOLVE_OK) return rc;
  const size_t n_sol = size_t(ctx->n_cb) * ctx->n_ant * ctx->n_sub * ctx->n_pol;
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->d_sol.ptr, solutions, n_sol * sizeof(double2),
                                      cudaMemcpyHostToDevice, ctx->stream));
  if ((rc = LaunchIteration(ctx, true, false, false)) != DDSOLVE_OK) return rc;
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(next_solutions, ctx->d_next.ptr,
                                      n_sol * sizeof(double2), cudaMemcpyDeviceToHost,
                                      ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->last_launches = 2;
  return DDSOLVE_OK;
}

int ddsolve_time_stream_kernel(ddsolve_ctx* ctx, uint32_t n_launches, float* mean_ms) {
  if (!ctx || !mean_ms || n_launches == 0) return DDSOLVE_E_INVALID;
  cudaSetDevice(ctx->device);
  int rc;
  if (ctx->plan_dirty && (rc = BuildPlan(ctx)) != DDSOLVE_OK) return rc;
  cudaEvent_t a, b;
  DDS_CHECK_CUDA(ctx, cudaEventCreate(&a));
  DDS_CHECK_CUDA(ctx, cudaEventCreate(&b));
  const StreamParams sp = MakeStreamParams(ctx);
  // warm-up launch
  ctx->stream_fn<<<ctx->n_ctas, kThreads, ctx->stream_smem, ctx->stream>>>(sp);
  DDS_CHECK_CUDA(ctx, cudaEventRecord(a, ctx->stream));
  for (uint32_t i = 0; i < n_launches; ++i)
    ctx->stream_fn<<<ctx->n_ctas, kThreads, ctx->stream_smem, ctx->stream>>>(sp);
  DDS_CHECK_CUDA(ctx, cudaEventRecord(b, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaEventSynchronize(b));
  float ms = 0;
  DDS_CHECK_CUDA(ctx, cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *mean_ms = ms / float(n_launches);
  return DDSOLVE_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free entry point: one direction-iterative pass over regular
// data that the caller already holds in device memory, with the per-antenna
// accumulators in a fixed-size array that lives in the library's own device
// image. Some callers cannot let a library allocate device memory: code that
// runs while a CUDA graph is being captured (cudaMalloc is not allowed
// during capture), frameworks that hand all device memory out of their own
// pool or arena, and hosts whose device memory is already fully budgeted.
// This variant only uses that static array; it never calls cudaMalloc,
// cudaFree or an allocating library routine.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocScratchFloats = size_t(1) << 20;  // 4 MiB
constexpr uint32_t kNoAllocMaxChannelBlocks = 256;
constexpr uint32_t kNoAllocMaxDirections = 64;
constexpr uint32_t kNoAllocMaxChannels = 16;  // channels per block
constexpr int kNoAllocThreads = 128;

// Per-antenna accumulators [cb][ant][sub][pol][num.re, num.im, den]. Every
// GPU that loads this library holds these 4 MiB until the process exits.
static __device__ __align__(256) float g_noalloc_scratch[kNoAllocScratchFloats];

struct NoAllocParams {
  const float* data;
  const float* model;
  const uint32_t* antenna1;
  const uint32_t* antenna2;
  const double2* solutions;
  double2* next;
  float* acc;
  uint32_t n_ant, n_dir, n_sub, n_cb, n_times, n_bl;
  uint32_t cb_channels[kNoAllocMaxChannelBlocks];
  uint64_t cb_vis_offset[kNoAllocMaxChannelBlocks];  // first visibility of cb
  uint32_t n_sol[kNoAllocMaxDirections];             // min(n_sol, n_times)
  uint32_t sol_start[kNoAllocMaxDirections];
};

// One thread per (channel block, time step, baseline): residual over the
// block's channels, then per direction P = sum R conj(M), Q = sum |M|^2 and
// the antenna contributions added atomically into the scratch accumulators.
template <int NCORR, int NPOL>
__global__ void __launch_bounds__(kNoAllocThreads)
    noalloc_accumulate_kernel(const NoAllocParams p) {
  const uint32_t bl = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t t = blockIdx.y;
  const uint32_t cb = blockIdx.z;
  if (bl >= p.n_bl) return;
  const uint32_t a1 = p.antenna1[bl];
  const uint32_t a2 = p.antenna2[bl];
  if (a1 >= p.n_ant || a2 >= p.n_ant) return;  // invalid pairs are ignored
  const uint32_t L = p.cb_channels[cb];
  const uint64_t n_vis_cb = uint64_t(p.n_times) * p.n_bl * L;
  const uint64_t v0 = (uint64_t(t) * p.n_bl + bl) * L;
  const float* data = p.data + p.cb_vis_offset[cb] * NCORR * 2;
  const float* model = p.model + p.cb_vis_offset[cb] * p.n_dir * NCORR * 2;

  float2 R[kNoAllocMaxChannels][NCORR];
#pragma unroll
  for (uint32_t ch = 0; ch < kNoAllocMaxChannels; ++ch)
    if (ch < L) LoadVis<NCORR>(data, v0 + ch, R[ch]);

  auto gain = [&](uint32_t ant, uint32_t s, int q) {
    const double2 g = p.solutions[(size_t(cb * p.n_ant + ant) * p.n_sub + s) * NPOL + q];
    return make_float2(float(g.x), float(g.y));
  };
  auto sol_of = [&](uint32_t d) {
    return uint32_t(uint64_t(t) * p.n_sol[d] / p.n_times) + p.sol_start[d];
  };
  // Residual: R = D - sum_d G_d M_d
  for (uint32_t d = 0; d < p.n_dir; ++d) {
    const uint32_t s = sol_of(d);
    float2 ga[NPOL], gb[NPOL];
#pragma unroll
    for (int q = 0; q < NPOL; ++q) {
      ga[q] = gain(a1, s, q);
      gb[q] = gain(a2, s, q);
    }
#pragma unroll
    for (uint32_t ch = 0; ch < kNoAllocMaxChannels; ++ch) {
      if (ch >= L) break;
      float2 M[NCORR];
      LoadVis<NCORR>(model, d * n_vis_cb + v0 + ch, M);
#pragma unroll
      for (int c = 0; c < NCORR; ++c) {
        const float2 G = cmul_conj(ga[RowPol<NCORR, NPOL>(c)], gb[ColPol<NCORR, NPOL>(c)]);
        const float2 gm = cmul(G, M[c]);
        R[ch][c].x -= gm.x;
        R[ch][c].y -= gm.y;
      }
    }
  }
  // Normal equations of every direction.
  for (uint32_t d = 0; d < p.n_dir; ++d) {
    const uint32_t s = sol_of(d);
    float2 P[NCORR];
    float Q[NCORR];
#pragma unroll
    for (int c = 0; c < NCORR; ++c) {
      P[c] = make_float2(0.f, 0.f);
      Q[c] = 0.f;
    }
#pragma unroll
    for (uint32_t ch = 0; ch < kNoAllocMaxChannels; ++ch) {
      if (ch >= L) break;
      float2 M[NCORR];
      LoadVis<NCORR>(model, d * n_vis_cb + v0 + ch, M);
#pragma unroll
      for (int c = 0; c < NCORR; ++c) {
        const float2 rm = cmul_conj(R[ch][c], M[c]);
        P[c].x += rm.x;
        P[c].y += rm.y;
        Q[c] += cnorm(M[c]);
      }
    }
    float2 ga[NPOL], gb[NPOL];
#pragma unroll
    for (int q = 0; q < NPOL; ++q) {
      ga[q] = gain(a1, s, q);
      gb[q] = gain(a2, s, q);
    }
#pragma unroll
    for (int q = 0; q < NPOL; ++q) {
      float2 n1 = make_float2(0.f, 0.f), n2 = make_float2(0.f, 0.f);
      float d1 = 0.f, d2 = 0.f;
#pragma unroll
      for (int c = 0; c < NCORR; ++c) {
        const int rp = RowPol<NCORR, NPOL>(c);
        const int cp = ColPol<NCORR, NPOL>(c);
        if (rp == q) {
          const float2 t1 = cmul(gb[cp], P[c]);
          n1.x += t1.x;
          n1.y += t1.y;
          d1 += cnorm(gb[cp]) * Q[c];
        }
        if (cp == q) {
          const float2 t2 = cmul(ga[rp], cconj(P[c]));
          n2.x += t2.x;
          n2.y += t2.y;
          d2 += cnorm(ga[rp]) * Q[c];
        }
      }
      float* acc1 = p.acc + ((size_t(cb * p.n_ant + a1) * p.n_sub + s) * NPOL + q) * 3;
      float* acc2 = p.acc + ((size_t(cb * p.n_ant + a2) * p.n_sub + s) * NPOL + q) * 3;
      atomicAdd(acc1 + 0, n1.x);
      atomicAdd(acc1 + 1, n1.y);
      atomicAdd(acc1 + 2, d1);
      atomicAdd(acc2 + 0, n2.x);
      atomicAdd(acc2 + 1, n2.y);
      atomicAdd(acc2 + 2, d2);
    }
  }
}

// next = g_a + num / den per (cb, ant, sub, pol); NaN where den == 0.
template <int NPOL>
__global__ void __launch_bounds__(kThreads)
    noalloc_finalize_kernel(const float* __restrict__ acc,
                            const double2* __restrict__ solutions,
                            double2* __restrict__ next, uint32_t n_items) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_items) return;
#pragma unroll
  for (int q = 0; q < NPOL; ++q) {
    const size_t e = size_t(i) * NPOL + q;
    const float den = acc[e * 3 + 2];
    if (den == 0.f) {
      next[e] = make_double2(nan(""), 0.0);
    } else {
      const double2 g = solutions[e];
      next[e] = make_double2(double(float(g.x)) + double(acc[e * 3]) / double(den),
                             double(float(g.y)) + double(acc[e * 3 + 1]) / double(den));
    }
  }
}

// Device address of g_noalloc_scratch, looked up once per device (with that
// device current) and cached.
int NoAllocScratchAddress(int device, float** out) {
  static std::mutex mu;
  static std::map<int, float*> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(device);
  if (it != cache.end()) {
    *out = it->second;
    return DDSOLVE_OK;
  }
  float* ptr = nullptr;
  const cudaError_t e =
      cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_noalloc_scratch);
  if (e != cudaSuccess || !ptr) {
    g_last_error = std::string("ddsolve_perform_iteration_noalloc: "
                               "cudaGetSymbolAddress failed: ") +
                   cudaGetErrorString(e);
    return DDSOLVE_E_CUDA;
  }
  cache[device] = ptr;
  *out = ptr;
  return DDSOLVE_OK;
}

template <int NCORR, int NPOL>
void LaunchNoAlloc(const NoAllocParams& p, uint32_t n_items, cudaStream_t s) {
  const dim3 grid((p.n_bl + kNoAllocThreads - 1) / kNoAllocThreads, p.n_times, p.n_cb);
  noalloc_accumulate_kernel<NCORR, NPOL><<<grid, kNoAllocThreads, 0, s>>>(p);
  noalloc_finalize_kernel<NPOL><<<(n_items + kThreads - 1) / kThreads, kThreads, 0, s>>>(
      p.acc, p.solutions, p.next, n_items);
}

}  // namespace

extern "C" int ddsolve_perform_iteration_noalloc(
    const ddsolve_dims* dims, uint32_t n_times, uint32_t n_baselines,
    const uint32_t* cb_channels, const float* data, const float* model,
    const uint32_t* antenna1, const uint32_t* antenna2, const double* solutions,
    double* next_solutions, void* stream) {
  const char* who = "ddsolve_perform_iteration_noalloc: ";
  const int dc = CheckDims(dims);
  if (dc != DDSOLVE_OK) {
    g_last_error = std::string(who) + "invalid or unsupported dimensions";
    return dc;
  }
  if (!cb_channels || !data || !model || !antenna1 || !antenna2 || !solutions ||
      !next_solutions || n_times == 0 || n_baselines == 0) {
    g_last_error = std::string(who) + "NULL pointer or empty interval";
    return DDSOLVE_E_INVALID;
  }
  const uint32_t n_cb = dims->n_channel_blocks, n_dir = dims->n_directions;
  const uint32_t n_ant = dims->n_antennas, n_pol = dims->n_solution_polarizations;
  uint32_t n_sub = 0;
  for (uint32_t d = 0; d < n_dir; ++d) n_sub += dims->n_solutions_per_direction[d];
  if (n_cb > kNoAllocMaxChannelBlocks || n_dir > kNoAllocMaxDirections) {
    g_last_error = std::string(who) + "more than 256 channel blocks or 64 directions";
    return DDSOLVE_E_UNSUPPORTED;
  }
  const uint64_t acc_floats = uint64_t(n_cb) * n_ant * n_sub * n_pol * 3;
  if (acc_floats > kNoAllocScratchFloats) {
    g_last_error = std::string(who) + "channel blocks x antennas x sub-solutions x "
                   "polarizations x 3 = " + std::to_string(acc_floats) +
                   " exceeds the static scratch of " +
                   std::to_string(kNoAllocScratchFloats) + " floats";
    return DDSOLVE_E_UNSUPPORTED;
  }
  NoAllocParams p;
  p.data = data;
  p.model = model;
  p.antenna1 = antenna1;
  p.antenna2 = antenna2;
  p.solutions = reinterpret_cast<const double2*>(solutions);
  p.next = reinterpret_cast<double2*>(next_solutions);
  p.n_ant = n_ant;
  p.n_dir = n_dir;
  p.n_sub = n_sub;
  p.n_cb = n_cb;
  p.n_times = n_times;
  p.n_bl = n_baselines;
  uint64_t off = 0;
  for (uint32_t c = 0; c < n_cb; ++c) {
    if (cb_channels[c] == 0 || cb_channels[c] > kNoAllocMaxChannels) {
      g_last_error = std::string(who) + "channels per block must be 1..16";
      return DDSOLVE_E_UNSUPPORTED;
    }
    p.cb_channels[c] = cb_channels[c];
    p.cb_vis_offset[c] = off;
    off += uint64_t(n_times) * n_baselines * cb_channels[c];
  }
  uint32_t start = 0;
  for (uint32_t d = 0; d < n_dir; ++d) {
    p.n_sol[d] = std::min(dims->n_solutions_per_direction[d], n_times);
    p.sol_start[d] = start;
    start += p.n_sol[d];
  }
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) {
    g_last_error = std::string(who) + cudaGetErrorString(e);
    return DDSOLVE_E_CUDA;
  }
  float* scratch = nullptr;
  const int rc = NoAllocScratchAddress(device, &scratch);
  if (rc != DDSOLVE_OK) return rc;
  p.acc = scratch;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  e = cudaMemsetAsync(scratch, 0, acc_floats * sizeof(float), s);
  if (e != cudaSuccess) {
    g_last_error = std::string(who) + cudaGetErrorString(e);
    return DDSOLVE_E_CUDA;
  }
  const uint32_t n_items = n_cb * n_ant * n_sub;
  const uint32_t nc = dims->n_correlations;
  if (nc == 2 && n_pol == 2) LaunchNoAlloc<2, 2>(p, n_items, s);
  else if (nc == 4 && n_pol == 2) LaunchNoAlloc<4, 2>(p, n_items, s);
  else if (nc == 1 && n_pol == 1) LaunchNoAlloc<1, 1>(p, n_items, s);
  else if (nc == 2 && n_pol == 1) LaunchNoAlloc<2, 1>(p, n_items, s);
  else LaunchNoAlloc<4, 1>(p, n_items, s);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    g_last_error = std::string(who) + cudaGetErrorString(e);
    return DDSOLVE_E_CUDA;
  }
  return DDSOLVE_OK;
}
