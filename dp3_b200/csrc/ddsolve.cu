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
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <type_traits>
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
// A slab's visibilities, packed tile by tile: for every (time, channel) row,
// its runs are cut into tiles of W runs (the last one shorter), and a tile
// holds the data and then every direction's model for its runs,
//   [T][L][tile][1 + n_dir][runs of the tile],
// so that one row of one tile, with all its directions, is one contiguous
// block (one bulk copy of the pipelined kernel).
struct SlabDesc {
  const void* vis;          // data and model, packed as above
  const uint32_t* run_ant;  // [R] antenna1 | antenna2 << 16
  uint32_t cb, T, L, R;
  uint32_t W;        // runs per tile (a multiple of 4)
  uint32_t sol_off;  // first of n_dir entries in slab_sol
  uint32_t table;    // gain table of the slab (pipe_kernel)
};

// Element index in a packed slab of run r, row (t * L + l), and j = 0 for the
// data or 1 + d for direction d's model; nd1 = 1 + n_dir.
__host__ __device__ __forceinline__ uint64_t SlabElem(uint32_t R, uint32_t W, uint32_t nd1,
                                                      uint64_t row, uint32_t j, uint32_t r) {
  const uint32_t k = r / W;
  const uint32_t base = k * W;
  const uint32_t w = R - base < W ? R - base : W;
  return row * R * nd1 + uint64_t(base) * nd1 + uint64_t(j) * w + (r - base);
}

// pipe_kernel work item: rows [row_lo, row_hi) of the (t, channel) rows of
// the tile of runs [r0, r0 + n_runs) of a slab; fragments of one CTA that
// share a slab form a visit (one partial slot).
struct Frag {
  uint32_t slab, r0, n_runs, flags, row_lo, row_hi, visit, tile;
  uint32_t group_end[2];  // direct reduction: end run (exclusive) of groups
                          // 0..7, one byte each; groups partition [0, n_runs)
};
constexpr uint32_t kFragDirect = 1u;  // runs split into <= 8 groups, each with
                                      // distinct first and second antennas
constexpr uint32_t kMaxGroups = 8;
constexpr uint32_t kFragPower = 2u;   // the fragment adds its tile's precomputed
                                      // model powers sum |M|^2 (one per tile)

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

// Finalisation modes of a solve iteration. Fused: merge, FP64 division,
// SolverBase::Step, AssignSolutions and the iteration control in one pass.
// With device constraints the iteration is split around them
// (IterativeDiagonalSolver.cc:77-83: Step, ApplyConstraints, AssignSolutions):
// StepOnly writes the stepped next solutions to next_out and stops there;
// AssignOnly reads the constrained next solutions from next_out and does the
// rest (norm, solutions, gain tables, non-finite flags, control).
constexpr int32_t kFinFused = 0;
constexpr int32_t kFinStepOnly = 1;
constexpr int32_t kFinAssignOnly = 2;

struct FinParams {
  const float* partials;
  const uint32_t* fin_off;     // [n_cb * n_sub + 1]
  const uint32_t* fin_visits;  // visit indices
  const uint32_t* dir_of_sub;  // [n_sub]
  double2* solutions;          // [n_cb][n_ant][n_sub][NPOL]
  double2* next_out;           // host mode output; the constrained passes' buffer
  uint32_t n_cb, n_ant, n_dir, n_sub;
  int32_t host_mode;
  int32_t fin_mode;            // FinFused / FinStepOnly / FinAssignOnly
  const DevSettings* settings;
  double* block_sum;
  uint32_t* block_cnt;
  LoopState* state;
  uint32_t* nonfinite;  // [n_cb]
  double* step_magnitudes;
  cudaGraphConditionalHandle handle;
  int32_t use_handle;
  // independent solution intervals (groups of channel blocks): finalisation
  // block b covers items [block_item0[b], block_item_end[b]) of interval
  // block_group[b]; interval g owns blocks [group_blocks[g], group_blocks[g+1])
  // and its loop state state[g] and step magnitudes step_magnitudes[g * mags_stride]
  const uint32_t* block_group;
  const uint32_t* block_item0;
  const uint32_t* block_item_end;
  const uint32_t* group_blocks;
  uint32_t n_groups;
  uint32_t mags_stride;
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
//   src_base + t * tstride + run_src[r] + ch   (zero if ch >= run length)
// A run whose length carries kRunFlipped stores the baseline with its
// antennas swapped: visibility and model are Hermitian-transposed
// (conjugated, with XY and YX exchanged for full 2x2 data), which leaves the
// solver's normal equations unchanged (the contribution of antenna 1 of the
// flipped run is that of antenna 2 of the original one, and vice versa).
// ---------------------------------------------------------------------------
constexpr uint32_t kRunFlipped = 0x80000000u;

struct PackSlab {
  uint64_t dst_elem_off;  // into the cb's packed buffer, in units of 1 + n_dir elements
  uint64_t src_base;
  uint64_t tstride;
  uint32_t T, L, R, run_off, W;
};

template <int NCORR>
__device__ __forceinline__ void CopyVis(const float2* __restrict__ src, float2* __restrict__ dst,
                                        bool valid, bool flip) {
  float2 v[NCORR];
#pragma unroll
  for (int c = 0; c < NCORR; ++c) v[c] = valid ? src[c] : make_float2(0.f, 0.f);
  if (flip) {
#pragma unroll
    for (int c = 0; c < NCORR; ++c) v[c].y = -v[c].y;
    if constexpr (NCORR == 4) {
      const float2 t = v[1];
      v[1] = v[2];
      v[2] = t;
    }
  }
#pragma unroll
  for (int c = 0; c < NCORR; ++c) dst[c] = v[c];
}

template <int NCORR>
__global__ void pack_kernel(const PackSlab s, const uint32_t* __restrict__ run_src,
                            const uint32_t* __restrict__ run_len,
                            const float2* __restrict__ src_data,
                            const float2* __restrict__ src_model, uint64_t n_vis,
                            uint32_t n_dir, uint32_t n_models_copied,
                            float2* __restrict__ dst_vis) {
  const uint64_t tlr = uint64_t(s.T) * s.L * s.R;
  for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e < tlr;
       e += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t r = uint32_t(e % s.R);
    const uint64_t tl = e / s.R;
    const uint32_t ch = uint32_t(tl % s.L);
    const uint32_t t = uint32_t(tl / s.L);
    const uint32_t len = run_len[s.run_off + r];
    const bool flip = (len & kRunFlipped) != 0;
    const bool valid = ch < (len & ~kRunFlipped);
    const uint64_t v = valid ? s.src_base + t * s.tstride + run_src[s.run_off + r] + ch : 0;
    float2* dst = dst_vis + (uint64_t(1 + n_dir) * s.dst_elem_off) * NCORR;
    CopyVis<NCORR>(src_data + v * NCORR,
                   dst + SlabElem(s.R, s.W, 1 + n_dir, tl, 0, r) * NCORR, valid, flip);
    for (uint32_t d = 0; d < n_models_copied; ++d)
      CopyVis<NCORR>(src_model + (d * n_vis + v) * NCORR,
                     dst + SlabElem(s.R, s.W, 1 + n_dir, tl, 1 + d, r) * NCORR, valid, flip);
  }
}

// ---------------------------------------------------------------------------
// predict_kernel: model visibilities of point sources for one regular
// channel block, written in the reference layout model[dir][vis][corr] that
// pack_kernel reads -- DP3's predict of a point source (base/Simulator.cc:
// 112-245 visit(PointSource), station phases :477-520, flat Stokes spectrum
// :522-547): per source and station phi_p = 2 pi / c (u_p l + v_p m + w_p
// (n - 1)), the station shift exp(i phi_p nu), and V_pq(nu) += S shift_q(nu)
// conj(shift_p(nu)), with S = I + Q, U + iV, U - iV, I - Q for XX, XY, YX,
// YY (NCORR = 4), XX and YY (NCORR = 2) or I (NCORR = 1: DP3's
// single-correlation data is (XX + YY) / 2). FP64 throughout, stored
// complex64.
//
// station_phasor_kernel evaluates the station shifts once per (time,
// direction, source, station), as the reference's Simulator does, into a
// table: where the block's channels are evenly spaced, exp(i phi_p nu) at
// the first channel of every chunk of CH = kPredictChunk / NCORR channels
// and the per-channel step exp(i phi_p df); else exp(i phi_p nu) at every
// channel. predict_kernel (one thread per (time, baseline, direction),
// channels of a chunk in registers) forms each source's baseline phasor
// shift_q conj(shift_p) from the table and, for even spacing, advances it
// by the baseline step per channel (exp(i dphi (nu0 + k df)) = exp(i dphi
// nu0) exp(i dphi df)^k, restarted per chunk; relative drift ~ chunk *
// 1e-16, far below the complex64 rounding of the result). The sincos work
// is per station instead of per baseline.
// ---------------------------------------------------------------------------
constexpr int kPredictChunk = 16;
constexpr int kPredictThreads = 128;
constexpr double kTwoPiOverC = 2.0 * 3.14159265358979323846 / 299792458.0;

struct PredictParams {
  const double* src;        // [n_src_total][8]: l, m, n - 1, I, Q, U, V, 0
  const uint32_t* src_off;  // [n_dir + 1]: sources of direction d
  const double2* table;     // [n_times][n_dir][max_src][n_ant][n_slots] station phasors
  const uint32_t* a1;       // [n_bl]
  const uint32_t* a2;
  float2* model;            // [n_dir][n_times * n_bl * L][NCORR]
  uint32_t n_times, n_bl, L, n_ant, n_dir, max_src, n_slots;
  int uniform;              // channels evenly spaced: chunk starts + step in the table
  // Packed mode (run_ant non-null): thread bl is run bl of a packed channel
  // block, between the run's oriented antennas (a flipped baseline's model
  // is then the conjugate transpose its packing stores), written straight
  // into the packed layout: element t_elem[t] + SlabElem(n_bl, W, n_dir + 1,
  // t_row[t] + channel, 1 + d, bl) of vis.
  const uint32_t* run_ant;
  float2* vis;
  const uint64_t* t_elem;   // [n_times]
  const uint32_t* t_row;    // [n_times]
  uint32_t W;
  const uint32_t* unpol;    // [n_dir]: nonzero when all the direction's sources have Q = U = V = 0
};

struct PhasorParams {
  const double* uvw;        // [n_times][n_ant][3] station UVW (m)
  const double* src;
  const uint32_t* src_off;
  const double* freq;       // [L] channel frequencies of the block (Hz)
  double2* table;
  uint32_t n_times, n_ant, n_dir, max_src, L, n_slots, chunk;
  int uniform;
  double df;
};

__global__ void __launch_bounds__(kPredictThreads) station_phasor_kernel(const PhasorParams p) {
  const uint32_t st = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t t = blockIdx.y;
  if (st >= p.n_ant) return;
  const double* u = p.uvw + (size_t(t) * p.n_ant + st) * 3;
  for (uint32_t z = blockIdx.z; z < p.n_dir * p.max_src; z += gridDim.z) {
    const uint32_t d = z / p.max_src, s = z % p.max_src;
    const uint32_t s0 = p.src_off[d];
    if (s >= p.src_off[d + 1] - s0) continue;
    const double* q = p.src + size_t(s0 + s) * 8;
    const double phi = kTwoPiOverC * (u[0] * q[0] + u[1] * q[1] + u[2] * q[2]);
    double2* out =
        p.table + (((size_t(t) * p.n_dir + d) * p.max_src + s) * p.n_ant + st) * p.n_slots;
    double sn, cs;
    if (p.uniform) {
      const uint32_t n_chunks = p.n_slots - 1;
      for (uint32_t k = 0; k < n_chunks; ++k) {
        sincos(phi * p.freq[k * p.chunk], &sn, &cs);
        out[k] = make_double2(cs, sn);
      }
      sincos(phi * p.df, &sn, &cs);
      out[n_chunks] = make_double2(cs, sn);
    } else {
      for (uint32_t c = 0; c < p.L; ++c) {
        sincos(phi * p.freq[c], &sn, &cs);
        out[c] = make_double2(cs, sn);
      }
    }
  }
}

// a conj(b) of two unit phasors (cos, sin)
__device__ __forceinline__ void PhasorProduct(double2 a, double2 b, double& c, double& s) {
  c = a.x * b.x + a.y * b.y;
  s = a.y * b.x - a.x * b.y;
}

// One source's baseline phasor across the channels of a chunk and its
// correlation fluxes (XX = I + Q, XY = U + iV, YX = U - iV, YY = I - Q; for 1
// and 2 correlations real, so a term is two multiply-adds per correlation).
template <int NCORR, int CH>
struct PredictSource {
  double zs, zc, ss = 0.0, sc = 1.0;
  const double2* tp;
  const double2* tq;
  double re[NCORR], im[NCORR];
  // the four station phasors a Start needs: the chunk's first channel and
  // the step (evenly spaced channels) of both stations
  struct Loads {
    double2 q, p, qs, ps;
  };
  static __device__ __forceinline__ Loads Load(const double2* tp_, const double2* tq_,
                                               const PredictParams& p, uint32_t c0) {
    const uint32_t k = p.uniform ? c0 / CH : c0;
    Loads l;
    l.q = __ldg(tq_ + k);
    l.p = __ldg(tp_ + k);
    if (p.uniform) {
      l.qs = __ldg(tq_ + p.n_slots - 1);
      l.ps = __ldg(tp_ + p.n_slots - 1);
    }
    return l;
  }
  __device__ __forceinline__ void Start(const double* q, const double2* tp_, const double2* tq_,
                                        const PredictParams& p, uint32_t c0) {
    Start(q, tp_, tq_, p, Load(tp_, tq_, p, c0));
  }
  __device__ __forceinline__ void Start(const double* q, const double2* tp_, const double2* tq_,
                                        const PredictParams& p, const Loads& l) {
    tp = tp_;
    tq = tq_;
    PhasorProduct(l.q, l.p, zc, zs);
    if (p.uniform) PhasorProduct(l.qs, l.ps, sc, ss);
    if (NCORR == 1) {
      re[0] = q[3];
    } else if (NCORR == 2) {
      re[0] = q[3] + q[4];
      re[NCORR - 1] = q[3] - q[4];
    } else {
      re[0] = q[3] + q[4];
      re[1] = q[5];
      re[2] = q[5];
      re[NCORR - 1] = q[3] - q[4];
      im[0] = im[NCORR - 1] = 0.0;
      im[1] = q[6];
      im[2] = -q[6];
    }
  }
  __device__ __forceinline__ void Advance(const PredictParams& p, uint32_t ch) {
    if (p.uniform) {
      const double r = zc * sc - zs * ss;
      zs = zc * ss + zs * sc;
      zc = r;
    } else {
      PhasorProduct(__ldg(tq + ch), __ldg(tp + ch), zc, zs);
    }
  }
  __device__ __forceinline__ void AddTo(double2 (&acc)[NCORR]) const {
#pragma unroll
    for (int k = 0; k < NCORR; ++k) {
      if (NCORR == 4) {
        acc[k].x += re[k] * zc - im[k] * zs;
        acc[k].y += re[k] * zs + im[k] * zc;
      } else {
        acc[k].x += re[k] * zc;
        acc[k].y += re[k] * zs;
      }
    }
  }
};

// The channel chunks of one (time, baseline, direction): NA accumulators,
// NCORR, or one for a direction whose sources are all unpolarized (Stokes Q =
// U = V = 0: XX = YY = the same sum of I terms, XY = YX = 0, so one sum gives
// every correlation with the same products and additions).
template <int NCORR, int NA>
__device__ __forceinline__ void PredictChunks(const PredictParams& p, const double* src,
                                              uint32_t ns, const double2* tp0, const double2* tq0,
                                              size_t src_stride, float2* out, uint64_t cstride) {
  constexpr int CH = kPredictChunk / NCORR;
  for (uint32_t c0 = 0; c0 < p.L; c0 += CH) {
    const uint32_t nc = min(uint32_t(CH), p.L - c0);
    double2 acc[CH][NA];
#pragma unroll
    for (int c = 0; c < CH; ++c)
#pragma unroll
      for (int k = 0; k < NA; ++k) acc[c][k] = make_double2(0.0, 0.0);
    // Two sources at a time: their phasor chains are independent, so the
    // FP64 rotations of one fill the latency of the other's. Per channel the
    // sources are still added in order.
    // The next pair's table phasors are loaded before this pair's channel
    // work, so that their latency hides under it.
    using Src = PredictSource<NA, CH>;
    uint32_t s = 0;
    typename Src::Loads la, lb;
    if (ns >= 2) {
      la = Src::Load(tp0, tq0, p, c0);
      lb = Src::Load(tp0 + src_stride, tq0 + src_stride, p, c0);
    }
    for (; s + 2 <= ns; s += 2) {
      Src a, b;
      a.Start(src + s * 8, tp0 + s * src_stride, tq0 + s * src_stride, p, la);
      b.Start(src + (s + 1) * 8, tp0 + (s + 1) * src_stride, tq0 + (s + 1) * src_stride, p, lb);
      if (s + 4 <= ns) {
        la = Src::Load(tp0 + (s + 2) * src_stride, tq0 + (s + 2) * src_stride, p, c0);
        lb = Src::Load(tp0 + (s + 3) * src_stride, tq0 + (s + 3) * src_stride, p, c0);
      }
#pragma unroll
      for (int c = 0; c < CH; ++c) {
        if (c < int(nc)) {
          if (c > 0) {
            a.Advance(p, c0 + c);
            b.Advance(p, c0 + c);
          }
          a.AddTo(acc[c]);
          b.AddTo(acc[c]);
        }
      }
    }
    if (s < ns) {
      PredictSource<NA, CH> a;
      a.Start(src + s * 8, tp0 + s * src_stride, tq0 + s * src_stride, p, c0);
#pragma unroll
      for (int c = 0; c < CH; ++c) {
        if (c < int(nc)) {
          if (c > 0) a.Advance(p, c0 + c);
          a.AddTo(acc[c]);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < CH; ++c)
      if (c < int(nc)) {
        float2* o = out + uint64_t(c0 + c) * cstride;
#pragma unroll
        for (int k = 0; k < NCORR; ++k) {
          if (NA == NCORR) {
            o[k] = make_float2(float(acc[c][k].x), float(acc[c][k].y));
          } else {
            const bool diag = k == 0 || k == NCORR - 1;
            o[k] = diag ? make_float2(float(acc[c][0].x), float(acc[c][0].y))
                        : make_float2(0.f, 0.f);
          }
        }
      }
  }
}

// ALL_UNPOL: every direction of the launch is unpolarized (one accumulator
// per channel throughout, so the kernel's registers are those of that path).
template <int NCORR, bool ALL_UNPOL>
__global__ void __launch_bounds__(kPredictThreads) predict_kernel(const PredictParams p) {
  constexpr int CH = kPredictChunk / NCORR;
  extern __shared__ double predict_smem[];
  const uint32_t t = blockIdx.y, d = blockIdx.z;
  double* src = predict_smem;  // [n_src][8]
  const uint32_t s0 = p.src_off[d], ns = p.src_off[d + 1] - s0;
  for (uint32_t i = threadIdx.x; i < ns * 8; i += blockDim.x) src[i] = p.src[size_t(s0) * 8 + i];
  __syncthreads();
  const uint32_t bl = blockIdx.x * blockDim.x + threadIdx.x;
  if (bl >= p.n_bl) return;
  const bool packed = p.run_ant != nullptr;
  uint32_t ap, aq;
  if (packed) {
    const uint32_t x = p.run_ant[bl];
    ap = x & 0xFFFFu;
    aq = x >> 16;
  } else {
    ap = p.a1[bl];
    aq = p.a2[bl];
  }
  // channel c's model at out + c * cstride (packed: one slab row per channel)
  float2* out;
  uint64_t cstride;
  if (packed) {
    const uint64_t row_elems = uint64_t(p.n_bl) * (p.n_dir + 1);
    out = p.vis + (p.t_elem[t] + SlabElem(p.n_bl, p.W, p.n_dir + 1, p.t_row[t], 1 + d, bl)) *
                      NCORR;
    cstride = row_elems * NCORR;
  } else {
    const uint64_t n_vis = uint64_t(p.n_times) * p.n_bl * p.L;
    const uint64_t v0 = (uint64_t(t) * p.n_bl + bl) * p.L;
    out = p.model + (uint64_t(d) * n_vis + v0) * NCORR;
    cstride = NCORR;
  }
  auto at = [&](uint32_t c) -> float2* { return out + c * cstride; };
  if (ap == aq) {  // autocorrelations stay zero (Simulator.cc:162-163)
    for (uint32_t c = 0; c < p.L; ++c)
      for (int k = 0; k < NCORR; ++k) at(c)[k] = make_float2(0.f, 0.f);
    return;
  }
  // this (time, direction)'s table: [source][station][slot]
  const size_t src_stride = size_t(p.n_ant) * p.n_slots;
  const double2* tab = p.table + (size_t(t) * p.n_dir + d) * p.max_src * src_stride;
  const double2* tp0 = tab + size_t(ap) * p.n_slots;
  const double2* tq0 = tab + size_t(aq) * p.n_slots;
  if (ALL_UNPOL || NCORR == 1)
    PredictChunks<NCORR, 1>(p, src, ns, tp0, tq0, src_stride, out, cstride);
  else if (p.unpol[d])
    PredictChunks<NCORR, 1>(p, src, ns, tp0, tq0, src_stride, out, cstride);
  else
    PredictChunks<NCORR, NCORR>(p, src, ns, tp0, tq0, src_stride, out, cstride);
}

// ---------------------------------------------------------------------------
// weigh_kernel: DDECal's AssignAndWeight (ddecal/gain_solvers/SolverTools.cc:
// 81-167) and the regular SolveData conversion (SolveData.cc:18-31, 77-188)
// of one channel block, from DP3's raw buffer layout ([time][baseline]
// [channel][XX XY YX YY]) into the reference layout that pack_kernel reads.
// Per visibility: flagged if any correlation is flagged or non-finite in the
// data or in any direction's model (:112-124); data and every model weighted
// by sqrt(w) (or w in linear mode) per correlation (:131-139, Weigh :48-79);
// flagged visibilities zeroed (:145-162); then ToSpecificMatrix (XX, YY for
// 2 correlations, (XX + YY) / 2 for 1). One thread per (time, cross
// baseline, channel of the block); autocorrelations are not visited (the
// SolveData constructor drops them, :100,137).
// ---------------------------------------------------------------------------
struct WeighParams {
  const float2* data;            // [n_times][n_bl][n_ch][4]
  const float* weights;          // [n_times][n_bl][n_ch][4]
  const uint8_t* flags;          // [n_times][n_bl][n_ch][4] or null
  const float2* model;           // raw [dir][t][bl][ch][4], or predicted [dir][t][bx][L][4]
  const uint32_t* bl_of_cross;   // [n_bx] buffer baseline of each cross baseline
  float2* out;                   // data [n_vis][NCORR], then model [dir][n_vis][NCORR]
  uint32_t n_times, n_bl, n_ch, n_bx, c0, L, n_dir;
  int model_predicted, linear;
};

template <int NCORR>
__global__ void weigh_kernel(const WeighParams p) {
  const uint64_t n_vis = uint64_t(p.n_times) * p.n_bx * p.L;
  for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < n_vis;
       v += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t ch = uint32_t(v % p.L);
    const uint32_t bx = uint32_t((v / p.L) % p.n_bx);
    const uint32_t t = uint32_t(v / (uint64_t(p.L) * p.n_bx));
    const uint32_t bl = p.bl_of_cross[bx];
    const uint64_t ri = (uint64_t(t) * p.n_bl + bl) * p.n_ch + p.c0 + ch;
    auto model_at = [&](uint32_t d) -> const float2* {
      const uint64_t mi = p.model_predicted
                              ? (uint64_t(d) * p.n_times + t) * p.n_bx * p.L +
                                    uint64_t(bx) * p.L + ch
                              : (uint64_t(d) * p.n_times + t) * p.n_bl * p.n_ch +
                                    uint64_t(bl) * p.n_ch + p.c0 + ch;
      return p.model + mi * 4;
    };
    auto finite = [](float2 z) { return isfinite(z.x) && isfinite(z.y); };
    float2 dv[4];
    float pw[4];
    bool flag = false;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      dv[k] = p.data[ri * 4 + k];
      const float w = p.weights[ri * 4 + k];
      pw[k] = p.linear ? w : sqrtf(w);
      flag = flag || (p.flags && p.flags[ri * 4 + k]) || !finite(dv[k]);
    }
    for (uint32_t d = 0; d < p.n_dir && !flag; ++d) {
      const float2* m = model_at(d);
#pragma unroll
      for (int k = 0; k < 4; ++k) flag = flag || !finite(m[k]);
    }
    // Products and the 1-correlation sum rounded separately (no fused
    // multiply-add), as the reference's complex<float> arithmetic rounds them.
    auto put = [&](float2* dst, const float2 (&z)[4]) {
      if (NCORR == 4) {
#pragma unroll
        for (int k = 0; k < 4; ++k) dst[k] = z[k];
      } else if (NCORR == 2) {
        dst[0] = z[0];
        dst[1] = z[3];
      } else {
        dst[0] = make_float2(0.5f * __fadd_rn(z[0].x, z[3].x), 0.5f * __fadd_rn(z[0].y, z[3].y));
      }
    };
    float2 z[4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
      z[k] = flag ? make_float2(0.f, 0.f)
                  : make_float2(__fmul_rn(dv[k].x, pw[k]), __fmul_rn(dv[k].y, pw[k]));
    put(p.out + v * NCORR, z);
    for (uint32_t d = 0; d < p.n_dir; ++d) {
      const float2* m = model_at(d);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float2 mk = m[k];
        z[k] = flag ? make_float2(0.f, 0.f)
                    : make_float2(__fmul_rn(mk.x, pw[k]), __fmul_rn(mk.y, pw[k]));
      }
      put(p.out + (n_vis * (1 + d) + v) * NCORR, z);
    }
  }
}

// ---------------------------------------------------------------------------
// correct_subtract_kernel: DDECal::CorrectAndSubtractModels
// (steps/DDECal.cc:1081-1125) with ApplySolutionAndSubtract (:1031-1079) for
// one interval in DP3's buffer layout. Per visibility (autocorrelations
// included) and direction the corrected model C = G_1 M G_2^H in FP64, as the
// reference's aocommon::MC2x2 (complex<double>) arithmetic: full-Jones
// J_1.Multiply(M).MultiplyHerm(J_2) (:1004-1011), diagonal
// (diag(g_1) M) diag(g_2)^H (:1013-1019), scalar M (g_1 conj(g_2))
// (:1021-1027), every product and sum rounded on its own (no fused
// multiply-add, as the host's separate multiplies and adds). C is summed over
// directions from zero in direction order; kept models are stored as
// complex<float> (AssignTo), and the data become
// float(double(data) - sum) (complex<float> -= complex<double>). Channel ch
// belongs to the even-split channel block of the solve (DDECal.cc:308-313).
// One thread per (time, baseline, channel): 32 bytes of data and 32 bytes of
// model per direction read, the same written back: an HBM-bound stream.
// ---------------------------------------------------------------------------
struct CorrectParams {
  const float4* data;                // [n_vis][2]: XX XY | YX YY
  const float4* const* model;        // [n_dir] -> [n_vis][2]
  float4* data_out;                  // or null (no subtraction)
  float4* const* model_out;          // [n_dir] -> [n_vis][2], or null (models not kept)
  const double2* solutions;  // [n_cb][n_ant][n_dir][NPOL]
  const uint32_t* a1;        // [n_bl]
  const uint32_t* a2;
  uint64_t n_vis;
  uint32_t n_bl, n_ch, n_cb, n_ant, n_dir;
};

__device__ __forceinline__ double2 zmul_rn(double2 a, double2 b) {
  return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                      __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 zadd_rn(double2 a, double2 b) {
  return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y));
}
__device__ __forceinline__ double2 zconj(double2 a) { return make_double2(a.x, -a.y); }

template <int NPOL>
__global__ void __launch_bounds__(256) correct_subtract_kernel(const CorrectParams p) {
  for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < p.n_vis;
       v += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t ch = uint32_t(v % p.n_ch);
    const uint32_t bl = uint32_t((v / p.n_ch) % p.n_bl);
    // the block cb with cb n_ch / n_cb <= ch < (cb + 1) n_ch / n_cb
    const uint32_t cb = uint32_t((uint64_t(ch + 1) * p.n_cb - 1) / p.n_ch);
    const double2* s1 = p.solutions + (size_t(cb) * p.n_ant + p.a1[bl]) * p.n_dir * NPOL;
    const double2* s2 = p.solutions + (size_t(cb) * p.n_ant + p.a2[bl]) * p.n_dir * NPOL;
    double2 sum[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) sum[k] = make_double2(0.0, 0.0);
#pragma unroll 2
    for (uint32_t d = 0; d < p.n_dir; ++d) {
      const float4* md = p.model[d] + v * 2;
      const float4 ma = __ldcs(md), mb = __ldcs(md + 1);
      const double2 m[4] = {make_double2(ma.x, ma.y), make_double2(ma.z, ma.w),
                            make_double2(mb.x, mb.y), make_double2(mb.z, mb.w)};
      double2 c[4];
      if constexpr (NPOL == 4) {
        const double2* j1 = s1 + size_t(d) * 4;
        const double2* j2 = s2 + size_t(d) * 4;
        const double2 t0 = zadd_rn(zmul_rn(j1[0], m[0]), zmul_rn(j1[1], m[2]));
        const double2 t1 = zadd_rn(zmul_rn(j1[0], m[1]), zmul_rn(j1[1], m[3]));
        const double2 t2 = zadd_rn(zmul_rn(j1[2], m[0]), zmul_rn(j1[3], m[2]));
        const double2 t3 = zadd_rn(zmul_rn(j1[2], m[1]), zmul_rn(j1[3], m[3]));
        const double2 h0 = zconj(j2[0]), h1 = zconj(j2[1]), h2 = zconj(j2[2]),
                      h3 = zconj(j2[3]);
        c[0] = zadd_rn(zmul_rn(t0, h0), zmul_rn(t1, h1));
        c[1] = zadd_rn(zmul_rn(t0, h2), zmul_rn(t1, h3));
        c[2] = zadd_rn(zmul_rn(t2, h0), zmul_rn(t3, h1));
        c[3] = zadd_rn(zmul_rn(t2, h2), zmul_rn(t3, h3));
      } else if constexpr (NPOL == 2) {
        const double2 g0 = s1[size_t(d) * 2], g1 = s1[size_t(d) * 2 + 1];
        const double2 h0 = zconj(s2[size_t(d) * 2]), h1 = zconj(s2[size_t(d) * 2 + 1]);
        c[0] = zmul_rn(zmul_rn(g0, m[0]), h0);
        c[1] = zmul_rn(zmul_rn(g0, m[1]), h1);
        c[2] = zmul_rn(zmul_rn(g1, m[2]), h0);
        c[3] = zmul_rn(zmul_rn(g1, m[3]), h1);
      } else {
        const double2 f = zmul_rn(s1[d], zconj(s2[d]));
#pragma unroll
        for (int k = 0; k < 4; ++k) c[k] = zmul_rn(m[k], f);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) sum[k] = zadd_rn(sum[k], c[k]);
      if (p.model_out) {
        float4* mo = p.model_out[d] + v * 2;
        __stcs(mo, make_float4(float(c[0].x), float(c[0].y), float(c[1].x), float(c[1].y)));
        __stcs(mo + 1, make_float4(float(c[2].x), float(c[2].y), float(c[3].x), float(c[3].y)));
      }
    }
    if (p.data_out) {
      const float4 da = __ldcs(p.data + v * 2), db = __ldcs(p.data + v * 2 + 1);
      __stcs(p.data_out + v * 2,
             make_float4(float(__dsub_rn(da.x, sum[0].x)), float(__dsub_rn(da.y, sum[0].y)),
                         float(__dsub_rn(da.z, sum[1].x)), float(__dsub_rn(da.w, sum[1].y))));
      __stcs(p.data_out + v * 2 + 1,
             make_float4(float(__dsub_rn(db.x, sum[2].x)), float(__dsub_rn(db.y, sum[2].y)),
                         float(__dsub_rn(db.z, sum[3].x)), float(__dsub_rn(db.w, sum[3].y))));
    }
  }
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
                       int use_handle, const uint32_t* cb_group, const LoopState* state) {
  if (use_handle && blockIdx.x == 0 && threadIdx.x == 0)
    cudaGraphSetConditional(handle, 0);
  const uint32_t cb = blockIdx.x;
  if (nonfinite[cb] == 0) return;
  // a finished interval keeps its solutions as they were when it stopped
  if (cb_group && state[cb_group[cb]].done) return;
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
    const uint32_t nd1 = 1 + n_dir;
    const size_t row_elems = size_t(sl.R) * nd1;

    for (uint32_t run0 = vis.run_lo; run0 < vis.run_hi; run0 += runs_per_block) {
      const uint32_t run = run0 + slot;
      const bool active = run < vis.run_hi;
      // the run's data in row 0, and the distance between its directions
      const size_t e0 = active ? SlabElem(sl.R, sl.W, nd1, 0, 0, run) : 0;
      const size_t jstep = active ? SlabElem(sl.R, sl.W, nd1, 0, 1, run) - e0 : 0;
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
          const size_t e = (size_t(t) * sl.L + ch) * row_elems + e0;
          float2 Rv[NCORR];
#pragma unroll
          for (int c = 0; c < NCORR; ++c) Rv[c] = make_float2(0.f, 0.f);
          if (active && g == 0) LoadVis<NCORR>(sl.vis, e, Rv);
          float2 M[DMAX][NCORR];
#pragma unroll
          for (int k = 0; k < DMAX; ++k) {
            if (active && k < nd) {
              LoadVis<NCORR>(sl.vis, e + size_t(1 + g + k * ng) * jstep, M[k]);
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

// One interval's AssignSolutions norm, stopping criterion and stall
// detection after an iteration whose norm sum / count are given; returns
// whether the interval stops.
__device__ bool ControlStep(LoopState& ls, const DevSettings& st, double sum, uint64_t cnt,
                            double* step_magnitudes) {
  // AssignSolutions (SolverBase.cc:297-306), no constraints: accuracy.
  const double mag = cnt == 0 ? 0.0 : sum / st.step_size / double(cnt);
  const uint32_t it = ls.iteration + 1;
  ls.iteration = it;
  if (it <= st.hard_cap) step_magnitudes[it - 1] = mag;
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
  return stop;
}

template <int NPOL>
__global__ void __launch_bounds__(kThreads) finalize_kernel(const FinParams p) {
  const uint32_t group = p.block_group[blockIdx.x];
  const uint32_t item = p.block_item0[blockIdx.x] + threadIdx.x;
  double norm_sum = 0.0;
  uint32_t norm_cnt = 0;
  const DevSettings st = *p.settings;
  // an interval that has stopped keeps its solutions
  const bool frozen = !p.host_mode && p.state[group].done;
  if (item < p.block_item_end[blockIdx.x] && !frozen) {
    const uint32_t cb = item / (p.n_ant * p.n_sub);
    const uint32_t rem = item - cb * p.n_ant * p.n_sub;
    const uint32_t ant = rem / p.n_sub;
    const uint32_t s = rem - ant * p.n_sub;
    const uint32_t d = p.dir_of_sub[s];
    const uint32_t acc_n = p.n_ant * p.n_dir * NPOL * 3;
    NeumaierSum nr[NPOL], ni[NPOL], dn[NPOL];
    const uint32_t j0 = p.fin_off[cb * p.n_sub + s];
    const uint32_t j1 = p.fin_mode == kFinAssignOnly ? j0 : p.fin_off[cb * p.n_sub + s + 1];
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
    double2* out = p.next_out + (size_t(cb) * p.n_ant * p.n_sub +
                                 size_t(ant) * p.n_sub + s) * NPOL;
    if (p.host_mode) {
#pragma unroll
      for (int q = 0; q < NPOL; ++q) out[q] = nxt[q];
    } else if (p.fin_mode == kFinAssignOnly) {
      // the stepped and constrained next solutions of this iteration
#pragma unroll
      for (int q = 0; q < NPOL; ++q) nxt[q] = out[q];
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
      if (p.fin_mode == kFinStepOnly) {
#pragma unroll
        for (int q = 0; q < NPOL; ++q) out[q] = nxt[q];
      }
    }
    if (!p.host_mode && p.fin_mode != kFinStepOnly) {
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
  if (p.host_mode || p.fin_mode == kFinStepOnly) return;

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
    const uint32_t prev = atomicAdd(&p.state[0].blocks_done, 1u);
    s_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  // The last block runs the control step of every interval still going, one
  // thread per interval, in a fixed block order.
  bool active = false;
  for (uint32_t g = threadIdx.x; g < p.n_groups; g += blockDim.x) {
    LoopState& ls = p.state[g];
    if (ls.done) continue;
    double sum = 0.0;
    uint64_t cnt = 0;
    for (uint32_t b = p.group_blocks[g]; b < p.group_blocks[g + 1]; ++b) {
      sum += reinterpret_cast<volatile double*>(p.block_sum)[b];
      cnt += reinterpret_cast<volatile uint32_t*>(p.block_cnt)[b];
    }
    const bool stop = ControlStep(ls, st, sum, cnt, p.step_magnitudes + size_t(g) * p.mags_stride);
    active = active || !stop;
  }
  if (threadIdx.x == 0) p.state[0].blocks_done = 0;
  active = __syncthreads_or(active);
  if (threadIdx.x == 0 && p.use_handle) cudaGraphSetConditional(p.handle, active ? 1u : 0u);
}


// ---------------------------------------------------------------------------
// pipe_kernel: the Blackwell streaming path. Per CTA one producer thread
// moves the (time, channel) rows of each tile from HBM into a ring of
// shared-memory stages, one 1-D bulk copy per row (cp.async.bulk, completion
// on an mbarrier, no multicast; the tile-packed slab layout makes a row of a
// tile, data and every direction, contiguous). Seven consumer warps compute
// the residual and the per-direction P/Q sums from shared memory, one lane per
// run (or four lanes per run for 13-48 directions), and reduce each tile into
// the CTA's shared-memory antenna accumulators in barrier-separated phases
// over groups of runs with distinct antennas (runs are stored in
// cyclic-diagonal order), or by a counting sort where a tile has no such
// grouping. No shared-memory float atomics.
//
// The finalisation is fused: after a grid-wide arrival count, every CTA
// finalises a slice of the (channel block, antenna, sub-solution) items (merge
// of the partial slots, FP64 update, step, norm, non-finite detection for the
// lazy MakeSolutionsFinite), interval by interval, and the last CTA to finish
// runs the iteration control of every interval still going. One launch per
// iteration. Every wait is bounded by a 4 s device timer; a timeout sets an
// error flag that the host reports as DDSOLVE_E_TIMEOUT, and all later waits
// of that CTA return at once so that the kernel still ends.
// ---------------------------------------------------------------------------
constexpr int kPipeConsumerWarps = 7;
constexpr int kPipeRuns = kPipeConsumerWarps * 32;  // runs per tile
constexpr int kPipeThreads = kPipeRuns + 32;         // + one producer warp
constexpr int kPipeMaxStages = 8;
static_assert(kPipeRuns <= 256 && kPipeRuns % 32 == 0, "tree reductions assume <= 256 consumers");
constexpr uint64_t kWaitBudgetNs = 4000000000ull;

struct PipeParams {
  const SlabDesc* slabs;
  const Frag* frags;
  const uint32_t* cta_frag_off;
  const uint32_t* slab_sol;
  double2* solutions;
  float* partials;
  float2* tables;         // gain tables [n_tables][table_f2]
  uint32_t table_f2;      // float2 per table (n_ant * gain_stride, even)
  const uint32_t* tab_off;  // finalisation: (cb, s) -> [tab_off, tab_off+1)
  const uint32_t* tab_ent;  //   entries table * 256 + direction
  uint32_t n_ant, n_dir, n_sub, n_cb;
  uint32_t acc_stride;    // floats per antenna in the accumulator table (PipeAccStride)
  uint32_t gain_stride;   // float2 per antenna in a gain table (PipeGainStride)
  uint32_t stages;
  uint32_t acc_floats;    // n_ant * acc_stride = one partial slot
  uint32_t owner_groups;  // direction groups per antenna in the sorted reduction
  uint32_t n_gbuf;        // gain table buffers in shared memory (1 or 2)
  const float* powers;    // model powers per tile [tile][dir][corr][kPipeRuns],
                          // or null: accumulated in the row loop
  uint32_t power_floats;  // floats per tile in `powers`
  // shared-memory layout (byte offsets)
  uint32_t off_acc, off_gtab, off_stg, off_cnt, off_off, off_pair, off_ent,
      off_wsum, off_stages;
  const uint32_t* fin_off;
  const uint32_t* fin_visits;
  const uint32_t* fin_first;  // first visit of each list when all lists are ranges, else null
  const uint32_t* dir_of_sub;
  uint32_t* cb_flag;     // channel block holds non-finite solutions
  double* cb_avg;        // replacement value for them (MakeSolutionsFinite)
  uint32_t* cb_newflag;  // set during the finalisation that produced them
  double* block_sum;     // per-CTA norm partials
  uint32_t* block_cnt;
  uint32_t* counters;    // [0] CTAs finalised, [1] error flag, [2] grid barrier
  double2* next_out;
  int32_t host_mode;
  int32_t fin_mode;      // FinFused / FinStepOnly / FinAssignOnly
  const DevSettings* settings;
  LoopState* state;
  double* step_magnitudes;
  cudaGraphConditionalHandle handle;
  int32_t use_handle;
  // Independent intervals (batched solve): interval g owns channel blocks
  // [group_cb[g], group_cb[g + 1]) (cb_group[cb] = g), its loop state
  // state[g], step magnitudes step_magnitudes[g * mags_stride] and norm
  // partials block_sum[g * gridDim.x + CTA]. One interval: n_groups = 1.
  uint32_t n_groups;
  const uint32_t* cb_group;
  const uint32_t* group_cb;
  uint32_t mags_stride;
};

// A fragment of an interval that has stopped: skipped by the producer and the
// consumers alike (the loop states do not change during a launch).
__device__ __forceinline__ bool FragFrozen(const PipeParams& p, uint32_t slab) {
  if (p.n_groups <= 1 || p.host_mode) return false;
  const uint32_t g = p.cb_group[p.slabs[slab].cb];
  return static_cast<volatile const LoopState*>(p.state)[g].done != 0;
}

__device__ __forceinline__ uint32_t SmemAddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void MbarInit(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)),
               "r"(count)
               : "memory");
}
__device__ __forceinline__ void MbarArriveExpectTx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                   SmemAddr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void MbarArrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(SmemAddr(bar))
               : "memory");
}
__device__ __forceinline__ bool MbarTryWait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n"
      " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(SmemAddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void BulkCopyG2S(void* dst, const void* src,
                                            uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(SmemAddr(dst)),
      "l"(src), "r"(bytes), "r"(SmemAddr(bar))
      : "memory");
}
__device__ __forceinline__ uint64_t GlobalTimerNs() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Named barrier of the consumer warps: the warp-aligned form, entered by
// whole warps (__syncwarp first, so lane-divergent code before it is
// reconverged), at the same place by every consumer warp. Measured on B200:
// the non-aligned `barrier.sync 1, 224` let six waiting warps through while
// the seventh was still busy, and so did `bar.sync` after a loop that only
// one warp ran; waits of that kind are done by every warp instead.
__device__ __forceinline__ void ConsumerBarrier() {
  __syncwarp();
  asm volatile("bar.sync 1, %0;" ::"n"(kPipeRuns) : "memory");
}

// Bounded wait on an mbarrier phase. Returns false on timeout (or when the CTA
// is already in error), after recording the error.
__device__ __forceinline__ bool PipeWait(uint64_t* bar, uint32_t parity,
                                      volatile int* s_err, uint32_t* g_err) {
  if (MbarTryWait(bar, parity)) return true;
  const uint64_t t0 = GlobalTimerNs();
  for (uint32_t n = 1;; ++n) {
    if (*s_err) return false;
    if (MbarTryWait(bar, parity)) return true;
    if ((n & 63u) == 0 && GlobalTimerNs() - t0 > kWaitBudgetNs) {
      *s_err = 1;
      atomicExch(g_err, 1u);
      return false;
    }
  }
}

template <int NCORR>
__device__ __forceinline__ void LoadVisShared(const char* base, uint32_t idx,
                                              float2 (&v)[NCORR]) {
  if constexpr (NCORR == 2) {
    const float4 x = reinterpret_cast<const float4*>(base)[idx];
    v[0] = make_float2(x.x, x.y);
    v[1] = make_float2(x.z, x.w);
  } else {
    const float4 x = reinterpret_cast<const float4*>(base)[2 * idx];
    const float4 y = reinterpret_cast<const float4*>(base)[2 * idx + 1];
    v[0] = make_float2(x.x, x.y);
    v[1] = make_float2(x.z, x.w);
    v[2] = make_float2(y.x, y.y);
    v[3] = make_float2(y.z, y.w);
  }
}

// Accumulator table of pipe_kernel, per antenna `stride` floats: the
// numerators of every direction (NPOL complex values each), then the
// denominators (NPOL real values each), so that one direction's update is
// one vector read-modify-write of each (stride = 4 mod 8: distinct
// shared-memory banks for consecutive antennas).
template <int NPOL>
__device__ __forceinline__ void AccAdd(float* acc, uint32_t a, uint32_t stride, uint32_t n_dir,
                                       uint32_t d, const float2 (&num)[NPOL],
                                       const float (&den)[NPOL]) {
  float* row = acc + size_t(a) * stride;
  if constexpr (NPOL == 2) {
    float4* pn = reinterpret_cast<float4*>(row) + d;
    float4 v = *pn;
    v.x += num[0].x;
    v.y += num[0].y;
    v.z += num[1].x;
    v.w += num[1].y;
    *pn = v;
    float2* pd = reinterpret_cast<float2*>(row + 4 * n_dir) + d;
    float2 w = *pd;
    w.x += den[0];
    w.y += den[1];
    *pd = w;
  } else {
    float2* pn = reinterpret_cast<float2*>(row) + d;
    float2 v = *pn;
    v.x += num[0].x;
    v.y += num[0].y;
    *pn = v;
    row[2 * n_dir + d] += den[0];
  }
}
__host__ __device__ constexpr uint32_t AccNumOffset(uint32_t npol, uint32_t d, uint32_t q) {
  return (d * npol + q) * 2;
}
__host__ __device__ constexpr uint32_t AccDenOffset(uint32_t npol, uint32_t n_dir, uint32_t d,
                                                    uint32_t q) {
  return 2 * npol * n_dir + d * npol + q;
}

// Gains of antenna `ant`, direction d from a gain table (NPOL float2 per
// direction; for two polarizations one 16-byte load: stride = 2 mod 4).
template <int NPOL>
__device__ __forceinline__ void LoadGains(const float2* gtab, uint32_t ant, uint32_t stride,
                                          uint32_t d, float2 (&g)[NPOL]) {
  if constexpr (NPOL == 2) {
    const float4 v = *reinterpret_cast<const float4*>(gtab + size_t(ant) * stride + 2 * d);
    g[0] = make_float2(v.x, v.y);
    g[1] = make_float2(v.z, v.w);
  } else {
    g[0] = gtab[size_t(ant) * stride + d];
  }
}

// Writes the FP32 gain-table entries of solution (cb, ant, s): one entry per
// gain table of that channel block whose slab uses sub-solution s.
template <int NPOL>
__device__ __forceinline__ void WriteTables(const PipeParams& p, uint32_t cb,
                                            uint32_t ant, uint32_t s,
                                            const double2 (&v)[NPOL]) {
  const uint32_t k0 = p.tab_off[cb * p.n_sub + s];
  const uint32_t k1 = p.tab_off[cb * p.n_sub + s + 1];
  for (uint32_t k = k0; k < k1; ++k) {
    const uint32_t e = p.tab_ent[k];
    float2* t = p.tables + size_t(e >> 8) * p.table_f2 + size_t(ant) * p.gain_stride +
                (e & 255u) * NPOL;
#pragma unroll
    for (int q = 0; q < NPOL; ++q) t[q] = make_float2(float(v[q].x), float(v[q].y));
  }
}

// Grid-wide finalisation of pipe_kernel, after the grid barrier: the
// consumer threads of all CTAs take (channel block, antenna, sub-solution)
// items in a grid-stride loop, one round per independent interval (one round
// for a single interval): fixed-order compensated merge of the item's
// partial slots, FP64 add-back and division (IterativeDiagonalSolver.cc:206-221,
// IterativeScalarSolver.cc:184-194), SolverBase::Step (SolverBase.cc:88-158),
// the AssignSolutions norm (SolverBase.cc:234-285), and the FP32 gain tables
// of the next iteration. The last CTA to finish sums each interval's per-CTA
// norms in CTA order, runs ReachedStoppingCriterion / DetectStall (SolverBase.h:274-285,
// SolverBase.cc:63-86), and prepares the next iteration's
// MakeSolutionsFinite{1,2}Pol (SolverBase.cc:316-371) for channel blocks that
// got non-finite solutions. With device constraints the work is split by
// p.fin_mode: kFinStepOnly (pipe_kernel) stops after the step, writing the
// stepped solutions to next_out; kFinAssignOnly (assign_kernel) starts from
// the constrained ones in next_out.
template <int NPOL>
__device__ __forceinline__ void FinalizeDistributed(const PipeParams& p, int ctid,
                                                 double* s_sum, uint32_t* s_cnt,
                                                 uint32_t* s_last) {
  const DevSettings st = *p.settings;
  const uint32_t n_items_cb = p.n_ant * p.n_sub;
  const uint32_t n_items = p.n_cb * n_items_cb;
  double nsum = 0.0;
  uint32_t ncnt = 0;
  // One item: the merged sums and the old solutions in, the next solutions,
  // their norm terms, the gain tables and the non-finite flag out.
  auto finish = [&](uint32_t item, uint32_t cb, uint32_t ant, uint32_t s,
                    const double2 (&old_in)[NPOL], const NeumaierSum (&nr)[NPOL],
                    const NeumaierSum (&ni)[NPOL], const NeumaierSum (&dn)[NPOL]) {
    double2* sol = p.solutions + size_t(item) * NPOL;
    double2 old[NPOL], nxt[NPOL];
    bool pair_ok = true;
#pragma unroll
    for (int q = 0; q < NPOL; ++q) {
      old[q] = old_in[q];
      pair_ok = pair_ok && dfinite(old[q]);
    }
    // the lazy MakeSolutionsFinite of a solve (next-solutions passes use the
    // solutions they are given, as PerformIteration does)
    if (!pair_ok && !p.host_mode && p.cb_flag[cb]) {
      const double rv = p.cb_avg[cb];
#pragma unroll
      for (int q = 0; q < NPOL; ++q) old[q] = make_double2(rv, 0.0);
    }
#pragma unroll
    for (int q = 0; q < NPOL; ++q) {
      const float den = dn[q].Value();
      if (den == 0.f) {
        nxt[q] = make_double2(nan(""), 0.0);
      } else {
        nxt[q] = make_double2(
            double(float(old[q].x)) + double(nr[q].Value()) / double(den),
            double(float(old[q].y)) + double(ni[q].Value()) / double(den));
      }
    }
    double2* out = p.next_out + size_t(item) * NPOL;
    if (p.host_mode) {
#pragma unroll
      for (int q = 0; q < NPOL; ++q) out[q] = nxt[q];
      // the gain tables of a chained next pass, which starts from `nxt`
      // (every other launch rebuilds them from its own solutions first)
      WriteTables<NPOL>(p, cb, ant, s, nxt);
      return;
    }
    if (p.fin_mode == kFinAssignOnly) {
      // the stepped and constrained next solutions of this iteration
#pragma unroll
      for (int q = 0; q < NPOL; ++q) nxt[q] = out[q];
    } else {
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
      if (p.fin_mode == kFinStepOnly) {
#pragma unroll
        for (int q = 0; q < NPOL; ++q) out[q] = nxt[q];
        return;
      }
    }
    if (NPOL == 1) {
      if (old[0].x != 0.0 || old[0].y != 0.0) {
        const double2 diff = dmul(
            make_double2(nxt[0].x - old[0].x, nxt[0].y - old[0].y), dinv(old[0]));
        const double a = hypot(diff.x, diff.y);
        if (isfinite(a)) {
          nsum += a;
          ncnt += 1;
        }
      }
    } else {
      const double2 inv0 = dinv(old[0]);
      const double2 inv1 = dinv(old[NPOL - 1]);
      if (dfinite(inv0) && dfinite(inv1)) {
        const double2 d0 =
            dmul(make_double2(nxt[0].x - old[0].x, nxt[0].y - old[0].y), inv0);
        const double2 d1 = dmul(make_double2(nxt[NPOL - 1].x - old[NPOL - 1].x,
                                             nxt[NPOL - 1].y - old[NPOL - 1].y),
                                inv1);
        const double sumabs = hypot(d0.x, d0.y) + hypot(d1.x, d1.y);
        if (isfinite(sumabs)) {
          nsum += sumabs;
          ncnt += 2;
        }
      }
    }
    bool all_finite = true;
#pragma unroll
    for (int q = 0; q < NPOL; ++q) {
      sol[q] = nxt[q];
      all_finite = all_finite && dfinite(nxt[q]);
    }
    WriteTables<NPOL>(p, cb, ant, s, nxt);
    if (!all_finite) p.cb_newflag[cb] = 1u;
  };
  // A thread's items, kFinBatch at a time: their index, slot-list and
  // solution reads are issued together and their partial slots merged in
  // rounds, so that the chains of dependent L2 reads of the items overlap
  // (each item's slots are still added in slot order).
  // Interval by interval (one round for a single interval): its items spread
  // over all CTAs, its norm partial per CTA. An interval that has stopped
  // keeps its solutions.
  for (uint32_t g = 0; g < p.n_groups; ++g) {
    nsum = 0.0;
    ncnt = 0;
    const bool frozen = p.n_groups > 1 && !p.host_mode &&
                        static_cast<volatile const LoopState*>(p.state)[g].done != 0;
    const uint32_t i_lo = p.n_groups > 1 ? p.group_cb[g] * n_items_cb : 0u;
    const uint32_t i_hi = frozen ? i_lo : p.n_groups > 1 ? p.group_cb[g + 1] * n_items_cb : n_items;
    constexpr int kFinBatch = 4;
    const uint32_t item_step = gridDim.x * kPipeRuns;
    for (uint32_t item0 = i_lo + blockIdx.x * kPipeRuns + ctid; item0 < i_hi;
         item0 += kFinBatch * item_step) {
      uint32_t cbv[kFinBatch], antv[kFinBatch], sv[kFinBatch], dv[kFinBatch];
      uint32_t j0v[kFinBatch], j1v[kFinBatch], v0v[kFinBatch];
      double2 oldv[kFinBatch][NPOL];
  #pragma unroll
      for (int b = 0; b < kFinBatch; ++b) {
        const uint32_t item = item0 + b * item_step;
        cbv[b] = antv[b] = sv[b] = dv[b] = 0;
        j0v[b] = j1v[b] = v0v[b] = 0;
  #pragma unroll
        for (int q = 0; q < NPOL; ++q) oldv[b][q] = make_double2(0.0, 0.0);
        if (item < i_hi) {
          const uint32_t cb = item / n_items_cb;
          const uint32_t it = item - cb * n_items_cb;
          const uint32_t ant = it / p.n_sub;
          const uint32_t s = it - ant * p.n_sub;
          cbv[b] = cb;
          antv[b] = ant;
          sv[b] = s;
          dv[b] = p.dir_of_sub[s];
          j0v[b] = p.fin_off[cb * p.n_sub + s];
          j1v[b] = p.fin_off[cb * p.n_sub + s + 1];
          if (p.fin_first) v0v[b] = p.fin_first[cb * p.n_sub + s];
          const double2* sol = p.solutions + size_t(item) * NPOL;
  #pragma unroll
          for (int q = 0; q < NPOL; ++q) oldv[b][q] = sol[q];
        }
      }
      uint32_t n_rounds = 0;
  #pragma unroll
      for (int b = 0; b < kFinBatch; ++b) n_rounds = max(n_rounds, j1v[b] - j0v[b]);
      if (p.fin_mode == kFinAssignOnly) n_rounds = 0;  // no partial slots to merge
      NeumaierSum nr[kFinBatch][NPOL], ni[kFinBatch][NPOL], dn[kFinBatch][NPOL];
      constexpr int kR = 4;  // slots per item and round
      for (uint32_t k = 0; k < n_rounds; k += kR) {
        uint32_t vis[kFinBatch][kR];
  #pragma unroll
        for (int b = 0; b < kFinBatch; ++b)
  #pragma unroll
          for (int u = 0; u < kR; ++u)
            vis[b][u] = j0v[b] + k + u >= j1v[b] ? 0xFFFFFFFFu
                        : p.fin_first            ? v0v[b] + k + u
                                                 : p.fin_visits[j0v[b] + k + u];
        float v[kFinBatch][kR][NPOL * 3];
  #pragma unroll
        for (int b = 0; b < kFinBatch; ++b) {
          // the item's numerators and denominators in a partial slot (AccAdd)
          const size_t off_n = size_t(antv[b]) * p.acc_stride + AccNumOffset(NPOL, dv[b], 0);
          const size_t off_d =
              size_t(antv[b]) * p.acc_stride + AccDenOffset(NPOL, p.n_dir, dv[b], 0);
  #pragma unroll
          for (int u = 0; u < kR; ++u) {
            if (vis[b][u] == 0xFFFFFFFFu) continue;
            const float* a = p.partials + size_t(vis[b][u]) * p.acc_floats;
  #pragma unroll
            for (int e = 0; e < NPOL * 2; ++e) v[b][u][e] = __ldcg(a + off_n + e);
  #pragma unroll
            for (int q = 0; q < NPOL; ++q) v[b][u][NPOL * 2 + q] = __ldcg(a + off_d + q);
          }
        }
  #pragma unroll
        for (int b = 0; b < kFinBatch; ++b)
  #pragma unroll
          for (int u = 0; u < kR; ++u) {
            if (vis[b][u] == 0xFFFFFFFFu) continue;
  #pragma unroll
            for (int q = 0; q < NPOL; ++q) {
              nr[b][q].Add(v[b][u][q * 2 + 0]);
              ni[b][q].Add(v[b][u][q * 2 + 1]);
              dn[b][q].Add(v[b][u][NPOL * 2 + q]);
            }
          }
      }
  #pragma unroll
      for (int b = 0; b < kFinBatch; ++b) {
        const uint32_t item = item0 + b * item_step;
        if (item < i_hi) finish(item, cbv[b], antv[b], sv[b], oldv[b], nr[b], ni[b], dn[b]);
      }
    }
    s_sum[ctid] = nsum;
    s_cnt[ctid] = ncnt;
    ConsumerBarrier();
    for (int w = 128; w > 0; w >>= 1) {
      if (ctid < w && ctid + w < kPipeRuns) {
        s_sum[ctid] += s_sum[ctid + w];
        s_cnt[ctid] += s_cnt[ctid + w];
      }
      ConsumerBarrier();
    }
    if (ctid == 0) {
      p.block_sum[size_t(g) * gridDim.x + blockIdx.x] = s_sum[0];
      p.block_cnt[size_t(g) * gridDim.x + blockIdx.x] = s_cnt[0];
    }
    ConsumerBarrier();  // s_sum is reused by the next interval
  }
  // The last CTA finishes the iteration.
  if (ctid == 0) {
    __threadfence();
    const uint32_t prev = atomicAdd(&p.counters[0], 1u);
    *s_last = (prev == gridDim.x - 1) ? 1u : 0u;
  }
  ConsumerBarrier();
  if (!*s_last) return;
  __threadfence();
  if (p.fin_mode == kFinStepOnly) {
    // the assignment pass after the constraints finishes the iteration
    if (ctid == 0) {
      p.counters[0] = 0;
      p.counters[2] = 0;
    }
    return;
  }
  // Channel blocks with new non-finite solutions, checked by all consumer
  // threads at once (the serial pass below runs only when there are some).
  uint32_t any_bad = 0;
  if (!p.host_mode) {
    ConsumerBarrier();  // every thread has read *s_last above
    if (ctid == 0) *s_last = 0u;
    ConsumerBarrier();
    for (uint32_t cb = ctid; cb < p.n_cb; cb += kPipeRuns) {
      const bool bad = reinterpret_cast<volatile uint32_t*>(p.cb_newflag)[cb] != 0;
      if (!bad)
        p.cb_flag[cb] = 0u;
      else
        atomicOr(s_last, 1u);
    }
    ConsumerBarrier();
    any_bad = *s_last;
  }
  if (!p.host_mode && any_bad) {
    // Replacement values for channel blocks with new non-finite solutions:
    // mean |pol 0| over finite pairs; the gain tables take the replacement
    // now, the solutions when the next finalisation reads them.
    for (uint32_t cb = 0; cb < p.n_cb; ++cb) {
      const bool bad = reinterpret_cast<volatile uint32_t*>(p.cb_newflag)[cb] != 0;
      if (!bad) {
        if (ctid == 0) p.cb_flag[cb] = 0u;
        continue;
      }
      double asum = 0.0;
      uint32_t acnt = 0;
      for (uint32_t it = ctid; it < n_items_cb; it += kPipeRuns) {
        const double2* sol = p.solutions + (size_t(cb) * n_items_cb + it) * NPOL;
        bool ok = true;
        double2 v[NPOL];
#pragma unroll
        for (int q = 0; q < NPOL; ++q) {
          v[q] = __ldcg(sol + q);
          ok = ok && dfinite(v[q]);
        }
        if (ok) {
          asum += hypot(v[0].x, v[0].y);
          ++acnt;
        }
      }
      s_sum[ctid] = asum;
      s_cnt[ctid] = acnt;
      ConsumerBarrier();
      for (int w = 128; w > 0; w >>= 1) {
        if (ctid < w && ctid + w < kPipeRuns) {
          s_sum[ctid] += s_sum[ctid + w];
          s_cnt[ctid] += s_cnt[ctid + w];
        }
        ConsumerBarrier();
      }
      const double avg = s_cnt[0] == 0 ? 1.0 : s_sum[0] / double(s_cnt[0]);
      for (uint32_t it = ctid; it < n_items_cb; it += kPipeRuns) {
        const double2* sol = p.solutions + (size_t(cb) * n_items_cb + it) * NPOL;
        bool ok = true;
#pragma unroll
        for (int q = 0; q < NPOL; ++q) ok = ok && dfinite(__ldcg(sol + q));
        if (!ok) {
          double2 r[NPOL];
#pragma unroll
          for (int q = 0; q < NPOL; ++q) r[q] = make_double2(avg, 0.0);
          WriteTables<NPOL>(p, cb, it / p.n_sub, it % p.n_sub, r);
        }
      }
      ConsumerBarrier();
      if (ctid == 0) {
        p.cb_avg[cb] = avg;
        p.cb_flag[cb] = 1u;
        p.cb_newflag[cb] = 0u;
      }
      ConsumerBarrier();
    }
  }
  if (p.n_groups > 1 && !p.host_mode) {
    // Several intervals: one thread per interval still going sums its norm
    // partials in CTA order and runs its control step; the loop goes on while
    // any interval does.
    ConsumerBarrier();  // every thread has read *s_last
    if (ctid == 0) *s_last = 0u;
    ConsumerBarrier();
    const bool error = reinterpret_cast<volatile uint32_t*>(p.counters)[1] != 0;
    for (uint32_t g = ctid; g < p.n_groups; g += kPipeRuns) {
      LoopState& ls = p.state[g];
      if (ls.done) continue;
      double sum = 0.0;
      uint64_t cnt = 0;
      for (uint32_t b = 0; b < gridDim.x; ++b) {
        sum += reinterpret_cast<volatile double*>(p.block_sum)[size_t(g) * gridDim.x + b];
        cnt += reinterpret_cast<volatile uint32_t*>(p.block_cnt)[size_t(g) * gridDim.x + b];
      }
      bool stop = ControlStep(ls, st, sum, cnt, p.step_magnitudes + size_t(g) * p.mags_stride);
      if (error) {
        ls.done = 1;
        stop = true;
      }
      if (!stop) atomicOr(s_last, 1u);
    }
    ConsumerBarrier();
    if (ctid == 0) {
      p.counters[0] = 0;
      p.counters[2] = 0;
      if (p.use_handle) cudaGraphSetConditional(p.handle, *s_last ? 1u : 0u);
    }
    return;
  }
  // The per-CTA norm partials, summed by all consumer threads of the last CTA
  // in a fixed tree order (a serial sum by one thread sat on the critical
  // path of every iteration).
  {
    double sum_t = 0.0;
    uint32_t cnt_t = 0;
    for (uint32_t b = ctid; b < gridDim.x; b += kPipeRuns) {
      sum_t += reinterpret_cast<volatile double*>(p.block_sum)[b];
      cnt_t += reinterpret_cast<volatile uint32_t*>(p.block_cnt)[b];
    }
    s_sum[ctid] = sum_t;
    s_cnt[ctid] = cnt_t;
    ConsumerBarrier();
    for (int w = 128; w > 0; w >>= 1) {
      if (ctid < w && ctid + w < kPipeRuns) {
        s_sum[ctid] += s_sum[ctid + w];
        s_cnt[ctid] += s_cnt[ctid + w];
      }
      ConsumerBarrier();
    }
  }
  if (ctid != 0) return;
  const double sum = s_sum[0];
  const uint64_t cnt = s_cnt[0];
  p.counters[0] = 0;
  p.counters[2] = 0;
  if (p.host_mode) return;
  LoopState& ls = *p.state;
  const double mag = cnt == 0 ? 0.0 : sum / st.step_size / double(cnt);
  const uint32_t itn = ls.iteration + 1;
  ls.iteration = itn;
  if (itn <= st.hard_cap) p.step_magnitudes[itn - 1] = mag;
  const bool converged = mag <= st.accuracy;
  bool stalled = false;
  if (st.detect_stalling) {
    if (itn == 1) {
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
    if (itn >= 30)
      stalled = ls.step_mean <
                st.step_diff_sigma * sqrt(ls.step_var / double(ls.n_var_count));
  }
  const bool ready = itn >= st.max_iterations || converged || stalled;
  const bool error = p.counters[1] != 0;
  const bool stop =
      (itn >= st.min_iterations && ready) || itn >= st.hard_cap || error;
  ls.has_converged = converged;
  ls.has_stalled = stalled;
  ls.done = stop;
  if (p.use_handle) cudaGraphSetConditional(p.handle, stop ? 0u : 1u);
}

// Builds the FP32 gain tables from the FP64 solutions: one thread per
// (table, antenna, direction). tab_cb / tab_sol give each table's channel
// block and per-direction sub-solution.
template <int NPOL>
__global__ void build_tables_kernel(const double2* __restrict__ solutions,
                                    float2* __restrict__ tables,
                                    const uint32_t* __restrict__ tab_cb,
                                    const uint32_t* __restrict__ tab_sol,
                                    uint32_t n_tables, uint32_t n_ant, uint32_t n_dir,
                                    uint32_t n_sub, uint32_t gain_stride,
                                    uint32_t table_f2) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_tables * n_ant * n_dir) return;
  const uint32_t tab = i / (n_ant * n_dir);
  const uint32_t rem = i - tab * n_ant * n_dir;
  const uint32_t ant = rem / n_dir;
  const uint32_t d = rem - ant * n_dir;
  const uint32_t s = tab_sol[tab * n_dir + d];
  const double2* src = solutions + (size_t(tab_cb[tab] * n_ant + ant) * n_sub + s) * NPOL;
  float2* dst = tables + size_t(tab) * table_f2 + size_t(ant) * gain_stride + d * NPOL;
#pragma unroll
  for (int q = 0; q < NPOL; ++q) dst[q] = make_float2(float(src[q].x), float(src[q].y));
}

// Launched cooperatively (all CTAs co-resident), one CTA per SM.
// Model powers of the pipelined path: for every tile of runs, direction and
// correlation, sum over the tile's (time, channel) rows of |M|^2. They depend
// on the model alone, so they are computed once per upload instead of in
// every iteration's row loop. One block per (tile, direction), one thread per
// run; FP64 sums, stored as FP32.
struct PowerTile {
  uint32_t slab, r0, n, pad;
};

template <int NCORR>
__global__ void __launch_bounds__(kPipeRuns) power_kernel(const SlabDesc* __restrict__ slabs,
                                                          const PowerTile* __restrict__ tiles,
                                                          uint32_t n_dir, uint32_t power_floats,
                                                          float* __restrict__ powers) {
  const uint32_t tile = blockIdx.x / n_dir;
  const uint32_t k = blockIdx.x - tile * n_dir;
  const PowerTile t = tiles[tile];
  const SlabDesc sl = slabs[t.slab];
  const uint32_t r = threadIdx.x;
  double q[NCORR];
#pragma unroll
  for (int c = 0; c < NCORR; ++c) q[c] = 0.0;
  if (r < t.n) {
    const size_t rows = size_t(sl.T) * sl.L;
    const uint32_t nd1 = 1 + n_dir;
    const float2* m = static_cast<const float2*>(sl.vis) +
                      SlabElem(sl.R, sl.W, nd1, 0, 1 + k, t.r0 + r) * NCORR;
    for (size_t row = 0; row < rows; ++row, m += size_t(sl.R) * nd1 * NCORR) {
#pragma unroll
      for (int c = 0; c < NCORR; ++c) {
        const float2 v = __ldcs(m + c);
        q[c] += double(v.x) * v.x + double(v.y) * v.y;
      }
    }
  }
  float* out = powers + size_t(tile) * power_floats + size_t(k) * NCORR * kPipeRuns;
#pragma unroll
  for (int c = 0; c < NCORR; ++c) out[c * kPipeRuns + r] = float(q[c]);
}

// NG lanes per run (1, 2 or 4): a tile has kPipeRuns / NG runs and lane g of a
// run owns directions g, g + NG, ... (DMAX of them); the residual is the sum
// over the run's lanes (warp shuffles). NG = 1: one run per lane, exactly DMAX
// directions.
template <int NCORR, int NPOL, int DMAX, int NG>
__global__ void __launch_bounds__(kPipeThreads, 1) pipe_kernel(const PipeParams p) {
  static_assert(kPipeRuns % NG == 0 && 32 % NG == 0, "lanes per run must divide a warp");
  static_assert(NG == 1 || NCORR == 2, "lane groups are laid out for two correlations");
  constexpr int RUNS = kPipeRuns / NG;  // runs per tile
  // An unrolled graph body launches the kernel more than once per loop test:
  // a launch after the loop has stopped does nothing.
  if (!p.host_mode && p.use_handle) {
    bool all_done = true;
    for (uint32_t g = 0; g < p.n_groups && all_done; ++g)
      all_done = static_cast<volatile const LoopState*>(p.state)[g].done != 0;
    if (all_done) return;
  }
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + kPipeMaxStages;
  uint64_t* gfull = empty + kPipeMaxStages;  // gain table buffer loaded
  uint64_t* gfree = gfull + 2;               // gain table buffer released
  int* s_err = reinterpret_cast<int*>(gfree + 2);
  uint32_t* s_last = reinterpret_cast<uint32_t*>(s_err + 1);
  double* s_sum = reinterpret_cast<double*>(smem + 256);
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(s_sum + kPipeRuns);
  float* acc = reinterpret_cast<float*>(smem + p.off_acc);
  float2* gtab_buf = reinterpret_cast<float2*>(smem + p.off_gtab);
  float* stg = reinterpret_cast<float*>(smem + p.off_stg);
  uint32_t* a_cnt = reinterpret_cast<uint32_t*>(smem + p.off_cnt);
  uint32_t* a_off = reinterpret_cast<uint32_t*>(smem + p.off_off);
  uint32_t* t_pair = reinterpret_cast<uint32_t*>(smem + p.off_pair);
  uint16_t* ent = reinterpret_cast<uint16_t*>(smem + p.off_ent);
  uint32_t* s_wsum = reinterpret_cast<uint32_t*>(smem + p.off_wsum);
  char* stages = reinterpret_cast<char*>(smem + p.off_stages);
  constexpr uint32_t E = NCORR * 8;  // bytes per visibility
  const uint32_t acc_n = p.acc_floats;
  // NG = 1: each instantiation serves exactly DMAX directions (no padded
  // ones); NG > 1: up to NG * DMAX.
  const uint32_t n_dir = NG == 1 ? uint32_t(DMAX) : p.n_dir;
  // stage: [run antennas of the fragment, first row only][data][model 0..]
  constexpr uint32_t kRunsBytes = RUNS * 4;
  const uint32_t stage_bytes = kRunsBytes + (1 + n_dir) * RUNS * E;
  const uint32_t table_bytes = p.table_f2 * 8;
  const uint32_t S = p.stages;

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  if (tid == 0) {
    for (uint32_t s = 0; s < S; ++s) {
      MbarInit(&full[s], 1);
      MbarInit(&empty[s], kPipeConsumerWarps);
    }
    for (int b = 0; b < 2; ++b) {
      MbarInit(&gfull[b], 1);
      MbarInit(&gfree[b], kPipeConsumerWarps);
    }
    *s_err = 0;
    *s_last = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    if (p.use_handle && blockIdx.x == 0) cudaGraphSetConditional(p.handle, 0);
  }
  __syncthreads();

  const uint32_t f_begin = p.cta_frag_off[blockIdx.x];
  const uint32_t f_end = p.cta_frag_off[blockIdx.x + 1];

  if (warp == kPipeConsumerWarps) {
    // ---------------- producer warp: one thread issues all bulk copies ----
    if (lane != 0) return;
    uint32_t row = 0, nvis = 0, cur_visit = 0xFFFFFFFFu;
    uint32_t st = 0, ph = 0;  // stage of `row` and the parity of its use
    bool ok = true;
    for (uint32_t fi = f_begin; fi < f_end && ok; ++fi) {
      const Frag f = p.frags[fi];
      if (FragFrozen(p, f.slab)) continue;
      const SlabDesc sl = p.slabs[f.slab];
      if (f.visit != cur_visit) {  // new visit: its gain table first
        const uint32_t b = nvis % p.n_gbuf;
        const uint32_t use = nvis / p.n_gbuf;  // earlier uses of buffer b
        if (use >= 1 && !PipeWait(&gfree[b], (use - 1) & 1u, s_err, &p.counters[1])) {
          ok = false;
          break;
        }
        MbarArriveExpectTx(&gfull[b], table_bytes);
        BulkCopyG2S(gtab_buf + size_t(b) * p.table_f2,
                    p.tables + size_t(sl.table) * p.table_f2, table_bytes, &gfull[b]);
        cur_visit = f.visit;
        ++nvis;
      }
      // The fragment's tile is one tile of the packed slab: a row of it,
      // data and all directions, is one contiguous block.
      const uint32_t seg = (1 + n_dir) * f.n_runs * E;
      const size_t row_step = size_t(sl.R) * (1 + n_dir) * E;
      const char* src = static_cast<const char*>(sl.vis) + size_t(f.row_lo) * row_step +
                        size_t(f.r0) * (1 + n_dir) * E;
      for (uint32_t rr = f.row_lo; rr < f.row_hi; ++rr, ++row) {
        if (row >= S && !PipeWait(&empty[st], ph ^ 1u, s_err, &p.counters[1])) {
          ok = false;
          break;
        }
        // The fragment's run antennas travel with its first row (the run
        // arrays are padded to whole 16-byte groups).
        const uint32_t runs_bytes = rr == f.row_lo ? ((f.n_runs + 3u) & ~3u) * 4u : 0u;
        MbarArriveExpectTx(&full[st], seg + runs_bytes);
        char* dst = stages + size_t(st) * stage_bytes;
        if (runs_bytes) BulkCopyG2S(dst, sl.run_ant + f.r0, runs_bytes, &full[st]);
        BulkCopyG2S(dst + kRunsBytes, src, seg, &full[st]);
        src += row_step;
        if (++st == S) {
          st = 0;
          ph ^= 1u;
        }
      }
      if (NG == 1 && ok && (f.flags & kFragPower)) {
        // one more stage: the tile's model powers [dir][corr][run]
        if (row >= S && !PipeWait(&empty[st], ph ^ 1u, s_err, &p.counters[1])) {
          ok = false;
          break;
        }
        const uint32_t pb = n_dir * NCORR * kPipeRuns * 4;
        MbarArriveExpectTx(&full[st], pb);
        BulkCopyG2S(stages + size_t(st) * stage_bytes,
                    p.powers + size_t(f.tile) * p.power_floats, pb, &full[st]);
        ++row;
        if (++st == S) {
          st = 0;
          ph ^= 1u;
        }
      }
    }
    // Wait for the last copies, so none is in flight when the CTA ends.
    for (uint32_t k = 0; k < S && k < row; ++k) {
      const uint32_t r = row - 1 - k;
      PipeWait(&full[r % S], (r / S) & 1u, s_err, &p.counters[1]);
    }
    for (uint32_t k = 0; k < p.n_gbuf && k < nvis; ++k) {
      const uint32_t v = nvis - 1 - k;
      PipeWait(&gfull[v % p.n_gbuf], (v / p.n_gbuf) & 1u, s_err, &p.counters[1]);
    }
    return;
  }

  // ---------------- consumer warps ----------------
  const int ctid = tid;  // 0 .. kPipeRuns - 1
  // A warp holds 32 / NG runs; lane g * (32 / NG) + i serves run i of the
  // warp for directions g, g + NG, ...: the 8 lanes of a quarter warp read 8
  // consecutive runs of one direction row (distinct shared-memory banks).
  constexpr int kRunsPerWarp = 32 / NG;
  const int run = warp * kRunsPerWarp + lane % kRunsPerWarp;  // run within the tile
  const int g = lane / kRunsPerWarp;  // the lane's first direction
  const bool powers_pre = NG == 1 && p.powers != nullptr;
  uint32_t nvis = 0, cur_visit = 0xFFFFFFFFu;
  uint32_t st = 0, ph = 0;  // stage of the next row and the parity of its use
  const float2* gtab = gtab_buf;
  auto end_visit = [&]() {
    // all consumers are done with the visit: release its gain table buffer
    // and flush the accumulators into the visit's partial slot
    ConsumerBarrier();
    __syncwarp();
    if (lane == 0) MbarArrive(&gfree[(nvis - 1) % p.n_gbuf]);
    float* out = p.partials + size_t(cur_visit) * acc_n;
    for (uint32_t i = ctid; i < acc_n; i += kPipeRuns) __stcg(out + i, acc[i]);
    ConsumerBarrier();
  };
  // The next fragment's descriptor is fetched one fragment ahead, so that its
  // global-memory latency overlaps the current fragment's rows; the run
  // antennas arrive in shared memory with the fragment's first row.
  Frag nf{};
  if (f_begin < f_end) nf = p.frags[f_begin];
  for (uint32_t fi = f_begin; fi < f_end; ++fi) {
    const Frag f = nf;
    if (fi + 1 < f_end) nf = p.frags[fi + 1];
    if (FragFrozen(p, f.slab)) continue;
    if (f.visit != cur_visit) {
      if (cur_visit != 0xFFFFFFFFu) end_visit();
      for (uint32_t i = ctid; i < acc_n; i += kPipeRuns) acc[i] = 0.f;
      const uint32_t b = nvis % p.n_gbuf;
      PipeWait(&gfull[b], (nvis / p.n_gbuf) & 1u, s_err, &p.counters[1]);
      gtab = gtab_buf + size_t(b) * p.table_f2;
      cur_visit = f.visit;
      ++nvis;
      ConsumerBarrier();
    }
    const bool active = uint32_t(run) < f.n_runs;
    const uint32_t pitch = f.n_runs * E;  // bytes per direction row in a stage
    const bool warp_busy = uint32_t(warp) * (32u / NG) < f.n_runs;
    uint32_t a1 = 0, a2 = 0;
    float2 G[DMAX][NCORR];
    float2 P[DMAX][NCORR];
    float Q[DMAX][NCORR];
#pragma unroll
    for (int k = 0; k < DMAX; ++k)
#pragma unroll
      for (int c = 0; c < NCORR; ++c) {
        P[k][c] = make_float2(0.f, 0.f);
        Q[k][c] = 0.f;
      }
    for (uint32_t rr = f.row_lo; rr < f.row_hi; ++rr) {
      const uint32_t s = st;
      PipeWait(&full[s], ph, s_err, &p.counters[1]);
      if (++st == S) {
        st = 0;
        ph ^= 1u;
      }
      // Warps without runs in this tile only release the stage.
      if (warp_busy) {
        if (rr == f.row_lo) {
          // first row of the fragment: run antennas and the run's gain products
          const uint32_t ap =
              active ? reinterpret_cast<const uint32_t*>(stages + size_t(s) * stage_bytes)[run] : 0u;
          a1 = ap & 0xFFFFu;
          a2 = ap >> 16;
#pragma unroll
          for (int k = 0; k < DMAX; ++k) {
            float2 ga[NPOL], gb[NPOL];
#pragma unroll
            for (int q = 0; q < NPOL; ++q) {
              ga[q] = make_float2(0.f, 0.f);
              gb[q] = make_float2(0.f, 0.f);
            }
            const uint32_t d = g + k * NG;
            if (d < n_dir) {
              LoadGains<NPOL>(gtab, a1, p.gain_stride, d, ga);
              LoadGains<NPOL>(gtab, a2, p.gain_stride, d, gb);
            }
#pragma unroll
            for (int c = 0; c < NCORR; ++c)
              G[k][c] = cmul_conj(ga[RowPol<NCORR, NPOL>(c)], gb[ColPol<NCORR, NPOL>(c)]);
          }
        }
        const char* base = stages + size_t(s) * stage_bytes + kRunsBytes;
        // Residual R = D - sum_d G_d M_d, then P_d += R conj(M_d), and
        // Q_d += |M_d|^2 unless the model powers were precomputed. The model
        // row stays in registers between the two passes when it fits next to
        // the accumulators (shared-memory bandwidth is the row loop's limit),
        // else it is read from shared memory twice.
        auto row_body = [&](auto with_q) {
          constexpr bool kQ = decltype(with_q)::value;
          constexpr bool kKeepM = kQ ? DMAX * NCORR <= 12 : DMAX * NCORR <= 20;
          // The residual is summed in two halves (even and odd directions) to
          // halve its chain of dependent multiply-adds.
          // With NG > 1 each lane sums its own directions' terms and the
          // run's lanes then add theirs up (shuffles) before D is added.
          float2 Rv[NCORR], Ro[NCORR];
          if constexpr (NG == 1) {
            LoadVisShared<NCORR>(base, run, Rv);
          } else {
#pragma unroll
            for (int c = 0; c < NCORR; ++c) Rv[c] = make_float2(0.f, 0.f);
          }
#pragma unroll
          for (int c = 0; c < NCORR; ++c) Ro[c] = make_float2(0.f, 0.f);
          float2 Mk[kKeepM ? DMAX : 1][NCORR];
#pragma unroll
          for (int k = 0; k < DMAX; ++k) {
            float2 M[NCORR];
            if (g + k * NG < int(n_dir)) {
              LoadVisShared<NCORR>(base + size_t(1 + g + k * NG) * pitch, run, M);
            } else {
#pragma unroll
              for (int c = 0; c < NCORR; ++c) M[c] = make_float2(0.f, 0.f);
            }
            if constexpr (kKeepM) {
#pragma unroll
              for (int c = 0; c < NCORR; ++c) Mk[k][c] = M[c];
            }
#pragma unroll
            for (int c = 0; c < NCORR; ++c) {
              float2& r = (k & 1) ? Ro[c] : Rv[c];
              r.x = fmaf(-G[k][c].x, M[c].x, r.x);
              r.x = fmaf(G[k][c].y, M[c].y, r.x);
              r.y = fmaf(-G[k][c].x, M[c].y, r.y);
              r.y = fmaf(-G[k][c].y, M[c].x, r.y);
            }
          }
#pragma unroll
          for (int c = 0; c < NCORR; ++c) {
            Rv[c].x += Ro[c].x;
            Rv[c].y += Ro[c].y;
          }
          if constexpr (NG > 1) {
#pragma unroll
            for (int m = kRunsPerWarp; m < 32; m <<= 1)
#pragma unroll
              for (int c = 0; c < NCORR; ++c) {
                Rv[c].x += __shfl_xor_sync(0xFFFFFFFFu, Rv[c].x, m);
                Rv[c].y += __shfl_xor_sync(0xFFFFFFFFu, Rv[c].y, m);
              }
            float2 D[NCORR];
            LoadVisShared<NCORR>(base, run, D);
#pragma unroll
            for (int c = 0; c < NCORR; ++c) {
              Rv[c].x += D[c].x;
              Rv[c].y += D[c].y;
            }
          }
#pragma unroll
          for (int k = 0; k < DMAX; ++k) {
            float2 M[NCORR];
            if constexpr (kKeepM) {
#pragma unroll
              for (int c = 0; c < NCORR; ++c) M[c] = Mk[k][c];
            } else if (g + k * NG < int(n_dir)) {
              LoadVisShared<NCORR>(base + size_t(1 + g + k * NG) * pitch, run, M);
            } else {
#pragma unroll
              for (int c = 0; c < NCORR; ++c) M[c] = make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int c = 0; c < NCORR; ++c) {
              P[k][c].x = fmaf(Rv[c].x, M[c].x, P[k][c].x);
              P[k][c].x = fmaf(Rv[c].y, M[c].y, P[k][c].x);
              P[k][c].y = fmaf(Rv[c].y, M[c].x, P[k][c].y);
              P[k][c].y = fmaf(-Rv[c].x, M[c].y, P[k][c].y);
              if constexpr (kQ) {
                Q[k][c] = fmaf(M[c].x, M[c].x, Q[k][c]);
                Q[k][c] = fmaf(M[c].y, M[c].y, Q[k][c]);
              }
            }
          }
        };
        if (powers_pre)
          row_body(std::false_type{});
        else
          row_body(std::true_type{});
      }
      __syncwarp();
      if (lane == 0) MbarArrive(&empty[s]);
    }
    if (NG == 1 && (f.flags & kFragPower)) {
      // the tile's precomputed model powers, in the stage after its rows
      const uint32_t s = st;
      PipeWait(&full[s], ph, s_err, &p.counters[1]);
      if (++st == S) {
        st = 0;
        ph ^= 1u;
      }
      if (active) {
        const float* pw = reinterpret_cast<const float*>(stages + size_t(s) * stage_bytes);
#pragma unroll
        for (int k = 0; k < DMAX; ++k)
#pragma unroll
          for (int c = 0; c < NCORR; ++c)
            if (k < int(n_dir)) Q[k][c] = pw[(k * NCORR + c) * kPipeRuns + ctid];
      }
      __syncwarp();
      if (lane == 0) MbarArrive(&empty[s]);
    }

    // ---- tile reduction into the visit's antenna accumulators ----
    ConsumerBarrier();  // the previous reduction is complete everywhere
    if (f.flags & kFragDirect) {
      // The runs form up to eight consecutive groups; within a group the
      // first antennas are distinct and so are the second antennas. Per
      // group, two conflict-free phases of plain shared-memory updates.
      const uint32_t n_groups_t = (f.flags >> 8) & 0xFu;
      uint32_t my_group = 0;
#pragma unroll
      for (int gi = 0; gi < int(kMaxGroups) - 1; ++gi)
        my_group += uint32_t(run) >= ((f.group_end[gi >> 2] >> ((gi & 3) * 8)) & 0xFFu) &&
                    uint32_t(gi + 1) < n_groups_t;
      for (uint32_t phase = 0; phase < 2 * n_groups_t; ++phase) {
        const int side = int(phase & 1u);
        if (phase > 0) ConsumerBarrier();
        if (active && my_group == (phase >> 1)) {
          const uint32_t a = side == 0 ? a1 : a2;
          const uint32_t b = side == 0 ? a2 : a1;
#pragma unroll
          for (int k = 0; k < DMAX; ++k) {
            const uint32_t d = g + k * NG;
            if (d < n_dir) {
              float2 gb[NPOL];
              LoadGains<NPOL>(gtab, b, p.gain_stride, d, gb);
              float2 num[NPOL];
              float den[NPOL];
#pragma unroll
              for (int q = 0; q < NPOL; ++q) {
                float2 n = make_float2(0.f, 0.f);
                float dd = 0.f;
#pragma unroll
                for (int c = 0; c < NCORR; ++c) {
                  const int rp = RowPol<NCORR, NPOL>(c);
                  const int cp = ColPol<NCORR, NPOL>(c);
                  if (side == 0 && rp == q) {  // num += g_b P, den += |g_b|^2 Q
                    const float2 t1 = cmul(gb[cp], P[k][c]);
                    n.x += t1.x;
                    n.y += t1.y;
                    dd += cnorm(gb[cp]) * Q[k][c];
                  }
                  if (side == 1 && cp == q) {  // num += g_a conj(P), den += |g_a|^2 Q
                    const float2 t2 = cmul(gb[rp], cconj(P[k][c]));
                    n.x += t2.x;
                    n.y += t2.y;
                    dd += cnorm(gb[rp]) * Q[k][c];
                  }
                }
                num[q] = n;
                den[q] = dd;
              }
              AccAdd<NPOL>(acc, a, p.acc_stride, n_dir, d, num, den);
            }
          }
        }
      }
      continue;
    }
    if constexpr (NG > 1) {
      // the plan gives lane-group kernels direct tiles only
      if (ctid == 0) atomicExch(&p.counters[1], 1u);
      continue;
    } else {
    // Sorted reduction: stage the run's P/Q, counting-sort the (run, side)
    // pairs by antenna, then (antenna, direction group) owner threads add
    // them up; each accumulator entry has exactly one writer.
    constexpr uint32_t NVPD = 3 * NCORR;  // staged values per direction
#pragma unroll
    for (int k = 0; k < DMAX; ++k) {
      if (k < int(n_dir)) {
#pragma unroll
        for (int c = 0; c < NCORR; ++c) {
          float* v = stg + ((k * NCORR + c) * 3) * kPipeRuns + ctid;
          v[0] = P[k][c].x;
          v[kPipeRuns] = P[k][c].y;
          v[2 * kPipeRuns] = Q[k][c];
        }
      }
    }
    (void)NVPD;
    t_pair[ctid] = active ? (a1 | (a2 << 16)) : 0xFFFFFFFFu;
    for (uint32_t i = ctid; i < p.n_ant; i += kPipeRuns) a_cnt[i] = 0;
    ConsumerBarrier();
    // Ranks in run order (entries (run, side) of an antenna sorted by run, so
    // that the owner's sum has a fixed order); the counts by atomics.
    uint32_t rank1 = 0, rank2 = 0;
    if (active) {
      for (uint32_t j = 0; j < uint32_t(ctid); ++j) {
        const uint32_t pr = t_pair[j];
        if (pr == 0xFFFFFFFFu) continue;
        const uint32_t x1 = pr & 0xFFFFu, x2 = pr >> 16;
        rank1 += uint32_t(x1 == a1) + uint32_t(x2 == a1);
        rank2 += uint32_t(x1 == a2) + uint32_t(x2 == a2);
      }
      atomicAdd(&a_cnt[a1], 1u);
      atomicAdd(&a_cnt[a2], 1u);
    }
    ConsumerBarrier();
    {
      const uint32_t chunk = (p.n_ant + kPipeRuns - 1) / kPipeRuns;
      const uint32_t lo = min(p.n_ant, ctid * chunk);
      const uint32_t hi = min(p.n_ant, lo + chunk);
      uint32_t local = 0;
      for (uint32_t i = lo; i < hi; ++i) local += a_cnt[i];
      uint32_t x = local;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
      }
      if (lane == 31) s_wsum[warp] = x;
      ConsumerBarrier();
      uint32_t base = 0;
      for (int w = 0; w < warp; ++w) base += s_wsum[w];
      uint32_t run_off = base + x - local;
      for (uint32_t i = lo; i < hi; ++i) {
        a_off[i] = run_off;
        run_off += a_cnt[i];
      }
    }
    ConsumerBarrier();
    if (active) {
      ent[a_off[a1] + rank1] = uint16_t(ctid << 1);
      ent[a_off[a2] + rank2] = uint16_t((ctid << 1) | 1);
    }
    ConsumerBarrier();
    const uint32_t n_groups = p.owner_groups;
    for (uint32_t task = ctid; task < p.n_ant * n_groups; task += kPipeRuns) {
      const uint32_t a = task / n_groups;
      const uint32_t grp = task - a * n_groups;
      const uint32_t e0 = a_off[a], e1 = e0 + a_cnt[a];
      if (e1 == e0) continue;
      // directions grp, grp + n_groups, ... (at most DMAX), summed in
      // registers over the antenna's entries, then one shared update each
      float sum[DMAX][NPOL][3];
#pragma unroll
      for (int i = 0; i < DMAX; ++i)
#pragma unroll
        for (int q = 0; q < NPOL; ++q) sum[i][q][0] = sum[i][q][1] = sum[i][q][2] = 0.f;
      for (uint32_t e = e0; e < e1; ++e) {
        const uint32_t en = ent[e];
        const uint32_t j = en >> 1;
        const bool second = (en & 1u) != 0;  // antenna a is antenna 2 of run j
        const uint32_t pr = t_pair[j];
        const uint32_t b = second ? (pr & 0xFFFFu) : (pr >> 16);
#pragma unroll
        for (int i = 0; i < DMAX; ++i) {
          const uint32_t k = grp + i * n_groups;
          if (k < n_dir) {
            float2 gb[NPOL];
            LoadGains<NPOL>(gtab, b, p.gain_stride, k, gb);
            float2 Pc[NCORR];
            float Qc[NCORR];
#pragma unroll
            for (int c = 0; c < NCORR; ++c) {
              const float* v = stg + ((k * NCORR + c) * 3) * kPipeRuns + j;
              Pc[c] = make_float2(v[0], v[kPipeRuns]);
              Qc[c] = v[2 * kPipeRuns];
            }
#pragma unroll
            for (int q = 0; q < NPOL; ++q) {
#pragma unroll
              for (int c = 0; c < NCORR; ++c) {
                const int rp = RowPol<NCORR, NPOL>(c);
                const int cp = ColPol<NCORR, NPOL>(c);
                if (!second && rp == q) {  // num += g_b P, den += |g_b|^2 Q
                  const float2 t1 = cmul(gb[cp], Pc[c]);
                  sum[i][q][0] += t1.x;
                  sum[i][q][1] += t1.y;
                  sum[i][q][2] += cnorm(gb[cp]) * Qc[c];
                }
                if (second && cp == q) {  // num += g_a conj(P), den += |g_a|^2 Q
                  const float2 t2 = cmul(gb[rp], cconj(Pc[c]));
                  sum[i][q][0] += t2.x;
                  sum[i][q][1] += t2.y;
                  sum[i][q][2] += cnorm(gb[rp]) * Qc[c];
                }
              }
            }
          }
        }
      }
#pragma unroll
      for (int i = 0; i < DMAX; ++i) {
        const uint32_t k = grp + i * n_groups;
        if (k < n_dir) {
          float2 num[NPOL];
          float den[NPOL];
#pragma unroll
          for (int q = 0; q < NPOL; ++q) {
            num[q] = make_float2(sum[i][q][0], sum[i][q][1]);
            den[q] = sum[i][q][2];
          }
          AccAdd<NPOL>(acc, a, p.acc_stride, n_dir, k, num, den);
        }
      }
    }
    }  // NG == 1
  }
  if (cur_visit != 0xFFFFFFFFu) end_visit();
  // Grid barrier: every CTA has flushed every partial slot (the launch is
  // cooperative, so all CTAs are resident). Every consumer warp waits on the
  // arrival count itself (lane 0 polls, the warp follows): a named barrier
  // after one warp's polling loop was measured to let the other warps
  // through early. Bounded: a timeout flags an error and the finalisation
  // goes ahead on whatever is there.
  __threadfence();
  ConsumerBarrier();  // this CTA's slots are written
  if (ctid == 0) atomicAdd(&p.counters[2], 1u);
  {
    volatile uint32_t* arrived = &p.counters[2];
    const uint64_t t0 = GlobalTimerNs();
    for (uint32_t n = 1;; ++n) {
      // lane 0 decides (all arrived, or out of time) and the warp follows
      uint32_t stop = 0;
      if (lane == 0) {
        stop = *arrived >= gridDim.x ? 1u : 0u;
        if (!stop && (n & 63u) == 0 && GlobalTimerNs() - t0 > kWaitBudgetNs) {
          atomicExch(&p.counters[1], 1u);
          stop = 1u;
        }
      }
      if (__shfl_sync(0xFFFFFFFFu, stop, 0)) break;
      __nanosleep(64);
    }
    __threadfence();
  }
  FinalizeDistributed<NPOL>(p, ctid, s_sum, s_cnt, s_last);
}

// The assignment pass of a constrained iteration on the pipelined path
// (fin_mode = kFinAssignOnly): FinalizeDistributed over the constrained next
// solutions, with kPipeRuns threads per CTA (its barriers span them) and the
// CTA count of pipe_kernel (its norm partials).
template <int NPOL>
__global__ void __launch_bounds__(kPipeRuns) assign_kernel(const PipeParams p) {
  if (p.use_handle && static_cast<volatile const LoopState*>(p.state)->done) return;
  __shared__ double s_sum[kPipeRuns];
  __shared__ uint32_t s_cnt[kPipeRuns];
  __shared__ uint32_t s_last;
  if (threadIdx.x == 0) s_last = 0;
  __syncthreads();
  FinalizeDistributed<NPOL>(p, int(threadIdx.x), s_sum, s_cnt, &s_last);
}

// ---------------------------------------------------------------------------
// Device constraints: DP3's SmoothnessConstraint, AntennaConstraint and
// Constraint::ApplyReferenceAntenna applied to the stepped next solutions
// [n_cb][n_ant][n_sub][NPOL] (complex128) of an iteration, between the
// step-only and the assignment passes, so that a constrained solve stays in
// the device loop. All FP64, in the reference's order of operations. Every
// kernel returns at once when the solve has stopped (unrolled graph bodies).
// ---------------------------------------------------------------------------
__device__ __forceinline__ bool SolveStopped(const LoopState* state, int use_handle) {
  return use_handle && static_cast<volatile const LoopState*>(state)->done;
}

struct SmoothParams {
  const double2* in;        // [n_cb][n_series]
  double2* out;             // [n_cb][n_series]
  uint32_t n_cb, n_series;  // series = (ant * n_sub + sub) * n_pol + pol
  uint32_t n_ant, n_sub, n_pol;
  const double* freq;       // [n_cb] channel-block frequencies (Hz)
  const double* fcorr;      // [n_cb] (local bandwidth / bandwidth)^exponent
  const uint32_t* band;     // [n_cb][2] first and end channel block of the kernel
  const double* weights;    // [n_weight_sets][n_ant * n_cb]
  uint32_t per_sub_weights; // weights per sub-solution (SetSubSolutionWeights)
  const double* factor;     // [n_ant * n_sub] kernel size factor (dd / antenna)
  double bandwidth;
  int32_t truncate;
  const LoopState* state;
  int32_t use_handle;
};

// SmoothnessConstraint::Apply (SmoothnessConstraint.cc:48-97) with
// KernelSmoother::Smooth / Kernel (KernelSmoother.h:69-98, 108-160), Gaussian
// kernel: one thread per (channel block i, series); output i of a series is
// the kernel-weighted mean of its finite values over the band of i.
__global__ void __launch_bounds__(256) smooth_kernel(const SmoothParams p) {
  if (SolveStopped(p.state, p.use_handle)) return;
  const uint64_t idx = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= uint64_t(p.n_cb) * p.n_series) return;
  const uint32_t i = uint32_t(idx / p.n_series);
  const uint32_t series = uint32_t(idx - uint64_t(i) * p.n_series);
  const uint32_t sub = (series / p.n_pol) % p.n_sub;
  const uint32_t ant = series / (p.n_sub * p.n_pol);
  const double* w = p.weights + (p.per_sub_weights ? size_t(sub) * p.n_ant * p.n_cb : 0) +
                    size_t(ant) * p.n_cb;
  const double kernel_correction = p.fcorr[i] * p.factor[size_t(ant) * p.n_sub + sub];
  double2 sum = make_double2(0.0, 0.0);
  double weight_sum = 0.0;
  for (uint32_t j = p.band[2 * i]; j < p.band[2 * i + 1]; ++j) {
    const double2 v = p.in[size_t(j) * p.n_series + series];
    if (!dfinite(v)) continue;  // data 0, weight 0: adds nothing
    const double x = ((p.freq[i] - p.freq[j]) * kernel_correction) / p.bandwidth;
    const double k = (p.truncate && (x < -1.0 || x > 1.0)) ? 0.0 : exp(-x * x * 9.0);
    const double wt = k * w[j];
    sum.x += v.x * wt;
    sum.y += v.y * wt;
    weight_sum += wt;
  }
  p.out[size_t(i) * p.n_series + series] =
      weight_sum == 0.0 ? make_double2(nan(""), nan(""))
                        : make_double2(sum.x / weight_sum, sum.y / weight_sum);
}

// AntennaConstraint::Apply (AntennaConstraint.h:39-76): per channel block,
// antenna set, sub-solution and polarization, the mean of the set's finite
// solutions (0 / 0 = NaN when there are none) replaces each member's. One
// thread per (channel block, sub-solution, polarization), the sets in order.
__global__ void __launch_bounds__(256)
    antenna_constraint_kernel(double2* sol, uint32_t n_cb, uint32_t n_ant, uint32_t n_sub,
                              uint32_t n_pol, const uint32_t* set_off, const uint32_t* members,
                              uint32_t n_sets, const LoopState* state, int use_handle) {
  if (SolveStopped(state, use_handle)) return;
  const uint32_t per_cb = n_sub * n_pol;
  const uint64_t idx = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (idx >= uint64_t(n_cb) * per_cb) return;
  const uint32_t cb = uint32_t(idx / per_cb);
  const uint32_t sp = uint32_t(idx - uint64_t(cb) * per_cb);  // sub * n_pol + pol
  double2* base = sol + size_t(cb) * n_ant * per_cb + sp;
  for (uint32_t k = 0; k < n_sets; ++k) {
    double2 sum = make_double2(0.0, 0.0);
    double count = 0.0;
    for (uint32_t m = set_off[k]; m < set_off[k + 1]; ++m) {
      const double2 v = base[size_t(members[m]) * per_cb];
      if (dfinite(v)) {
        sum.x += v.x;
        sum.y += v.y;
        count += 1.0;
      }
    }
    const double2 mean = make_double2(sum.x / count, sum.y / count);
    for (uint32_t m = set_off[k]; m < set_off[k + 1]; ++m) base[size_t(members[m]) * per_cb] = mean;
  }
}

// Constraint::ApplyReferenceAntenna (Constraint.cc:7-37), first half: per
// polarization the first antenna whose direction-0 solutions are finite in
// more than 20% of the channel blocks (antenna 0 when there is none).
__global__ void reference_antenna_select_kernel(const double2* sol, uint32_t n_cb,
                                                uint32_t n_ant, uint32_t n_sub, uint32_t n_pol,
                                                uint32_t* ref_ant, const LoopState* state,
                                                int use_handle) {
  if (SolveStopped(state, use_handle)) return;
  const uint32_t pol = threadIdx.x;
  if (pol >= n_pol) return;
  uint32_t ref = 0;
  for (; ref < n_ant; ++ref) {
    uint32_t n_finite = 0;
    for (uint32_t cb = 0; cb < n_cb; ++cb)
      n_finite += dfinite(sol[((size_t(cb) * n_ant + ref) * n_sub) * n_pol + pol]) ? 1u : 0u;
    if (double(n_finite) > 0.2 * double(n_cb)) break;
  }
  ref_ant[pol] = ref == n_ant ? 0u : ref;
}

// std::complex<double> division a / b as C99 Annex G (G.5.1) specifies it:
// the divisor scaled by a power of two before the products.
__device__ __forceinline__ double2 ddiv(double2 a, double2 b) {
  const double m = fmax(fabs(b.x), fabs(b.y));
  int ilogbw = 0;
  double c = b.x, d = b.y;
  const double lw = logb(m);
  if (isfinite(lw)) {
    ilogbw = int(lw);
    c = scalbn(c, -ilogbw);
    d = scalbn(d, -ilogbw);
  }
  const double denom = c * c + d * d;
  return make_double2(scalbn((a.x * c + a.y * d) / denom, -ilogbw),
                      scalbn((a.y * c - a.x * d) / denom, -ilogbw));
}

// Second half: one thread per (channel block, polarization); every other
// antenna's solutions (all sub-solutions) are divided by the reference
// antenna's, which become 1.
__global__ void __launch_bounds__(256)
    reference_antenna_apply_kernel(double2* sol, uint32_t n_cb, uint32_t n_ant, uint32_t n_sub,
                                   uint32_t n_pol, const uint32_t* ref_ant,
                                   const LoopState* state, int use_handle) {
  if (SolveStopped(state, use_handle)) return;
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_cb * n_pol) return;
  const uint32_t cb = idx / n_pol, pol = idx - cb * n_pol;
  const uint32_t ref = ref_ant[pol];
  double2* base = sol + size_t(cb) * n_ant * n_sub * n_pol + pol;
  for (uint32_t s = 0; s < n_sub; ++s) {
    const double2 r = base[(size_t(ref) * n_sub + s) * n_pol];
    for (uint32_t a = 0; a < n_ant; ++a)
      if (a != ref) {
        double2& v = base[(size_t(a) * n_sub + s) * n_pol];
        v = ddiv(v, r);
      }
  }
  for (uint32_t s = 0; s < n_sub; ++s) base[(size_t(ref) * n_sub + s) * n_pol] = make_double2(1.0, 0.0);
}

// ---------------------------------------------------------------------------
// Full-Jones solver: IterativeFullJonesSolver (ddecal/gain_solvers/
// IterativeFullJonesSolver.cc:17-228). 2x2 complex gains J per antenna and
// sub-solution on 4-correlation data; the model correction of direction d is
// J_1 M_d J_2^H. Per antenna a and sub-solution, with the residual R = D -
// sum_d J_1 M_d J_2^H and the add-back identity R_d = R + J_1 M_d J_2^H:
//   side 1 (a = antenna 1): X = J_2 M^H,  num = sum R_d X   = P_1 + J_a den_1,
//                           den_1 = sum X^H X
//   side 2 (a = antenna 2): Y = J_1 M,    num = sum R_d^H Y = P_2 + J_a den_2,
//                           den_2 = sum Y^H Y
// (IterativeFullJonesSolver.cc:107-187), next = num den^-1 (NaN where den is
// singular). fj_pass_kernel: one thread per part of a run of visibilities
// (fixed baseline and sub-solutions; the rows of a run are split into
// n_parts parts), FP32 products and sums as the reference's MC2x2F
// arithmetic, the part's P and den of every direction and side written to its
// own partial slot (no atomics); fj_finalize_kernel: one thread per
// (channel block, antenna, sub-solution), the slots of its list summed in
// FP64 in run order, the 2x2 inverse and product in FP64, then Step, the
// 4-polarization AssignSolutions norm (SolverBase.cc:268-284) and the loop
// control, as finalize_kernel does for 1 and 2 polarizations.
// ---------------------------------------------------------------------------
struct C22 {  // row-major [m0 m1; m2 m3]
  float2 m[4];
};
__device__ __forceinline__ float2 cfma(float2 a, float2 b, float2 c) {  // a b + c
  return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
}
__device__ __forceinline__ float2 cfma_conj(float2 a, float2 b, float2 c) {  // a conj(b) + c
  return make_float2(fmaf(a.x, b.x, fmaf(a.y, b.y, c.x)), fmaf(a.y, b.x, fmaf(-a.x, b.y, c.y)));
}
__device__ __forceinline__ float2 cconj_fma(float2 a, float2 b, float2 c) {  // conj(a) b + c
  return make_float2(fmaf(a.x, b.x, fmaf(a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(-a.y, b.x, c.y)));
}
__device__ __forceinline__ C22 Mul22(const C22& x, const C22& y) {  // x y
  C22 r;
  const float2 z = make_float2(0.f, 0.f);
  r.m[0] = cfma(x.m[1], y.m[2], cmul(x.m[0], y.m[0]));
  r.m[1] = cfma(x.m[1], y.m[3], cmul(x.m[0], y.m[1]));
  r.m[2] = cfma(x.m[3], y.m[2], cmul(x.m[2], y.m[0]));
  r.m[3] = cfma(x.m[3], y.m[3], cmul(x.m[2], y.m[1]));
  (void)z;
  return r;
}
__device__ __forceinline__ C22 MulHerm22(const C22& x, const C22& y) {  // x y^H
  C22 r;
  r.m[0] = cfma_conj(x.m[1], y.m[1], cmul_conj(x.m[0], y.m[0]));
  r.m[1] = cfma_conj(x.m[1], y.m[3], cmul_conj(x.m[0], y.m[2]));
  r.m[2] = cfma_conj(x.m[3], y.m[1], cmul_conj(x.m[2], y.m[0]));
  r.m[3] = cfma_conj(x.m[3], y.m[3], cmul_conj(x.m[2], y.m[2]));
  return r;
}
// acc += x^H y
__device__ __forceinline__ void AddHermMul22(C22& acc, const C22& x, const C22& y) {
  acc.m[0] = cconj_fma(x.m[2], y.m[2], cconj_fma(x.m[0], y.m[0], acc.m[0]));
  acc.m[1] = cconj_fma(x.m[2], y.m[3], cconj_fma(x.m[0], y.m[1], acc.m[1]));
  acc.m[2] = cconj_fma(x.m[3], y.m[2], cconj_fma(x.m[1], y.m[0], acc.m[2]));
  acc.m[3] = cconj_fma(x.m[3], y.m[3], cconj_fma(x.m[1], y.m[1], acc.m[3]));
}
// acc += x y
__device__ __forceinline__ void AddMul22(C22& acc, const C22& x, const C22& y) {
  acc.m[0] = cfma(x.m[1], y.m[2], cfma(x.m[0], y.m[0], acc.m[0]));
  acc.m[1] = cfma(x.m[1], y.m[3], cfma(x.m[0], y.m[1], acc.m[1]));
  acc.m[2] = cfma(x.m[3], y.m[2], cfma(x.m[2], y.m[0], acc.m[2]));
  acc.m[3] = cfma(x.m[3], y.m[3], cfma(x.m[2], y.m[1], acc.m[3]));
}
__device__ __forceinline__ C22 LoadC22(const float2* p) {
  C22 r;
  const float4 a = reinterpret_cast<const float4*>(p)[0];
  const float4 b = reinterpret_cast<const float4*>(p)[1];
  r.m[0] = make_float2(a.x, a.y);
  r.m[1] = make_float2(a.z, a.w);
  r.m[2] = make_float2(b.x, b.y);
  r.m[3] = make_float2(b.z, b.w);
  return r;
}
__device__ __forceinline__ C22 LoadJones(const double2* s) {  // FP32, as MC2x2F(&solutions[..])
  C22 r;
#pragma unroll
  for (int k = 0; k < 4; ++k) r.m[k] = make_float2(float(s[k].x), float(s[k].y));
  return r;
}

constexpr int kFjThreads = 128;
// Directions whose gains and sums one thread holds in registers: up to this
// many, one pass kernel does everything in one read of the visibilities; more
// directions go through fj_residual_kernel and fj_accumulate_kernel.
constexpr int kFjMaxDirections = 4;
constexpr uint32_t kFjSlotFloats = 32;  // per run and direction: P and den of both sides

struct FjPassParams {
  const SlabDesc* slabs;
  const uint32_t* slab_sol;   // [slab][n_dir]
  const uint32_t* run_start;  // [n_slabs + 1]: first global run of each slab
  const double2* solutions;   // [cb][ant][sub][4]
  float* partials;            // [part][global run][direction][kFjSlotFloats]
  uint32_t n_slabs, n_runs, n_ant, n_sub, n_dir;
  uint32_t n_parts;           // each run's rows split into this many parts
  float2* resid;              // more than kFjMaxDirections: the residual, [slab rows][R][4]
  const uint64_t* resid_off;  // [n_slabs]: first residual element of each slab
  const LoopState* state;
  int32_t use_handle;
};

// The slab holding global run gr (run_start is ascending).
__device__ __forceinline__ uint32_t FjSlabOf(const FjPassParams& p, uint32_t gr) {
  uint32_t lo = 0, hi = p.n_slabs;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (p.run_start[mid] <= gr)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// A Gram matrix sum X^H X, Hermitian: its real diagonal and the upper
// element. The products and sums of these three elements are those of
// AddHermMul22; the lower element is the conjugate of the upper one (as the
// host's non-fused complex arithmetic gives it) and the diagonal is real.
struct H22 {
  float d00, d11;
  float2 d01;
};
__device__ __forceinline__ void ZeroH22(H22& h) {
  h.d00 = h.d11 = 0.f;
  h.d01 = make_float2(0.f, 0.f);
}
// acc += x^H x
__device__ __forceinline__ void AddGram22(H22& acc, const C22& x) {
  acc.d00 = fmaf(x.m[2].x, x.m[2].x,
                 fmaf(x.m[2].y, x.m[2].y, fmaf(x.m[0].x, x.m[0].x, fmaf(x.m[0].y, x.m[0].y, acc.d00))));
  acc.d11 = fmaf(x.m[3].x, x.m[3].x,
                 fmaf(x.m[3].y, x.m[3].y, fmaf(x.m[1].x, x.m[1].x, fmaf(x.m[1].y, x.m[1].y, acc.d11))));
  acc.d01 = cconj_fma(x.m[2], x.m[3], cconj_fma(x.m[0], x.m[1], acc.d01));
}

template <int N>
__device__ __forceinline__ void FjStoreSlots(float* out, const C22* P1, const H22* D1,
                                             const C22* P2, const H22* D2) {
#pragma unroll
  for (int d = 0; d < N; ++d) {
    const C22* ps[2] = {&P1[d], &P2[d]};
    const H22* ds[2] = {&D1[d], &D2[d]};
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      float4* o = reinterpret_cast<float4*>(out + d * kFjSlotFloats + q * 16);
      o[0] = make_float4(ps[q]->m[0].x, ps[q]->m[0].y, ps[q]->m[1].x, ps[q]->m[1].y);
      o[1] = make_float4(ps[q]->m[2].x, ps[q]->m[2].y, ps[q]->m[3].x, ps[q]->m[3].y);
      o[2] = make_float4(ds[q]->d00, 0.f, ds[q]->d01.x, ds[q]->d01.y);
      o[3] = make_float4(ds[q]->d01.x, -ds[q]->d01.y, ds[q]->d11, 0.f);
    }
  }
}

// More than kFjMaxDirections directions: fj_residual_kernel first stores
// every visibility's residual R = V - sum_d J_1 M_d J_2^H (in direction
// order, with the same FP32 operations as fj_pass_kernel) in HBM, taking
// rows in batches of kFjRowBatch so that each direction's gains are loaded
// once per batch; then fj_accumulate_kernel reads R and each direction's
// model and accumulates the directions. A pass reads the data and every
// model once for the residual, then R once more.
constexpr int kFjRowBatch = 8;

__global__ void __launch_bounds__(kFjThreads) fj_residual_kernel(const FjPassParams p) {
  if (SolveStopped(p.state, p.use_handle)) return;
  const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
  if (gt >= p.n_runs * p.n_parts) return;
  const uint32_t gr = gt % p.n_runs, part = gt / p.n_runs;
  const uint32_t si = FjSlabOf(p, gr);
  const SlabDesc sl = p.slabs[si];
  const uint32_t r = gr - p.run_start[si];
  const uint32_t ap = sl.run_ant[r];
  const uint32_t a1 = ap & 0xFFFFu, a2 = ap >> 16;
  const uint32_t nd = p.n_dir;
  const double2* sol1 = p.solutions + (size_t(sl.cb) * p.n_ant + a1) * p.n_sub * 4;
  const double2* sol2 = p.solutions + (size_t(sl.cb) * p.n_ant + a2) * p.n_sub * 4;
  const float2* vis = static_cast<const float2*>(sl.vis);
  float2* res = p.resid + p.resid_off[si] * 4;
  const uint64_t rows = uint64_t(sl.T) * sl.L;
  const uint64_t row_end = rows * (part + 1) / p.n_parts;
  for (uint64_t rb = rows * part / p.n_parts; rb < row_end; rb += kFjRowBatch) {
    const uint64_t nb = row_end - rb < uint64_t(kFjRowBatch) ? row_end - rb : kFjRowBatch;
    C22 R[kFjRowBatch];
#pragma unroll
    for (int i = 0; i < kFjRowBatch; ++i)
      if (uint64_t(i) < nb) R[i] = LoadC22(vis + SlabElem(sl.R, sl.W, nd + 1, rb + i, 0, r) * 4);
    for (uint32_t e = 0; e < nd; ++e) {
      const uint32_t s = p.slab_sol[sl.sol_off + e];
      const C22 J1 = LoadJones(sol1 + size_t(s) * 4), J2 = LoadJones(sol2 + size_t(s) * 4);
#pragma unroll
      for (int i = 0; i < kFjRowBatch; ++i) {
        if (uint64_t(i) < nb) {
          const C22 M = LoadC22(vis + SlabElem(sl.R, sl.W, nd + 1, rb + i, 1 + e, r) * 4);
          const C22 t = MulHerm22(Mul22(J1, M), J2);
#pragma unroll
          for (int k = 0; k < 4; ++k)
            R[i].m[k] = make_float2(R[i].m[k].x - t.m[k].x, R[i].m[k].y - t.m[k].y);
        }
      }
    }
#pragma unroll
    for (int i = 0; i < kFjRowBatch; ++i) {
      if (uint64_t(i) < nb) {
        float4* o = reinterpret_cast<float4*>(res + ((rb + i) * sl.R + r) * 4);
        o[0] = make_float4(R[i].m[0].x, R[i].m[0].y, R[i].m[1].x, R[i].m[1].y);
        o[1] = make_float4(R[i].m[2].x, R[i].m[2].y, R[i].m[3].x, R[i].m[3].y);
      }
    }
  }
}

// More than kFjMaxDirections directions, after fj_residual_kernel: one
// thread per (part of a run, direction), the directions of a part on
// consecutive threads (so the part's residual is read once from HBM and then
// from cache), each reading R and its direction's model and accumulating
// that direction alone: a thread holds one direction's gains and sums, so
// the grid runs at high occupancy, in one launch for every direction.
__global__ void __launch_bounds__(kFjThreads) fj_accumulate_kernel(const FjPassParams p) {
  if (SolveStopped(p.state, p.use_handle)) return;
  const uint32_t nd = p.n_dir;
  const uint64_t gl = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
  const uint64_t unit = gl / nd;  // part * n_runs + global run
  const uint32_t d = uint32_t(gl % nd);
  if (unit >= uint64_t(p.n_runs) * p.n_parts) return;
  const uint32_t gr = uint32_t(unit % p.n_runs), part = uint32_t(unit / p.n_runs);
  const uint32_t si = FjSlabOf(p, gr);
  const SlabDesc sl = p.slabs[si];
  const uint32_t r = gr - p.run_start[si];
  const uint32_t ap = sl.run_ant[r];
  const uint32_t a1 = ap & 0xFFFFu, a2 = ap >> 16;
  const size_t cb_off = size_t(sl.cb) * p.n_ant * p.n_sub;
  const uint32_t s = p.slab_sol[sl.sol_off + d];
  const C22 J1 = LoadJones(p.solutions + (cb_off + size_t(a1) * p.n_sub + s) * 4);
  const C22 J2 = LoadJones(p.solutions + (cb_off + size_t(a2) * p.n_sub + s) * 4);
  C22 P1, P2;
  H22 D1, D2;
#pragma unroll
  for (int k = 0; k < 4; ++k) P1.m[k] = P2.m[k] = make_float2(0.f, 0.f);
  ZeroH22(D1);
  ZeroH22(D2);
  const float2* vis = static_cast<const float2*>(sl.vis);
  const float2* res = p.resid + p.resid_off[si] * 4;
  const uint64_t rows = uint64_t(sl.T) * sl.L;
  const uint64_t row_end = rows * (part + 1) / p.n_parts;
  for (uint64_t row = rows * part / p.n_parts; row < row_end; ++row) {
    const C22 R = LoadC22(res + (row * sl.R + r) * 4);
    const C22 M = LoadC22(vis + SlabElem(sl.R, sl.W, nd + 1, row, 1 + d, r) * 4);
    const C22 Y = Mul22(J1, M);
    const C22 X = MulHerm22(J2, M);
    AddMul22(P1, R, X);
    AddGram22(D1, X);
    AddHermMul22(P2, R, Y);
    AddGram22(D2, Y);
  }
  FjStoreSlots<1>(p.partials + (unit * nd + d) * kFjSlotFloats, &P1, &D1, &P2, &D2);
}


template <int ND>
__global__ void __launch_bounds__(kFjThreads) fj_pass_kernel(const FjPassParams p) {
  if (SolveStopped(p.state, p.use_handle)) return;
  const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
  if (gt >= p.n_runs * p.n_parts) return;
  const uint32_t gr = gt % p.n_runs, part = gt / p.n_runs;
  const uint32_t lo = FjSlabOf(p, gr);
  const SlabDesc sl = p.slabs[lo];
  const uint32_t r = gr - p.run_start[lo];
  const uint32_t ap = sl.run_ant[r];
  const uint32_t a1 = ap & 0xFFFFu, a2 = ap >> 16;
  const size_t cb_off = size_t(sl.cb) * p.n_ant * p.n_sub;
  C22 J1[ND], J2[ND], P1[ND], P2[ND];
  H22 D1[ND], D2[ND];
#pragma unroll
  for (int d = 0; d < ND; ++d) {
    const uint32_t s = p.slab_sol[sl.sol_off + d];
    J1[d] = LoadJones(p.solutions + (cb_off + size_t(a1) * p.n_sub + s) * 4);
    J2[d] = LoadJones(p.solutions + (cb_off + size_t(a2) * p.n_sub + s) * 4);
#pragma unroll
    for (int k = 0; k < 4; ++k)
      P1[d].m[k] = P2[d].m[k] = make_float2(0.f, 0.f);
    ZeroH22(D1[d]);
    ZeroH22(D2[d]);
  }
  const float2* vis = static_cast<const float2*>(sl.vis);
  const uint64_t rows = uint64_t(sl.T) * sl.L;
  const uint64_t row_end = rows * (part + 1) / p.n_parts;
  for (uint64_t row = rows * part / p.n_parts; row < row_end; ++row) {
    C22 M[ND];
#pragma unroll
    for (int d = 0; d < ND; ++d) M[d] = LoadC22(vis + SlabElem(sl.R, sl.W, ND + 1, row, 1 + d, r) * 4);
    C22 R = LoadC22(vis + SlabElem(sl.R, sl.W, ND + 1, row, 0, r) * 4);
    C22 Y[ND];  // J_1 M
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      Y[d] = Mul22(J1[d], M[d]);
      const C22 t = MulHerm22(Y[d], J2[d]);  // J_1 M J_2^H
#pragma unroll
      for (int k = 0; k < 4; ++k) R.m[k] = make_float2(R.m[k].x - t.m[k].x, R.m[k].y - t.m[k].y);
    }
#pragma unroll
    for (int d = 0; d < ND; ++d) {
      const C22 X = MulHerm22(J2[d], M[d]);  // J_2 M^H
      AddMul22(P1[d], R, X);
      AddGram22(D1[d], X);
      AddHermMul22(P2[d], R, Y[d]);
      AddGram22(D2[d], Y[d]);
    }
  }
  FjStoreSlots<ND>(p.partials + size_t(gt) * ND * kFjSlotFloats, P1, D1, P2, D2);
}

// NL lanes per part of a run (used for two directions: NL = 2, DPL = 1),
// lane l owning directions l * DPL .. l * DPL + DPL - 1 (those past n_dir
// idle). Per row
// every lane loads its own directions' models and the data, forms their
// terms J_1 M J_2^H, gathers the terms of the run's lanes by shuffles and
// subtracts them from the data in direction order, which gives every lane
// the residual of fj_pass_kernel (the same FP32 operations in the same
// order), and accumulates its own directions. A lane holds DPL directions'
// gains and sums instead of all of them, so an SM keeps more warps in flight.
template <int NL, int DPL>
__global__ void __launch_bounds__(kFjThreads) fj_lane_kernel(const FjPassParams p) {
  if (SolveStopped(p.state, p.use_handle)) return;
  const uint32_t gl = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t unit = gl / NL, l = gl % NL;  // unit: part * n_runs + global run
  if (unit >= p.n_runs * p.n_parts) return;    // the whole group of NL lanes
  const uint32_t lane = threadIdx.x & 31u;
  const unsigned group = ((1u << NL) - 1u) << (lane & ~uint32_t(NL - 1));
  const uint32_t first = lane & ~uint32_t(NL - 1);
  const uint32_t gr = unit % p.n_runs, part = unit / p.n_runs;
  const uint32_t si = FjSlabOf(p, gr);
  const SlabDesc sl = p.slabs[si];
  const uint32_t r = gr - p.run_start[si];
  const uint32_t ap = sl.run_ant[r];
  const uint32_t a1 = ap & 0xFFFFu, a2 = ap >> 16;
  const uint32_t nd = p.n_dir;
  C22 J1[DPL], J2[DPL], P1[DPL], P2[DPL];
  H22 D1[DPL], D2[DPL];
  const size_t cb_off = size_t(sl.cb) * p.n_ant * p.n_sub;
#pragma unroll
  for (int k = 0; k < DPL; ++k) {
#pragma unroll
    for (int q = 0; q < 4; ++q)
      J1[k].m[q] = J2[k].m[q] = P1[k].m[q] = P2[k].m[q] = make_float2(0.f, 0.f);
    ZeroH22(D1[k]);
    ZeroH22(D2[k]);
    const uint32_t d = l * DPL + k;
    if (d < nd) {
      const uint32_t s = p.slab_sol[sl.sol_off + d];
      J1[k] = LoadJones(p.solutions + (cb_off + size_t(a1) * p.n_sub + s) * 4);
      J2[k] = LoadJones(p.solutions + (cb_off + size_t(a2) * p.n_sub + s) * 4);
    }
  }
  const float2* vis = static_cast<const float2*>(sl.vis);
  const uint64_t rows = uint64_t(sl.T) * sl.L;
  const uint64_t row_end = rows * (part + 1) / p.n_parts;
  for (uint64_t row = rows * part / p.n_parts; row < row_end; ++row) {
    C22 M[DPL], Y[DPL], t[DPL];
#pragma unroll
    for (int k = 0; k < DPL; ++k) {
      const uint32_t d = l * DPL + k;
      if (d < nd) {
        M[k] = LoadC22(vis + SlabElem(sl.R, sl.W, nd + 1, row, 1 + d, r) * 4);
      } else {
#pragma unroll
        for (int q = 0; q < 4; ++q) M[k].m[q] = make_float2(0.f, 0.f);
      }
      Y[k] = Mul22(J1[k], M[k]);
      t[k] = MulHerm22(Y[k], J2[k]);  // J_1 M J_2^H of direction d
    }
    C22 R = LoadC22(vis + SlabElem(sl.R, sl.W, nd + 1, row, 0, r) * 4);
#pragma unroll
    for (int e = 0; e < NL; ++e)
#pragma unroll
      for (int k = 0; k < DPL; ++k) {
        C22 te;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          te.m[q].x = __shfl_sync(group, t[k].m[q].x, first + e);
          te.m[q].y = __shfl_sync(group, t[k].m[q].y, first + e);
        }
        if (uint32_t(e * DPL + k) < nd) {
#pragma unroll
          for (int q = 0; q < 4; ++q)
            R.m[q] = make_float2(R.m[q].x - te.m[q].x, R.m[q].y - te.m[q].y);
        }
      }
#pragma unroll
    for (int k = 0; k < DPL; ++k) {
      const C22 X = MulHerm22(J2[k], M[k]);  // J_2 M^H
      AddMul22(P1[k], R, X);
      AddGram22(D1[k], X);
      AddHermMul22(P2[k], R, Y[k]);
      AddGram22(D2[k], Y[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < DPL; ++k) {
    const uint32_t d = l * DPL + k;
    if (d < nd)
      FjStoreSlots<1>(p.partials + (size_t(unit) * nd + d) * kFjSlotFloats, &P1[k], &D1[k],
                      &P2[k], &D2[k]);
  }
}

struct D22 {
  double2 m[4];
};
__device__ __forceinline__ D22 DMul22(const D22& x, const D22& y) {
  D22 r;
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const double2 a = dmul(x.m[2 * i], y.m[j]), b = dmul(x.m[2 * i + 1], y.m[2 + j]);
      r.m[2 * i + j] = make_double2(a.x + b.x, a.y + b.y);
    }
  return r;
}
// x^-1, false when singular (det == 0), as aocommon's Matrix2x2::Invert.
__device__ __forceinline__ bool DInvert22(D22& x) {
  const double2 a = dmul(x.m[0], x.m[3]), b = dmul(x.m[1], x.m[2]);
  const double2 det = make_double2(a.x - b.x, a.y - b.y);
  if (det.x == 0.0 && det.y == 0.0) return false;
  const double2 inv = dinv(det);
  const double2 m0 = x.m[0];
  x.m[0] = dmul(x.m[3], inv);
  x.m[1] = dmul(make_double2(-x.m[1].x, -x.m[1].y), inv);
  x.m[2] = dmul(make_double2(-x.m[2].x, -x.m[2].y), inv);
  x.m[3] = dmul(m0, inv);
  return true;
}

struct FjFinParams {
  const float* partials;
  const uint32_t* list_off;   // [n_cb * n_ant * n_sub + 1]
  const uint32_t* list_ent;   // (slot index << 1) | side, slot = global run * n_dir + d
  double2* solutions;         // [cb][ant][sub][4]
  double2* next_out;          // host mode
  uint32_t n_items, n_dir;
  uint32_t n_ant, n_sub;
  int32_t host_mode;
  const DevSettings* settings;
  double* block_sum;
  uint32_t* block_cnt;
  LoopState* state;
  uint32_t* nonfinite;        // [n_cb]
  double* step_magnitudes;
  cudaGraphConditionalHandle handle;
  int32_t use_handle;
  uint32_t* blocks_done;
};

__global__ void __launch_bounds__(kThreads) fj_finalize_kernel(const FjFinParams p) {
  // one warp per item: the lanes sum interleaved entries of its list, a
  // butterfly combines them (a fixed order, so the result is reproducible),
  // lane 0 does the rest
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t item = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const DevSettings st = *p.settings;
  const bool stopped = !p.host_mode && p.state->done;
  double norm_sum = 0.0;
  uint32_t norm_cnt = 0;
  if (item < p.n_items && !stopped) {
    // the item's slots: P and den of its side
    double pn[8], dn[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) pn[k] = dn[k] = 0.0;
    for (uint32_t e = p.list_off[item] + lane; e < p.list_off[item + 1]; e += 32) {
      const uint32_t en = p.list_ent[e];
      const float4* slot = reinterpret_cast<const float4*>(
          p.partials + size_t(en >> 1) * kFjSlotFloats + (en & 1u) * 16);
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        const float4 a = __ldcg(slot + q), b = __ldcg(slot + 2 + q);
        pn[4 * q] += a.x;
        pn[4 * q + 1] += a.y;
        pn[4 * q + 2] += a.z;
        pn[4 * q + 3] += a.w;
        dn[4 * q] += b.x;
        dn[4 * q + 1] += b.y;
        dn[4 * q + 2] += b.z;
        dn[4 * q + 3] += b.w;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        pn[k] += __shfl_xor_sync(0xffffffffu, pn[k], o);
        dn[k] += __shfl_xor_sync(0xffffffffu, dn[k], o);
      }
    if (lane == 0) {
    double2* sol = p.solutions + size_t(item) * 4;
    D22 old, ja, den, num;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      old.m[k] = sol[k];
      ja.m[k] = make_double2(double(float(old.m[k].x)), double(float(old.m[k].y)));
      den.m[k] = make_double2(dn[2 * k], dn[2 * k + 1]);
    }
    // num = P + J_a den (the add-back of the item's own direction)
    num = DMul22(ja, den);
#pragma unroll
    for (int k = 0; k < 4; ++k) num.m[k] = make_double2(num.m[k].x + pn[2 * k], num.m[k].y + pn[2 * k + 1]);
    D22 nxt;
    if (DInvert22(den)) {
      nxt = DMul22(num, den);
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) nxt.m[k] = make_double2(nan(""), nan(""));
    }
    if (p.host_mode) {
      double2* out = p.next_out + size_t(item) * 4;
#pragma unroll
      for (int k = 0; k < 4; ++k) out[k] = nxt.m[k];
    } else {
      // SolverBase::Step (SolverBase.cc:88-158), element by element
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (!st.phase_only) {
          nxt.m[k] = make_double2(old.m[k].x * (1.0 - st.step_size) + nxt.m[k].x * st.step_size,
                                  old.m[k].y * (1.0 - st.step_size) + nxt.m[k].y * st.step_size);
        } else {
          const double from = atan2(old.m[k].y, old.m[k].x);
          double dist = atan2(nxt.m[k].y, nxt.m[k].x) - from;
          if (dist > M_PI)
            dist -= 2.0 * M_PI;
          else if (dist < -M_PI)
            dist += 2.0 * M_PI;
          double sn, cs;
          sincos(from + st.step_size * dist, &sn, &cs);
          nxt.m[k] = make_double2(cs, sn);
        }
      }
      // AssignSolutions, 4 polarizations (SolverBase.cc:268-284):
      // |(new - old) old^-1| summed over the four elements
      D22 inv = old;
      if (DInvert22(inv)) {
        D22 diff;
#pragma unroll
        for (int k = 0; k < 4; ++k)
          diff.m[k] = make_double2(nxt.m[k].x - old.m[k].x, nxt.m[k].y - old.m[k].y);
        const D22 ns = DMul22(diff, inv);
        double sumabs = 0.0;
#pragma unroll
        for (int k = 0; k < 4; ++k) sumabs += hypot(ns.m[k].x, ns.m[k].y);
        if (isfinite(sumabs)) {
          norm_sum += sumabs;
          norm_cnt += 4;
        }
      }
      bool all_finite = true;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        sol[k] = nxt.m[k];
        all_finite = all_finite && dfinite(nxt.m[k]);
      }
      if (!all_finite) p.nonfinite[item / (p.n_ant * p.n_sub)] = 1u;
    }
    }  // lane 0
  }
  if (p.host_mode) return;
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
    s_last = atomicAdd(p.blocks_done, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  *p.blocks_done = 0;
  LoopState& ls = *p.state;
  bool go = false;
  if (!ls.done) {
    double sum = 0.0;
    uint64_t cnt = 0;
    for (uint32_t b = 0; b < gridDim.x; ++b) {
      sum += reinterpret_cast<volatile double*>(p.block_sum)[b];
      cnt += reinterpret_cast<volatile uint32_t*>(p.block_cnt)[b];
    }
    go = !ControlStep(ls, st, sum, cnt, p.step_magnitudes);
  }
  if (p.use_handle) cudaGraphSetConditional(p.handle, go ? 1u : 0u);
}

// SolverBase::MakeSolutionsFinite4Pol (SolverBase.cc:372-403), one block per
// channel block flagged non-finite: matrices with a non-finite element get
// the mean |J_00| over the finite matrices in every element (the reference
// averages element 0 for all four), 1 where none is finite... as the
// reference: (1, 0, 0, 1) when no matrix is finite.
__global__ void __launch_bounds__(kThreads)
    make_finite4_kernel(double2* __restrict__ sols, uint32_t* nonfinite, uint32_t per_cb,
                        cudaGraphConditionalHandle handle, int use_handle, const LoopState* state) {
  if (use_handle && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(handle, 0);
  if (use_handle && state->done) return;
  const uint32_t cb = blockIdx.x;
  if (nonfinite[cb] == 0) return;
  double2* s = sols + size_t(cb) * per_cb;
  __shared__ double red_sum[kThreads];
  __shared__ uint32_t red_cnt[kThreads];
  auto finite4 = [&](uint32_t i) {
    return dfinite(s[i]) && dfinite(s[i + 1]) && dfinite(s[i + 2]) && dfinite(s[i + 3]);
  };
  double sum = 0.0;
  uint32_t cnt = 0;
  for (uint32_t i = threadIdx.x * 4; i < per_cb; i += blockDim.x * 4)
    if (finite4(i)) {
      sum += hypot(s[i].x, s[i].y);
      ++cnt;
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
  const bool none = red_cnt[0] == 0;
  const double avg = none ? 0.0 : red_sum[0] / double(red_cnt[0]);
  for (uint32_t i = threadIdx.x * 4; i < per_cb; i += blockDim.x * 4)
    if (!finite4(i))
      for (int k = 0; k < 4; ++k)
        s[i + k] = none ? make_double2(k == 0 || k == 3 ? 1.0 : 0.0, 0.0) : make_double2(avg, 0.0);
  __syncthreads();
  if (threadIdx.x == 0) nonfinite[cb] = 0;
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
  uint32_t W = 0;     // runs per tile of the packed layout
  uint64_t elem_off;  // within the channel block's packed buffer, in 1 + n_dir units
  uint64_t src_base, tstride;
  uint32_t run_off;
  std::vector<uint32_t> sol;  // [n_dir]
};

bool SameLayout(const std::vector<HostSlab>& a, const std::vector<HostSlab>& b) {
  if (a.size() != b.size()) return false;
  for (size_t i = 0; i < a.size(); ++i)
    if (a[i].T != b[i].T || a[i].L != b[i].L || a[i].R != b[i].R || a[i].W != b[i].W ||
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
  DevBuf vis, run_ant_dev;  // packed slabs (data and model), run antennas
  // Layout of the previous upload; an upload with the same layout into the
  // same buffers keeps the streaming plan (and its CUDA graph) valid.
  std::vector<HostSlab> prev_slabs;
  std::vector<uint32_t> prev_run_ant;
};

// Pads the run arrays to a whole number of 16-byte groups with empty runs.
void PadRuns(ChannelBlockStore& cb) {
  while (cb.run_ant.size() & 3u) {
    cb.run_ant.push_back(0u);
    cb.run_src.push_back(0u);
    cb.run_len.push_back(0u);
  }
}

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
  // plan knobs (ddsolve_tuning): -1 / 0 = automatic
  int32_t tune_pipe = -1, tune_powers = -1;
  uint32_t tune_stages = 0, tune_gbuf = 0;

  std::vector<ChannelBlockStore> cbs;
  DevBuf staging, run_src_dev, run_len_dev;
  // host copies of what run_src_dev / run_len_dev hold
  std::vector<uint32_t> staged_run_src, staged_run_len;
  // SetRegularBlock's baseline order for the antenna arrays it was made for
  // (every channel block and interval of one layout repeats them)
  std::vector<uint32_t> order_a1, order_a2, order_bl, order_ant;
  std::vector<uint8_t> order_flip;
  DevBuf predict_in;  // station UVW, sky, frequencies and antennas of a predict
  DevBuf predict_table;  // station phasors of a predict (station_phasor_kernel)
  // Pinned host image of predict_in (one copy per predict), reusable once
  // the copy recorded in predict_copied has run.
  void* predict_host = nullptr;
  size_t predict_host_bytes = 0;
  cudaEvent_t predict_copied = nullptr;
  // Pinned image of the small inputs of a synchronous call
  // (ddsolve_correct_and_subtract), free again when the call returns.
  void* small_host = nullptr;
  size_t small_host_bytes = 0;
  // Per channel block, for the sky path (ddsolve_set_channel_block_regular_sky),
  // whose uploads overlap a solve of another context: the predict's device
  // inputs and their pinned image (consecutive blocks do not wait for each
  // other's copies), and the data's staging buffer, filled on copy_stream so
  // that the copies run while the kernels of the upload wait for the solve.
  cudaStream_t copy_stream = nullptr;
  std::vector<DevBuf> blk_predict_in, blk_data_stage;
  std::vector<void*> blk_predict_host;
  std::vector<size_t> blk_predict_host_bytes;
  std::vector<cudaEvent_t> blk_predict_copied, blk_data_copied, blk_packed;
  DevBuf raw_in;      // DP3-layout interval buffers (ddsolve_set_interval_buffers)
  DevBuf raw_model;   // the 4-correlation predicted model of one block
  DevBuf cs_out;      // outputs of ddsolve_correct_and_subtract bound for the host

  // plan
  bool plan_dirty = true;
  uint32_t ng = 1, dmax = 1;
  StreamFn stream_fn = nullptr;
  size_t stream_smem = 0;
  // pipelined path (pipe_kernel): chosen when eligible
  bool use_pipe = false;
  const void* pipe_fn = nullptr;
  size_t pipe_smem = 0;
  uint32_t pipe_stages = 0, acc_stride = 0, gain_stride = 0;
  uint32_t pipe_ng = 1;  // lanes per run of the chosen pipe_kernel
  DevBuf d_cb_done /* new non-finite flags */, d_cb_flag, d_cb_avg, d_counters;
  DevBuf d_frags, d_cta_frag_off, d_tables, d_tab_cb, d_tab_sol, d_tab_off, d_tab_ent;
  uint32_t n_tables = 0, table_f2 = 0, owner_groups = 1, n_gbuf = 2;
  uint32_t off_acc = 0, off_gtab = 0, off_stg = 0, off_cnt = 0, off_off = 0,
           off_pair = 0, off_ent = 0, off_wsum = 0, off_stages = 0;
  uint32_t n_ctas = 0, n_visits = 0, fin_blocks = 0;
  // precomputed model powers (pipe_kernel), refreshed after every upload
  bool use_powers = false, powers_dirty = true;
  uint32_t n_power_tiles = 0, power_floats = 0;
  DevBuf d_power_tiles, d_powers;
  DevBuf d_slabs, d_visits, d_cta_off, d_slab_sol, d_partials, d_fin_off,
      d_fin_visits, d_fin_first, d_dir_of_sub, d_block_sum, d_block_cnt;
  bool fin_ranges = false;  // pipe plan: every finalisation list is a visit range
  // solver state
  DevBuf d_sol, d_next, d_state, d_nonfinite, d_mags, d_settings;
  DevBuf d_chain;  // outputs of ddsolve_perform_iterations
  // Device constraints (ddsolve_add_*_constraint), applied in the order they
  // were added between the step-only and the assignment passes of every
  // solve iteration.
  struct DeviceConstraint {
    int kind = 0;         // DDSOLVE_CONSTRAINT_*
    DevBuf buf;           // the constraint's device arrays, one allocation
    size_t off[6] = {};   // byte offsets of those arrays in buf
    uint32_t n_sets = 0;  // antenna constraint
    uint32_t per_sub_weights = 0;
    double bandwidth = 0.0;
    int32_t truncate = 0;
  };
  std::vector<DeviceConstraint> constraints;
  DevBuf d_cons, d_ref_ant;  // second next-solutions buffer; reference antennas
  // full-Jones plan: first global run of each slab, per (cb, antenna,
  // sub-solution) item the list of its partial slots
  DevBuf d_fj_run_start, d_fj_list_off, d_fj_list_ent, d_fj_resid, d_fj_resid_off;
  uint32_t fj_n_slabs = 0, fj_n_runs = 0, fj_blocks = 0, fj_parts = 1, fj_resid_parts = 1;
  // independent solution intervals (ddsolve_set_intervals): interval g owns
  // channel blocks [group_first_cb[g], group_first_cb[g + 1])
  uint32_t n_groups = 1;
  uint32_t graph_unroll = 4;  // pipe_kernel launches per graph loop test
  std::vector<uint32_t> group_first_cb;
  uint32_t mags_stride = 1;
  DevBuf d_block_group, d_block_item0, d_block_item_end, d_group_blocks, d_cb_group;
  DevBuf d_group_cb;  // pipe plan: first channel block of each interval, and n_cb
  // graph
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  cudaGraphConditionalHandle handle = 0;
  bool graph_ok = false;
  uint64_t last_launches = 0;
  uint64_t last_predict_launches = 0;  // predict launches (phasor table + model) since creation
  // Pinned host staging of the per-call read-backs (error counters, loop
  // state, step magnitudes), copied before the call's single synchronization.
  struct HostStage {
    uint32_t counters[4];
    LoopState ls;
    double mags[1];  // [mags_cap]
  };
  HostStage* h_stage = nullptr;
  size_t mags_cap = 0;

  int Fail(int code, const std::string& msg) {
    err = msg;
    return code;
  }
  ~ddsolve_ctx() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    if (stream) cudaStreamDestroy(stream);
    if (h_stage) cudaFreeHost(h_stage);
    if (predict_copied) cudaEventDestroy(predict_copied);
    if (predict_host) cudaFreeHost(predict_host);
    if (small_host) cudaFreeHost(small_host);
    for (void* h : blk_predict_host)
      if (h) cudaFreeHost(h);
    for (auto* evs : {&blk_predict_copied, &blk_data_copied, &blk_packed})
      for (cudaEvent_t ev : *evs)
        if (ev) cudaEventDestroy(ev);
    if (copy_stream) cudaStreamDestroy(copy_stream);
  }
  // A pinned image of at least n bytes that is free to overwrite: the copy
  // recorded in `ev` (created on first use) has run.
  static cudaError_t ReservePinned(void*& buf, size_t& bytes, cudaEvent_t& ev, size_t n) {
    if (ev) {
      const cudaError_t e = cudaEventSynchronize(ev);
      if (e != cudaSuccess) return e;
    } else {
      const cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
    if (buf && n <= bytes) return cudaSuccess;
    if (buf) cudaFreeHost(buf);
    buf = nullptr;
    bytes = 0;
    const cudaError_t e = cudaMallocHost(&buf, std::max<size_t>(n, 1 << 16));
    if (e == cudaSuccess) bytes = std::max<size_t>(n, 1 << 16);
    return e;
  }
  static cudaError_t EnsureEvent(cudaEvent_t& ev) {
    return ev ? cudaSuccess : cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
  }
  // The pinned image of small inputs, at least n bytes.
  cudaError_t ReserveSmallHost(size_t n) {
    if (small_host && n <= small_host_bytes) return cudaSuccess;
    if (small_host) cudaFreeHost(small_host);
    small_host = nullptr;
    small_host_bytes = 0;
    const cudaError_t e = cudaMallocHost(&small_host, std::max<size_t>(n, 1 << 16));
    if (e == cudaSuccess) small_host_bytes = std::max<size_t>(n, 1 << 16);
    return e;
  }
  // The pinned predict image, at least n bytes, free to overwrite.
  cudaError_t ReservePredictHost(size_t n) {
    if (predict_copied) {
      const cudaError_t e = cudaEventSynchronize(predict_copied);
      if (e != cudaSuccess) return e;
    } else {
      const cudaError_t e = cudaEventCreateWithFlags(&predict_copied, cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
    if (predict_host && n <= predict_host_bytes) return cudaSuccess;
    if (predict_host) cudaFreeHost(predict_host);
    predict_host = nullptr;
    predict_host_bytes = 0;
    const cudaError_t e = cudaMallocHost(&predict_host, std::max<size_t>(n, 1 << 16));
    if (e == cudaSuccess) predict_host_bytes = std::max<size_t>(n, 1 << 16);
    return e;
  }
  cudaError_t ReserveStage(size_t n_mags) {
    if (h_stage && n_mags <= mags_cap) return cudaSuccess;
    if (h_stage) cudaFreeHost(h_stage);
    h_stage = nullptr;
    const size_t cap = std::max<size_t>(n_mags, 64);
    void* p = nullptr;
    const cudaError_t e = cudaMallocHost(&p, sizeof(HostStage) + cap * sizeof(double));
    if (e != cudaSuccess) return e;
    h_stage = static_cast<HostStage*>(p);
    mags_cap = cap;
    return cudaSuccess;
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
  int ng = 1;  // pipe_kernel: lanes per run
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

// Registry of pipelined-kernel instantiations keyed by (ncorr, npol, dmax).
template <int NC, int NP, int DM>
constexpr KernelEntry PipeEntry() {
  return KernelEntry{NC, NP, DM,
                     reinterpret_cast<const void*>(&pipe_kernel<NC, NP, DM, 1>), 1};
}

// Lane-group variant: up to 4 * DM directions.
template <int NC, int NP, int DM>
constexpr KernelEntry PipeEntry4() {
  return KernelEntry{NC, NP, DM,
                     reinterpret_cast<const void*>(&pipe_kernel<NC, NP, DM, 4>), 4};
}

const std::vector<KernelEntry>& PipeKernels() {
  static const std::vector<KernelEntry> k = {
      // One instantiation per direction count: a padded direction would
      // cost a full share of the row loop, and exact counts need no guards.
      PipeEntry<2, 2, 1>(), PipeEntry<2, 2, 2>(), PipeEntry<2, 2, 3>(),
      PipeEntry<2, 2, 4>(), PipeEntry<2, 2, 5>(), PipeEntry<2, 2, 6>(),
      PipeEntry<2, 2, 7>(), PipeEntry<2, 2, 8>(), PipeEntry<2, 2, 9>(),
      PipeEntry<2, 2, 10>(), PipeEntry<2, 2, 11>(), PipeEntry<2, 2, 12>(),
      PipeEntry<2, 1, 1>(), PipeEntry<2, 1, 2>(), PipeEntry<2, 1, 3>(),
      PipeEntry<2, 1, 4>(), PipeEntry<2, 1, 5>(), PipeEntry<2, 1, 6>(),
      PipeEntry<2, 1, 7>(), PipeEntry<2, 1, 8>(), PipeEntry<2, 1, 9>(),
      PipeEntry<2, 1, 10>(), PipeEntry<2, 1, 11>(), PipeEntry<2, 1, 12>(),
      PipeEntry<4, 2, 1>(), PipeEntry<4, 2, 2>(), PipeEntry<4, 2, 3>(),
      PipeEntry<4, 2, 4>(),
      PipeEntry<4, 1, 1>(), PipeEntry<4, 1, 2>(), PipeEntry<4, 1, 3>(),
      PipeEntry<4, 1, 4>(),
      // 13..48 directions (XX/YY): four lanes per run
      PipeEntry4<2, 2, 4>(), PipeEntry4<2, 2, 6>(), PipeEntry4<2, 2, 8>(),
      PipeEntry4<2, 2, 10>(), PipeEntry4<2, 2, 12>(),
      PipeEntry4<2, 1, 4>(), PipeEntry4<2, 1, 6>(), PipeEntry4<2, 1, 8>(),
      PipeEntry4<2, 1, 10>(), PipeEntry4<2, 1, 12>(),
  };
  return k;
}

const KernelEntry* FindPipeKernel(int ncorr, int npol, int n_dir) {
  const KernelEntry* best = nullptr;
  for (const KernelEntry& e : PipeKernels())
    if (e.ng == 1 && e.ncorr == ncorr && e.npol == npol && e.dmax == n_dir) best = &e;
  if (best || std::getenv("DDSOLVE_NO_LANE_GROUPS")) return best;
  // more directions than one lane holds: four lanes per run, the smallest
  // instantiation with 4 * dmax >= n_dir (eight lanes per run with
  // half-width tiles measured slower on the 40-direction interval: 418 us
  // against 338 us per pass)
  for (const KernelEntry& e : PipeKernels())
    if (e.ng == 4 && e.ncorr == ncorr && e.npol == npol && 4 * e.dmax >= n_dir &&
        (!best || e.dmax < best->dmax))
      best = &e;
  return best;
}

uint32_t OddAtLeast(uint32_t x) { return x | 1u; }

// Strides of pipe_kernel's accumulator rows (floats; 4 mod 8, see AccAdd)
// and gain-table rows (float2; 2 mod 4 for two polarizations, see
// LoadGains, else odd).
uint32_t PipeAccStride(uint32_t n_dir, uint32_t n_pol) {
  uint32_t s = n_dir * n_pol * 3;
  while (s % 8 != 4) ++s;
  return s;
}
uint32_t PipeGainStride(uint32_t n_dir, uint32_t n_pol) {
  uint32_t s = n_dir * n_pol;
  if (n_pol == 2) {
    while (s % 4 != 2) ++s;
    return s;
  }
  return OddAtLeast(s);
}

// One pipeline stage of pipe_kernel: the fragment's run antennas (first row
// only), then one row of data and of every direction's model.
size_t PipeStageBytes(const ddsolve_ctx* ctx) {
  const size_t runs = kPipeRuns / ctx->pipe_ng;
  return runs * 4 + size_t(1 + ctx->n_dir) * runs * ctx->elem_bytes;
}

// Shared memory of pipe_kernel for `stages` stages, with one gain-table
// buffer and the scratch of the sorted tile reduction (the layout is fixed in
// BuildPipePlan, which adds the second gain-table buffer when it fits).
size_t PipeSmemBytes(const ddsolve_ctx* ctx, uint32_t stages, uint32_t acc_stride,
                     uint32_t gain_stride) {
  auto align = [](size_t x, size_t a) { return (x + a - 1) / a * a; };
  const size_t n_ant4 = align(ctx->n_ant, 4);
  const size_t table_f2 = (size_t(ctx->n_ant) * gain_stride + 1) & ~size_t(1);
  size_t off = align(256 + size_t(kPipeRuns) * 12, 16);
  off += align(size_t(ctx->n_ant) * acc_stride * 4, 16);
  off += table_f2 * 8;
  if (ctx->pipe_ng == 1)  // the sorted tile reduction (one run per lane only)
    off += size_t(3) * ctx->n_corr * ctx->n_dir * kPipeRuns * 4 + 2 * n_ant4 * 4 +
           size_t(kPipeRuns) * 4 + size_t(kPipeRuns) * 4;
  off += 128;
  off = align(off, 128);
  return off + size_t(stages) * PipeStageBytes(ctx);
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
        (nc == 2 && np == 1) || (nc == 4 && np == 1) || (nc == 4 && np == 4)))
    return DDSOLVE_E_UNSUPPORTED;
  for (uint32_t d = 0; d < dims->n_directions; ++d)
    if (dims->n_solutions_per_direction[d] == 0) return DDSOLVE_E_INVALID;
  return DDSOLVE_OK;
}

// Runs per tile of the packed layout: the tile of the pipelined kernel that
// the context's correlations and direction count select (equal tiles of at
// most kPipeRuns / NG runs, a multiple of 4, so that a tile's run antennas
// start on a 16-byte boundary; a short remainder tile would stream its rows
// at a fraction of the bytes per pipeline stage).
uint32_t LayoutTileRuns(const ddsolve_ctx* ctx, uint32_t R) {
  const KernelEntry* e = FindPipeKernel(int(ctx->n_corr), int(ctx->n_pol), int(ctx->n_dir));
  const uint32_t max_runs = kPipeRuns / (e ? uint32_t(e->ng) : 1u);
  if (R == 0) return max_runs;
  const uint32_t n_tiles = (R + max_runs - 1) / max_runs;
  return ((R + n_tiles - 1) / n_tiles + 3u) & ~3u;
}

// A point-source predict of one regular channel block (predict_kernel).
struct PredictJob {
  uint32_t n_times, n_bl, L;
  const double* freq;  // [L]
  const double* uvw;   // [n_times][n_ant][3]
  const uint32_t* a1;  // [n_bl]
  const uint32_t* a2;
  const ddsolve_sky_direction* sky;  // [n_dir]
};

constexpr size_t kPredictMaxSmem = 200 * 1024;

// Host-side checks of a predict job; DDSOLVE_OK or a status with the message.
int CheckPredictJob(ddsolve_ctx* ctx, const PredictJob& j) {
  if (!j.freq || !j.uvw || !j.a1 || !j.a2 || !j.sky)
    return ctx->Fail(DDSOLVE_E_INVALID, "predict: NULL pointer");
  uint32_t max_src = 0;
  for (uint32_t d = 0; d < ctx->n_dir; ++d) {
    if (j.sky[d].n_sources && (!j.sky[d].lmn || !j.sky[d].stokes))
      return ctx->Fail(DDSOLVE_E_INVALID, "predict: NULL source arrays");
    max_src = std::max(max_src, j.sky[d].n_sources);
  }
  const size_t smem = size_t(max_src) * 8 * sizeof(double);
  if (smem > kPredictMaxSmem)
    return ctx->Fail(DDSOLVE_E_UNSUPPORTED,
                     "predict: sources x 8 doubles exceed 200 KiB of shared memory (more than "
                     "3200 sources in one direction)");
  for (uint32_t b = 0; b < j.n_bl; ++b)
    if (j.a1[b] >= ctx->n_ant || j.a2[b] >= ctx->n_ant)
      return ctx->Fail(DDSOLVE_E_INVALID, "predict: antenna index out of range");
  return DDSOLVE_OK;
}

// A packed channel block the predict writes into directly (predict_kernel's
// packed mode): its runs' oriented antennas on the device, its packed
// visibilities, and per time step the slab element and row of the step.
struct PackedTarget {
  const uint32_t* run_ant;
  float2* vis;
  std::vector<uint64_t> t_elem;
  std::vector<uint32_t> t_row;
  uint32_t W;
};

// Uploads the job's inputs and launches predict_kernel into `model` (device
// memory, [n_dir][n_times * n_bl * L][n_corr]) on the context stream, or
// into the packed block `packed`; n_corr is the context's unless n_corr_out
// (1, 2 or 4) is given.
int LaunchPredict(ddsolve_ctx* ctx, const PredictJob& j, float2* model, uint32_t n_corr_out = 0,
                  const PackedTarget* packed = nullptr, int blk = -1) {
  const uint32_t nc = n_corr_out ? n_corr_out : ctx->n_corr;
  uint32_t n_src = 0, max_src = 0;
  std::vector<uint32_t> off(ctx->n_dir + 1, 0);
  for (uint32_t d = 0; d < ctx->n_dir; ++d) {
    off[d] = n_src;
    n_src += j.sky[d].n_sources;
    max_src = std::max(max_src, j.sky[d].n_sources);
  }
  off[ctx->n_dir] = n_src;
  std::vector<double> src(size_t(n_src) * 8, 0.0);
  for (uint32_t d = 0; d < ctx->n_dir; ++d)
    for (uint32_t s = 0; s < j.sky[d].n_sources; ++s) {
      double* o = &src[(size_t(off[d]) + s) * 8];
      o[0] = j.sky[d].lmn[3 * s];
      o[1] = j.sky[d].lmn[3 * s + 1];
      o[2] = j.sky[d].lmn[3 * s + 2] - 1.0;  // n - 1, as Simulator.cc:486 uses it
      for (int k = 0; k < 4; ++k) o[3 + k] = j.sky[d].stokes[4 * s + k];
    }
  // Evenly spaced channels (to 1e-6 Hz) use the phasor recurrence.
  double df = j.L > 1 ? (j.freq[j.L - 1] - j.freq[0]) / (j.L - 1) : 0.0;
  int uniform = j.L > 1;
  for (uint32_t c = 0; c < j.L && uniform; ++c)
    uniform = std::abs(j.freq[c] - (j.freq[0] + c * df)) <= 1e-6;
  auto align = [](size_t x) { return (x + 255) / 256 * 256; };
  const size_t b_uvw = size_t(j.n_times) * ctx->n_ant * 3 * 8, b_src = src.size() * 8 + 8;
  const size_t b_off = off.size() * 4, b_f = size_t(j.L) * 8, b_a = size_t(j.n_bl) * 4;
  const size_t o_src = align(b_uvw), o_off = o_src + align(b_src), o_f = o_off + align(b_off);
  const size_t b_te = packed ? size_t(j.n_times) * 8 : 0, b_tr = packed ? size_t(j.n_times) * 4 : 0;
  const size_t o_a1 = o_f + align(b_f), o_a2 = o_a1 + align(b_a), o_te = o_a2 + align(b_a);
  const size_t o_tr = o_te + align(b_te), o_up = o_tr + align(b_tr);
  const size_t b_up = size_t(ctx->n_dir) * 4, total = o_up + align(b_up);
  std::vector<uint32_t> unpol(ctx->n_dir, 1u);
  for (uint32_t d = 0; d < ctx->n_dir; ++d)
    for (uint32_t s = 0; s < j.sky[d].n_sources && unpol[d]; ++s)
      for (int k = 1; k < 4; ++k)
        if (j.sky[d].stokes[4 * s + k] != 0.0) unpol[d] = 0u;
  // the device inputs and their pinned image: the context's, or channel
  // block blk's own (blocks then do not wait for each other's copies)
  DevBuf& pin = blk >= 0 ? ctx->blk_predict_in[blk] : ctx->predict_in;
  cudaEvent_t& copied = blk >= 0 ? ctx->blk_predict_copied[blk] : ctx->predict_copied;
  DDS_CHECK_CUDA(ctx, pin.Reserve(total));
  char* base = pin.as<char>();
  // Host inputs go through one pinned image and one copy (each small copy
  // from pageable memory costs a staged transfer of its own); inputs in
  // device memory are copied device to device.
  auto on_host = [](const void* ptr) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, ptr) != cudaSuccess) {
      cudaGetLastError();
      return true;
    }
    return a.type == cudaMemoryTypeUnregistered || a.type == cudaMemoryTypeHost;
  };
  if (blk >= 0)
    DDS_CHECK_CUDA(ctx, ddsolve_ctx::ReservePinned(ctx->blk_predict_host[blk],
                                                   ctx->blk_predict_host_bytes[blk], copied,
                                                   total));
  else
    DDS_CHECK_CUDA(ctx, ctx->ReservePredictHost(total));
  char* host = static_cast<char*>(blk >= 0 ? ctx->blk_predict_host[blk] : ctx->predict_host);
  struct Piece {
    const void* src;
    size_t off, bytes;
  };
  constexpr int kPieces = 9;
  const Piece pieces[kPieces] = {
      {j.uvw, 0, b_uvw},          {src.data(), o_src, src.size() * 8},
      {off.data(), o_off, b_off}, {j.freq, o_f, b_f},
      {j.a1, o_a1, b_a},          {j.a2, o_a2, b_a},
      {packed ? static_cast<const void*>(packed->t_elem.data()) : nullptr, o_te, b_te},
      {packed ? static_cast<const void*>(packed->t_row.data()) : nullptr, o_tr, b_tr},
      {unpol.data(), o_up, b_up}};
  bool device_piece[kPieces];
  for (int k = 0; k < kPieces; ++k) {
    const Piece& pc = pieces[k];
    device_piece[k] = pc.bytes > 0 && !on_host(pc.src);
    if (pc.bytes > 0 && !device_piece[k]) std::memcpy(host + pc.off, pc.src, pc.bytes);
  }
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(base, host, total, cudaMemcpyHostToDevice, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaEventRecord(copied, ctx->stream));
  for (int k = 0; k < kPieces; ++k)  // after the image, which they overwrite
    if (device_piece[k])
      DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(base + pieces[k].off, pieces[k].src, pieces[k].bytes,
                                          cudaMemcpyDeviceToDevice, ctx->stream));
  // station phasors of every (time, direction, source, station)
  const uint32_t chunk = uint32_t(kPredictChunk) / nc;
  const uint32_t n_slots = uniform ? (j.L + chunk - 1) / chunk + 1 : j.L;
  const size_t table_entries =
      size_t(j.n_times) * ctx->n_dir * std::max(max_src, 1u) * ctx->n_ant * n_slots;
  DDS_CHECK_CUDA(ctx, ctx->predict_table.Reserve(table_entries * sizeof(double2)));
  PhasorParams ph;
  ph.uvw = reinterpret_cast<const double*>(base);
  ph.src = reinterpret_cast<const double*>(base + o_src);
  ph.src_off = reinterpret_cast<const uint32_t*>(base + o_off);
  ph.freq = reinterpret_cast<const double*>(base + o_f);
  ph.table = ctx->predict_table.as<double2>();
  ph.n_times = j.n_times;
  ph.n_ant = ctx->n_ant;
  ph.n_dir = ctx->n_dir;
  ph.max_src = max_src;
  ph.L = j.L;
  ph.n_slots = n_slots;
  ph.chunk = chunk;
  ph.uniform = uniform;
  ph.df = df;
  if (max_src > 0) {
    const dim3 pgrid((ctx->n_ant + kPredictThreads - 1) / kPredictThreads, j.n_times,
                     std::min<uint32_t>(ctx->n_dir * max_src, 65535u));
    station_phasor_kernel<<<pgrid, kPredictThreads, 0, ctx->stream>>>(ph);
    DDS_CHECK_CUDA(ctx, cudaGetLastError());
  }
  PredictParams p;
  p.src = reinterpret_cast<const double*>(base + o_src);
  p.src_off = reinterpret_cast<const uint32_t*>(base + o_off);
  p.table = ctx->predict_table.as<double2>();
  p.a1 = reinterpret_cast<const uint32_t*>(base + o_a1);
  p.a2 = reinterpret_cast<const uint32_t*>(base + o_a2);
  p.model = model;
  p.n_times = j.n_times;
  p.n_bl = j.n_bl;
  p.L = j.L;
  p.n_ant = ctx->n_ant;
  p.n_dir = ctx->n_dir;
  p.max_src = max_src;
  p.n_slots = n_slots;
  p.uniform = uniform;
  p.run_ant = packed ? packed->run_ant : nullptr;
  p.vis = packed ? packed->vis : nullptr;
  p.t_elem = reinterpret_cast<const uint64_t*>(base + o_te);
  p.t_row = reinterpret_cast<const uint32_t*>(base + o_tr);
  p.W = packed ? packed->W : 0;
  p.unpol = reinterpret_cast<const uint32_t*>(base + o_up);
  const size_t smem = size_t(max_src) * 8 * sizeof(double);
  const dim3 grid((j.n_bl + kPredictThreads - 1) / kPredictThreads, j.n_times, ctx->n_dir);
  const bool all_unpol = std::all_of(unpol.begin(), unpol.end(), [](uint32_t u) { return u != 0; });
  const void* fn =
      nc == 1 ? reinterpret_cast<const void*>(predict_kernel<1, true>)
      : nc == 2
          ? (all_unpol ? reinterpret_cast<const void*>(predict_kernel<2, true>)
                       : reinterpret_cast<const void*>(predict_kernel<2, false>))
          : (all_unpol ? reinterpret_cast<const void*>(predict_kernel<4, true>)
                       : reinterpret_cast<const void*>(predict_kernel<4, false>));
  DDS_CHECK_CUDA(ctx, cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(kPredictMaxSmem)));
  void* args[] = {&p};
  DDS_CHECK_CUDA(ctx, cudaLaunchKernel(fn, grid, dim3(kPredictThreads), args, smem,
                                       ctx->stream));
  ctx->last_predict_launches += max_src > 0 ? 2 : 1;
  return DDSOLVE_OK;
}

// Fills the staging buffer of one channel block (reference layout: data
// [n_vis][n_corr], then model [n_dir][n_vis][n_corr]) on the context stream.
using StageFn = std::function<int(char* staging)>;

// Stages a block and packs it into slabs. `stage` writes the reference-layout
// block into the staging buffer: copies of host or device arrays
// (StageCopy), a copy of the data plus the GPU predict of the model, or the
// GPU weighting of raw buffers.
int UploadAndPack(ddsolve_ctx* ctx, ChannelBlockStore& cb, const StageFn& stage,
                  bool models_in_place = false, int blk = -1) {
  const size_t E = ctx->elem_bytes;
  const size_t src_bytes = size_t(cb.n_vis) * E * (1 + ctx->n_dir);
  if (blk < 0) DDS_CHECK_CUDA(ctx, ctx->staging.Reserve(src_bytes));  // else the block's own
  cb.vis.realloc_flag = cb.run_ant_dev.realloc_flag = false;
  DDS_CHECK_CUDA(ctx, cb.vis.Reserve(cb.n_elems * E * (1 + ctx->n_dir)));
  DDS_CHECK_CUDA(ctx, cb.run_ant_dev.Reserve(cb.run_ant.size() * 4));
  DDS_CHECK_CUDA(ctx, ctx->run_src_dev.Reserve(cb.run_src.size() * 4));
  DDS_CHECK_CUDA(ctx, ctx->run_len_dev.Reserve(cb.run_len.size() * 4));
  std::vector<PackSlab> ps(cb.slabs.size());
  for (size_t i = 0; i < cb.slabs.size(); ++i) {
    HostSlab& s = cb.slabs[i];
    s.W = LayoutTileRuns(ctx, s.R);
    ps[i] = PackSlab{s.elem_off, s.src_base, s.tstride, s.T, s.L, s.R, s.run_off, s.W};
  }
  char* st = ctx->staging.as<char>();
  // The run arrays are copied only when they changed: a copy from pageable
  // memory waits for the stream, which would hold this host thread behind
  // the kernels already queued (the previous block's predict and pack, or a
  // solve of the other context). Consecutive blocks and intervals of one
  // layout repeat them. The run antennas go first: a stage that writes the
  // packed block directly reads them.
  if (cb.run_ant_dev.realloc_flag || !cb.set || cb.run_ant != cb.prev_run_ant)
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(cb.run_ant_dev.ptr, cb.run_ant.data(),
                                        cb.run_ant.size() * 4,
                                        cudaMemcpyHostToDevice, ctx->stream));
  if (cb.n_vis) {
    const int rc = stage(st);
    if (rc != DDSOLVE_OK) return rc;
  }
  if (ctx->run_src_dev.realloc_flag || ctx->run_len_dev.realloc_flag ||
      cb.run_src != ctx->staged_run_src || cb.run_len != ctx->staged_run_len) {
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->run_src_dev.ptr, cb.run_src.data(),
                                        cb.run_src.size() * 4,
                                        cudaMemcpyHostToDevice, ctx->stream));
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->run_len_dev.ptr, cb.run_len.data(),
                                        cb.run_len.size() * 4,
                                        cudaMemcpyHostToDevice, ctx->stream));
    ctx->staged_run_src = cb.run_src;
    ctx->staged_run_len = cb.run_len;
  }
  ctx->run_src_dev.realloc_flag = ctx->run_len_dev.realloc_flag = false;
  for (size_t i = 0; i < cb.slabs.size(); ++i) {
    const uint64_t tlr = uint64_t(cb.slabs[i].T) * cb.slabs[i].L * cb.slabs[i].R;
    if (tlr == 0) continue;
    const uint32_t blocks =
        uint32_t(std::min<uint64_t>((tlr + 255) / 256, uint64_t(ctx->n_sm) * 8));
    // the sky path stages the data in the block's own buffer (StagePredict)
    const float2* src_d = blk >= 0 ? ctx->blk_data_stage[blk].as<float2>()
                                   : reinterpret_cast<const float2*>(st);
    const float2* src_m = reinterpret_cast<const float2*>(st + size_t(cb.n_vis) * E);
    float2* dst = cb.vis.as<float2>();
    if (E == 8)
      pack_kernel<1><<<blocks, 256, 0, ctx->stream>>>(
          ps[i], ctx->run_src_dev.as<uint32_t>(),
          ctx->run_len_dev.as<uint32_t>(), src_d, src_m, cb.n_vis, ctx->n_dir,
          models_in_place ? 0u : ctx->n_dir, dst);
    else if (E == 16)
      pack_kernel<2><<<blocks, 256, 0, ctx->stream>>>(
          ps[i], ctx->run_src_dev.as<uint32_t>(),
          ctx->run_len_dev.as<uint32_t>(), src_d, src_m, cb.n_vis, ctx->n_dir,
          models_in_place ? 0u : ctx->n_dir, dst);
    else
      pack_kernel<4><<<blocks, 256, 0, ctx->stream>>>(
          ps[i], ctx->run_src_dev.as<uint32_t>(),
          ctx->run_len_dev.as<uint32_t>(), src_d, src_m, cb.n_vis, ctx->n_dir,
          models_in_place ? 0u : ctx->n_dir, dst);
    DDS_CHECK_CUDA(ctx, cudaGetLastError());
  }
  if (blk >= 0) {  // the block's data staging may be refilled after these packs
    DDS_CHECK_CUDA(ctx, ddsolve_ctx::EnsureEvent(ctx->blk_packed[blk]));
    DDS_CHECK_CUDA(ctx, cudaEventRecord(ctx->blk_packed[blk], ctx->stream));
  }
  // The staging and run arrays are reused by the next upload: keep the
  // stream order (a later upload's copies follow these kernels).
  const bool moved =
      cb.vis.realloc_flag || cb.run_ant_dev.realloc_flag;
  if (!cb.set || moved || !SameLayout(cb.slabs, cb.prev_slabs) ||
      cb.run_ant != cb.prev_run_ant) {
    ctx->plan_dirty = true;
    cb.prev_slabs = cb.slabs;
    cb.prev_run_ant = cb.run_ant;
  }
  cb.set = true;
  ctx->powers_dirty = true;
  return DDSOLVE_OK;
}

// Stager of data and model arrays in the reference layout (host or device).
StageFn StageCopy(ddsolve_ctx* ctx, const ChannelBlockStore& cb, const float* data,
                  const float* model) {
  const size_t n = size_t(cb.n_vis) * ctx->elem_bytes;
  return [ctx, n, data, model](char* st) {
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(st, data, n, cudaMemcpyDefault, ctx->stream));
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(st + n, model, n * ctx->n_dir, cudaMemcpyDefault,
                                        ctx->stream));
    return DDSOLVE_OK;
  };
}

// Stager of the data array plus the GPU predict of the model, written
// straight into the block's packed layout (UploadAndPack then packs the data
// only): every slab of a regular block holds all its runs for a range of
// time steps.
StageFn StagePredict(ddsolve_ctx* ctx, const ChannelBlockStore& cb, const float* data,
                     const PredictJob& job, uint32_t cbi) {
  const size_t n = size_t(cb.n_vis) * ctx->elem_bytes;
  return [ctx, n, data, job, &cb, cbi](char*) {
    // the data into the block's own staging on the copy stream, after the
    // previous pack of this block has read it; the context stream waits for
    // the copy before the pack
    DevBuf& ds = ctx->blk_data_stage[cbi];
    DDS_CHECK_CUDA(ctx, ds.Reserve(n));
    if (ctx->blk_packed[cbi])
      DDS_CHECK_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_stream, ctx->blk_packed[cbi], 0));
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ds.ptr, data, n, cudaMemcpyDefault, ctx->copy_stream));
    DDS_CHECK_CUDA(ctx, ddsolve_ctx::EnsureEvent(ctx->blk_data_copied[cbi]));
    DDS_CHECK_CUDA(ctx, cudaEventRecord(ctx->blk_data_copied[cbi], ctx->copy_stream));
    DDS_CHECK_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->blk_data_copied[cbi], 0));
    PackedTarget t;
    t.run_ant = cb.run_ant_dev.as<uint32_t>();
    t.vis = cb.vis.as<float2>();
    t.W = cb.slabs.empty() ? 0u : cb.slabs.front().W;
    t.t_elem.resize(job.n_times);
    t.t_row.resize(job.n_times);
    uint32_t t0 = 0;
    for (const HostSlab& s : cb.slabs) {
      if (s.R != job.n_bl || s.L != job.L || s.W != t.W || s.run_off != 0)
        return ctx->Fail(DDSOLVE_E_INVALID, "predict: block is not a regular layout");
      for (uint32_t k = 0; k < s.T && t0 + k < job.n_times; ++k) {
        t.t_elem[t0 + k] = uint64_t(1 + ctx->n_dir) * s.elem_off;
        t.t_row[t0 + k] = k * s.L;
      }
      t0 += s.T;
    }
    if (t0 != job.n_times) return ctx->Fail(DDSOLVE_E_INVALID, "predict: time steps do not match");
    return LaunchPredict(ctx, job, nullptr, 0, &t, int(cbi));
  };
}

constexpr int kPlanNoPipe = -1;  // BuildPipePlan: use the stream_kernel path

// Plan of the pipelined path: tiles of up to kPipeRuns runs (flagged direct
// when their first antennas are distinct and their second antennas are
// distinct), split along their (time, channel) rows into fragments so that
// every CTA streams the same weight of rows; visits (one partial slot each);
// gain tables (one per channel block and solution-index vector) with the
// lists the finalisation uses to refresh them; shared-memory layout.
int BuildPipePlan(ddsolve_ctx* ctx, std::vector<SlabDesc>& descs,
                  const std::vector<uint32_t>& slab_sol, int max_optin) {
  const uint32_t n_dir = ctx->n_dir, n_ant = ctx->n_ant, n_pol = ctx->n_pol;
  // ---- gain tables ----
  std::map<std::vector<uint32_t>, uint32_t> table_ids;
  std::vector<uint32_t> tab_cb, tab_sol;
  for (SlabDesc& sd : descs) {
    std::vector<uint32_t> key(1 + n_dir);
    key[0] = sd.cb;
    for (uint32_t d = 0; d < n_dir; ++d) key[1 + d] = slab_sol[sd.sol_off + d];
    auto it = table_ids.find(key);
    if (it == table_ids.end()) {
      it = table_ids.emplace(key, uint32_t(tab_cb.size())).first;
      tab_cb.push_back(sd.cb);
      tab_sol.insert(tab_sol.end(), key.begin() + 1, key.end());
    }
    sd.table = it->second;
  }
  const uint32_t n_tables = uint32_t(tab_cb.size());
  std::vector<std::vector<uint32_t>> tlists(size_t(ctx->n_cb) * ctx->n_sub);
  for (uint32_t t = 0; t < n_tables; ++t)
    for (uint32_t d = 0; d < n_dir; ++d)
      tlists[size_t(tab_cb[t]) * ctx->n_sub + tab_sol[t * n_dir + d]].push_back((t << 8) | d);
  std::vector<uint32_t> tab_off(tlists.size() + 1, 0), tab_ent;
  for (size_t i = 0; i < tlists.size(); ++i) {
    tab_off[i] = uint32_t(tab_ent.size());
    tab_ent.insert(tab_ent.end(), tlists[i].begin(), tlists[i].end());
  }
  tab_off[tlists.size()] = uint32_t(tab_ent.size());
  const uint32_t table_f2 = (n_ant * ctx->gain_stride + 1u) & ~1u;

  // ---- tiles ----
  struct Tile {
    uint32_t slab, r0, n, rows, flags;
    uint32_t group_end[2];
  };
  std::vector<Tile> tiles;
  std::vector<uint32_t> stamp1(n_ant, 0xFFFFFFFFu), stamp2(n_ant, 0xFFFFFFFFu);
  uint32_t group_id = 0;
  bool any_sorted = false;
  for (uint32_t gi = 0; gi < descs.size(); ++gi) {
    const SlabDesc& sd = descs[gi];
    const ChannelBlockStore& cbs = ctx->cbs[sd.cb];
    const uint32_t run_off = uint32_t(sd.run_ant - cbs.run_ant_dev.as<uint32_t>());
    // The tiles of the packed layout (LayoutTileRuns): a row of a tile is
    // one bulk copy.
    const uint32_t max_runs = kPipeRuns / ctx->pipe_ng;
    const uint32_t tile_runs = sd.W;
    if (tile_runs == 0 || tile_runs > max_runs || (tile_runs & 3u)) return kPlanNoPipe;
    for (uint32_t r0 = 0; r0 < sd.R; r0 += tile_runs) {
      const uint32_t n = std::min<uint32_t>(tile_runs, sd.R - r0);
      // Greedy split into consecutive groups whose first antennas are
      // distinct and whose second antennas are distinct (a cyclic diagonal
      // of the regular layout is one such group).
      Tile t{gi, r0, n, sd.T * sd.L, 0u, {0u, 0u}};
      uint32_t n_groups = 1;
      ++group_id;
      for (uint32_t r = r0; r < r0 + n; ++r) {
        const uint32_t ap = cbs.run_ant[run_off + r];
        const uint32_t a1 = ap & 0xFFFFu, a2 = ap >> 16;
        if (stamp1[a1] == group_id || stamp2[a2] == group_id) {
          if (n_groups == kMaxGroups) {
            n_groups = kMaxGroups + 1;
            break;
          }
          const uint32_t g = n_groups - 1;
          t.group_end[g >> 2] |= (r - r0) << ((g & 3) * 8);
          ++n_groups;
          ++group_id;
        }
        stamp1[a1] = group_id;
        stamp2[a2] = group_id;
      }
      if (n_groups <= kMaxGroups) {
        const uint32_t g = n_groups - 1;
        t.group_end[g >> 2] |= n << ((g & 3) * 8);
        t.flags = kFragDirect | (n_groups << 8);
      } else {
        t.group_end[0] = t.group_end[1] = 0;
        any_sorted = true;
      }
      tiles.push_back(t);
    }
  }
  // Model powers are precomputed (one stage per tile and iteration) when the
  // tiles are deep enough in rows for that stage to cost less than the two
  // multiply-adds per row, direction and correlation it replaces.
  uint64_t run_rows = 0, n_runs_all = 0;
  for (const Tile& t : tiles) {
    run_rows += uint64_t(t.n) * t.rows;
    n_runs_all += t.n;
  }
  if (ctx->pipe_ng > 1 && any_sorted) return kPlanNoPipe;
  const bool use_powers =
      ctx->pipe_ng == 1 && !std::getenv("DDSOLVE_NO_POWERS") && n_runs_all > 0 &&
      (ctx->tune_powers == 1 || (ctx->tune_powers < 0 && run_rows >= 16 * n_runs_all));
  // ---- fragments: rows balanced over the CTAs ----
  // A row weighs its runs plus a fixed cost; a tile adds the cost of its
  // reduction, about 1.25 rows per barrier phase (two per direct group; the
  // sorted reduction as 16 phases), so that CTAs with many short tiles get
  // fewer rows.
  auto tile_cost = [](const Tile& t) {
    const uint32_t phases = (t.flags & kFragDirect) ? 2u * ((t.flags >> 8) & 0xFu) : 16u;
    return 1.25 * phases * double(t.n + 32);
  };
  uint64_t total_rows = 0;
  double total_w = 0.0;
  for (const Tile& t : tiles) {
    total_rows += t.rows;
    total_w += double(t.rows) * double(t.n + 32) + tile_cost(t);
  }
  const uint32_t max_ctas = uint32_t(ctx->n_sm);
  const uint32_t n_ctas = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>(max_ctas, total_rows)));
  std::vector<Frag> frags;
  std::vector<uint32_t> cta_off(n_ctas + 1, 0);
  {
    double cum = 0.0;
    uint32_t cur_cta = 0;
    for (const Tile& t : tiles) {
      const double w = double(t.n + 32);
      cum += tile_cost(t);
      uint32_t lo = 0;
      while (lo < t.rows) {
        // last row of this tile that stays on cur_cta
        uint32_t hi = lo;
        while (hi < t.rows) {
          const double mid = cum + (double(hi - lo) + 0.5) * w;
          uint32_t c = uint32_t(mid * n_ctas / total_w);
          if (c >= n_ctas) c = n_ctas - 1;
          if (c != cur_cta) break;
          ++hi;
        }
        if (hi > lo) {
          const uint32_t ti = uint32_t(&t - tiles.data());
          const uint32_t fl = t.flags | (use_powers && lo == 0 ? kFragPower : 0u);
          frags.push_back({t.slab, t.r0, t.n, fl, lo, hi, 0, ti,
                           {t.group_end[0], t.group_end[1]}});
          cum += double(hi - lo) * w;
          lo = hi;
        }
        if (lo < t.rows) {
          ++cur_cta;
          cta_off[cur_cta] = uint32_t(frags.size());
        }
      }
    }
    for (uint32_t c = cur_cta + 1; c <= n_ctas; ++c) cta_off[c] = uint32_t(frags.size());
    for (uint32_t c = 1; c <= n_ctas; ++c) cta_off[c] = std::max(cta_off[c], cta_off[c - 1]);
    cta_off[n_ctas] = uint32_t(frags.size());
  }
  // ---- visits ----
  uint32_t n_visits = 0;
  std::vector<uint32_t> visit_slab;
  for (uint32_t c = 0; c < n_ctas; ++c) {
    uint32_t prev_slab = 0xFFFFFFFFu;
    for (uint32_t i = cta_off[c]; i < cta_off[c + 1]; ++i) {
      if (frags[i].slab != prev_slab) {
        prev_slab = frags[i].slab;
        visit_slab.push_back(prev_slab);
        ++n_visits;
      }
      frags[i].visit = n_visits - 1;
    }
  }
  std::vector<std::vector<uint32_t>> lists(size_t(ctx->n_cb) * ctx->n_sub);
  for (uint32_t v = 0; v < n_visits; ++v) {
    const SlabDesc& sd = descs[visit_slab[v]];
    for (uint32_t d = 0; d < n_dir; ++d) {
      const uint32_t sub = slab_sol[sd.sol_off + d];
      if (sub < ctx->n_sub) lists[size_t(sd.cb) * ctx->n_sub + sub].push_back(v);
    }
  }
  std::vector<uint32_t> fin_off(lists.size() + 1, 0), fin_visits;
  for (size_t i = 0; i < lists.size(); ++i) {
    fin_off[i] = uint32_t(fin_visits.size());
    fin_visits.insert(fin_visits.end(), lists[i].begin(), lists[i].end());
  }
  fin_off[lists.size()] = uint32_t(fin_visits.size());
  // Visits are numbered in CTA order and CTAs take the slabs in order, so a
  // (channel block, sub-solution) whose slabs are consecutive has a range of
  // visits: the finalisation then needs its first visit only.
  bool ranges = true;
  std::vector<uint32_t> fin_first(lists.size(), 0);
  for (size_t i = 0; i < lists.size() && ranges; ++i) {
    for (size_t k = 1; k < lists[i].size() && ranges; ++k)
      ranges = lists[i][k] == lists[i][k - 1] + 1;
    if (!lists[i].empty()) fin_first[i] = lists[i][0];
  }
  ctx->fin_ranges = ranges;

  // ---- shared-memory layout ----
  auto align = [](size_t x, size_t a) { return (x + a - 1) / a * a; };
  size_t off = 256 + size_t(kPipeRuns) * 12;
  ctx->off_acc = uint32_t(align(off, 16));
  off = ctx->off_acc + align(size_t(n_ant) * ctx->acc_stride * 4, 16);
  ctx->off_gtab = uint32_t(off);
  // Two gain-table buffers (the next visit's table loads while the current
  // one is in use) unless that leaves fewer than four stages.
  {
    const size_t stage_b = PipeStageBytes(ctx);
    const size_t rest = size_t(3) * ctx->n_corr * n_dir * kPipeRuns * 4 + 2 * align(n_ant, 4) * 4 +
                        size_t(kPipeRuns) * 8 + 256;
    const size_t with2 = off + 2 * size_t(table_f2) * 8 + (any_sorted ? rest : 256);
    ctx->n_gbuf = (with2 + 4 * stage_b <= size_t(max_optin)) ? 2u : 1u;
    // a requested count, where two buffers still leave two stages
    if (ctx->tune_gbuf == 1) ctx->n_gbuf = 1;
    if (ctx->tune_gbuf == 2 && with2 + 2 * stage_b <= size_t(max_optin)) ctx->n_gbuf = 2;
  }
  off += size_t(ctx->n_gbuf) * table_f2 * 8;
  const size_t n_ant4 = align(n_ant, 4);
  ctx->off_stg = uint32_t(off);
  if (any_sorted) off += size_t(3) * ctx->n_corr * n_dir * kPipeRuns * 4;
  ctx->off_cnt = uint32_t(off);
  if (any_sorted) off += n_ant4 * 4;
  ctx->off_off = uint32_t(off);
  if (any_sorted) off += n_ant4 * 4;
  ctx->off_pair = uint32_t(off);
  if (any_sorted) off += size_t(kPipeRuns) * 4;
  ctx->off_ent = uint32_t(off);
  if (any_sorted) off += size_t(kPipeRuns) * 2 * 2;
  ctx->off_wsum = uint32_t(off);
  off += 32 * 4;
  ctx->off_stages = uint32_t(align(off, 128));
  const size_t stage_bytes = PipeStageBytes(ctx);
  const size_t room = size_t(max_optin) > ctx->off_stages ? size_t(max_optin) - ctx->off_stages : 0;
  uint32_t stages = uint32_t(std::min<size_t>(kPipeMaxStages, room / stage_bytes));
  if (ctx->tune_stages >= 2) stages = std::min(stages, ctx->tune_stages);
  if (stages < 2)
    return ctx->Fail(DDSOLVE_E_UNSUPPORTED, "pipelined kernel does not fit in shared memory");
  ctx->pipe_stages = stages;
  ctx->pipe_smem = ctx->off_stages + stages * stage_bytes;
  DDS_CHECK_CUDA(ctx, cudaFuncSetAttribute(ctx->pipe_fn,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(ctx->pipe_smem)));
  ctx->n_ctas = n_ctas;
  ctx->n_visits = n_visits;
  ctx->n_tables = n_tables;
  ctx->table_f2 = table_f2;
  ctx->owner_groups = std::max<uint32_t>(1u, std::min<uint32_t>(n_dir, uint32_t(kPipeRuns) / n_ant));
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
  if ((rc = upload(ctx->d_frags, frags.data(), frags.size() * sizeof(Frag)))) return rc;
  if ((rc = upload(ctx->d_cta_frag_off, cta_off.data(), cta_off.size() * 4))) return rc;
  if ((rc = upload(ctx->d_slab_sol, slab_sol.data(), slab_sol.size() * 4))) return rc;
  if ((rc = upload(ctx->d_fin_off, fin_off.data(), fin_off.size() * 4))) return rc;
  if ((rc = upload(ctx->d_fin_visits, fin_visits.data(), fin_visits.size() * 4))) return rc;
  if ((rc = upload(ctx->d_fin_first, fin_first.data(), fin_first.size() * 4))) return rc;
  if ((rc = upload(ctx->d_dir_of_sub, ctx->dir_of_sub.data(), ctx->dir_of_sub.size() * 4)))
    return rc;
  if ((rc = upload(ctx->d_tab_cb, tab_cb.data(), tab_cb.size() * 4))) return rc;
  if ((rc = upload(ctx->d_tab_sol, tab_sol.data(), tab_sol.size() * 4))) return rc;
  if ((rc = upload(ctx->d_tab_off, tab_off.data(), tab_off.size() * 4))) return rc;
  if ((rc = upload(ctx->d_tab_ent, tab_ent.data(), tab_ent.size() * 4))) return rc;
  ctx->use_powers = use_powers;
  ctx->powers_dirty = true;
  ctx->n_power_tiles = uint32_t(tiles.size());
  ctx->power_floats = n_dir * ctx->n_corr * kPipeRuns;
  if (use_powers) {
    std::vector<PowerTile> pt(tiles.size());
    for (size_t i = 0; i < tiles.size(); ++i) pt[i] = {tiles[i].slab, tiles[i].r0, tiles[i].n, 0u};
    if ((rc = upload(ctx->d_power_tiles, pt.data(), pt.size() * sizeof(PowerTile)))) return rc;
    DDS_CHECK_CUDA(ctx, ctx->d_powers.Reserve(tiles.size() * ctx->power_floats * 4));
  }
  DDS_CHECK_CUDA(ctx, ctx->d_tables.Reserve(size_t(n_tables) * table_f2 * 8));
  DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_tables.ptr, 0, size_t(n_tables) * table_f2 * 8,
                                      ctx->stream));
  DDS_CHECK_CUDA(ctx, ctx->d_partials.Reserve(
                          std::max<size_t>(1, size_t(n_visits) * n_ant * ctx->acc_stride) * 4));
  // norm partials per (interval, CTA)
  {
    const size_t n_part = std::max<size_t>(size_t(n_ctas) * ctx->n_groups, ctx->fin_blocks);
    DDS_CHECK_CUDA(ctx, ctx->d_block_sum.Reserve(n_part * 8));
    DDS_CHECK_CUDA(ctx, ctx->d_block_cnt.Reserve(n_part * 4));
    std::vector<uint32_t> cb_group(ctx->n_cb, 0), group_cb(ctx->n_groups + 1, 0);
    for (uint32_t g = 0; g < ctx->n_groups; ++g) {
      group_cb[g] = ctx->n_groups == 1 ? 0u : ctx->group_first_cb[g];
      group_cb[g + 1] = ctx->n_groups == 1 ? ctx->n_cb : ctx->group_first_cb[g + 1];
      for (uint32_t cb = group_cb[g]; cb < group_cb[g + 1]; ++cb) cb_group[cb] = g;
    }
    if ((rc = upload(ctx->d_cb_group, cb_group.data(), cb_group.size() * 4))) return rc;
    if ((rc = upload(ctx->d_group_cb, group_cb.data(), group_cb.size() * 4))) return rc;
  }
  DDS_CHECK_CUDA(ctx, ctx->d_cb_done.Reserve(size_t(ctx->n_cb) * 4));
  DDS_CHECK_CUDA(ctx, ctx->d_cb_flag.Reserve(size_t(ctx->n_cb) * 4));
  DDS_CHECK_CUDA(ctx, ctx->d_cb_avg.Reserve(size_t(ctx->n_cb) * 8));
  DDS_CHECK_CUDA(ctx, ctx->d_counters.Reserve(16));
  DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_cb_done.ptr, 0, size_t(ctx->n_cb) * 4, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_cb_flag.ptr, 0, size_t(ctx->n_cb) * 4, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_counters.ptr, 0, 16, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->plan_dirty = false;
  ctx->DestroyGraph();
  return DDSOLVE_OK;
}

// Builds the streaming plan: kernel choice, CTA work split, partial slots and
// the finalisation lists.
// Plan of the full-Jones path: every slab's runs numbered globally (one
// fj_pass_kernel thread each) and, per (channel block, antenna,
// sub-solution) item, the list of partial slots (run, direction, side) that
// add up to its normal equations, in run order.
int BuildFullJonesPlan(ddsolve_ctx* ctx) {
  const uint32_t n_dir = ctx->n_dir, n_ant = ctx->n_ant, n_sub = ctx->n_sub;
  std::vector<SlabDesc> descs;
  std::vector<uint32_t> slab_sol, run_start{0};
  std::vector<std::vector<uint32_t>> lists(size_t(ctx->n_cb) * n_ant * n_sub);
  // Rows of a run split into parts (one thread each) so that the grid has
  // about four times the threads one wave holds (a thread of the four-
  // direction kernel needs most of its 255 registers: 256 threads per SM),
  // keeping at least 16 rows per part (the parts' slots then add at most a
  // quarter to the pass's bytes).
  uint64_t total_runs = 0, max_rows = 1;
  for (uint32_t c = 0; c < ctx->n_cb; ++c)
    for (const HostSlab& s : ctx->cbs[c].slabs) {
      total_runs += s.R;
      max_rows = std::max<uint64_t>(max_rows, uint64_t(s.T) * s.L);
    }
  // (two directions: two lanes per part, more than four: a thread per part
  // and direction in the accumulation, so fewer parts give the same waves)
  const uint64_t lanes = n_dir == 2 ? 2 : n_dir > uint32_t(kFjMaxDirections) ? n_dir : 1;
  const uint64_t want_threads = uint64_t(std::max(ctx->n_sm, 1)) * 256 * 4 / lanes;
  uint64_t parts = total_runs ? (want_threads + total_runs - 1) / total_runs : 1;
  parts = std::max<uint64_t>(1, std::min<uint64_t>({parts, max_rows / 16, 16}));
  if (total_runs * parts * n_dir >= (uint64_t(1) << 31)) parts = 1;
  uint64_t n_runs = 0, n_resid = 0;
  std::vector<uint64_t> resid_off;
  for (uint32_t c = 0; c < ctx->n_cb; ++c) {
    ChannelBlockStore& cb = ctx->cbs[c];
    for (const HostSlab& s : cb.slabs) {
      SlabDesc sd{};
      sd.vis = cb.vis.as<char>() + s.elem_off * (1 + n_dir) * ctx->elem_bytes;
      sd.W = s.W;
      sd.run_ant = cb.run_ant_dev.as<uint32_t>() + s.run_off;
      sd.cb = c;
      sd.T = s.T;
      sd.L = s.L;
      sd.R = s.R;
      sd.sol_off = uint32_t(slab_sol.size());
      slab_sol.insert(slab_sol.end(), s.sol.begin(), s.sol.end());
      descs.push_back(sd);
      for (uint32_t r = 0; r < s.R; ++r) {
        const uint32_t ap = cb.run_ant[s.run_off + r];
        const uint32_t a1 = ap & 0xFFFFu, a2 = ap >> 16;
        for (uint64_t part = 0; part < parts; ++part)
          for (uint32_t d = 0; d < n_dir; ++d) {
            const uint64_t slot = (part * total_runs + n_runs + r) * n_dir + d;
            if (slot >= (uint64_t(1) << 31))
              return ctx->Fail(DDSOLVE_E_UNSUPPORTED, "full-Jones: too many runs");
            const size_t base = size_t(c) * n_ant;
            lists[(base + a1) * n_sub + s.sol[d]].push_back(uint32_t(slot << 1));
            lists[(base + a2) * n_sub + s.sol[d]].push_back(uint32_t(slot << 1) | 1u);
          }
      }
      n_runs += s.R;
      run_start.push_back(uint32_t(n_runs));
      resid_off.push_back(n_resid);
      n_resid += uint64_t(s.T) * s.L * s.R;
    }
  }
  std::vector<uint32_t> off(lists.size() + 1, 0), ent;
  for (size_t i = 0; i < lists.size(); ++i) {
    off[i] = uint32_t(ent.size());
    ent.insert(ent.end(), lists[i].begin(), lists[i].end());
  }
  off[lists.size()] = uint32_t(ent.size());
  if (ent.empty()) ent.push_back(0);
  auto up = [&](DevBuf& b, const void* src, size_t bytes) -> int {
    DDS_CHECK_CUDA(ctx, b.Reserve(bytes));
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(b.ptr, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return DDSOLVE_OK;
  };
  int rc;
  if ((rc = up(ctx->d_slabs, descs.data(), descs.size() * sizeof(SlabDesc))) != DDSOLVE_OK ||
      (rc = up(ctx->d_slab_sol, slab_sol.data(), slab_sol.size() * 4)) != DDSOLVE_OK ||
      (rc = up(ctx->d_fj_run_start, run_start.data(), run_start.size() * 4)) != DDSOLVE_OK ||
      (rc = up(ctx->d_fj_list_off, off.data(), off.size() * 4)) != DDSOLVE_OK ||
      (rc = up(ctx->d_fj_list_ent, ent.data(), ent.size() * 4)) != DDSOLVE_OK)
    return rc;
  if (n_dir > uint32_t(kFjMaxDirections)) {  // the residual between the pass launches
    if ((rc = up(ctx->d_fj_resid_off, resid_off.data(), resid_off.size() * 8)) != DDSOLVE_OK)
      return rc;
    DDS_CHECK_CUDA(ctx, ctx->d_fj_resid.Reserve(std::max<uint64_t>(n_resid, 1) * 32));
  }
  DDS_CHECK_CUDA(ctx, ctx->d_partials.Reserve(
                          std::max<uint64_t>(n_runs * parts, 1) * n_dir * kFjSlotFloats * 4));
  const uint32_t n_items = ctx->n_cb * n_ant * n_sub;
  ctx->fj_blocks = uint32_t((uint64_t(n_items) * 32 + kThreads - 1) / kThreads);  // a warp per item
  DDS_CHECK_CUDA(ctx, ctx->d_block_sum.Reserve(size_t(ctx->fj_blocks) * 8));
  DDS_CHECK_CUDA(ctx, ctx->d_block_cnt.Reserve(size_t(ctx->fj_blocks) * 4));
  // keep the host vectors alive until the copies have been issued from pageable memory
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->fj_n_slabs = uint32_t(descs.size());
  ctx->fj_n_runs = uint32_t(n_runs);
  ctx->fj_parts = uint32_t(parts);
  // The residual kernel stores R per row, so its row split costs no partial
  // slots: about four waves of its threads (3 blocks of kFjThreads per SM),
  // at least 8 rows each.
  {
    const uint64_t want_resid = uint64_t(std::max(ctx->n_sm, 1)) * 3 * kFjThreads * 4;
    uint64_t rp = total_runs ? (want_resid + total_runs - 1) / total_runs : 1;
    rp = std::max<uint64_t>(1, std::min<uint64_t>({rp, max_rows / 8, 16}));
    ctx->fj_resid_parts = uint32_t(rp);
  }
  ctx->use_pipe = false;
  ctx->plan_dirty = false;
  return DDSOLVE_OK;
}

int BuildPlanImpl(ddsolve_ctx* ctx, bool allow_pipe) {
  for (uint32_t c = 0; c < ctx->n_cb; ++c)
    if (!ctx->cbs[c].set)
      return ctx->Fail(DDSOLVE_E_STATE,
                       "channel block " + std::to_string(c) + " has no data");
  if (ctx->n_pol == 4) return BuildFullJonesPlan(ctx);
  int max_optin = 0;
  DDS_CHECK_CUDA(ctx, cudaDeviceGetAttribute(
                          &max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                          ctx->device));
  // Pipelined kernel when the direction count, the correlation layout and the
  // shared memory allow it (and no lane groups were requested).
  ctx->use_pipe = false;
  ctx->pipe_ng = 1;
  if (allow_pipe && ctx->tune_ng == 0 && ctx->tune_pipe != 0 &&
      (ctx->n_corr == 2 || ctx->n_corr == 4) && !std::getenv("DDSOLVE_NO_PIPE")) {
    const KernelEntry* pe =
        FindPipeKernel(int(ctx->n_corr), int(ctx->n_pol), int(ctx->n_dir));
    if (pe) ctx->pipe_ng = uint32_t(pe->ng);
    const uint32_t acc_stride = PipeAccStride(ctx->n_dir, ctx->n_pol);
    const uint32_t gain_stride = PipeGainStride(ctx->n_dir, ctx->n_pol);
    uint32_t stages = 0;
    for (uint32_t st = kPipeMaxStages; st >= 2 && pe; --st)
      if (PipeSmemBytes(ctx, st, acc_stride, gain_stride) <= size_t(max_optin)) {
        stages = st;
        break;
      }
    if (pe && stages >= 2) {
      const size_t smem = PipeSmemBytes(ctx, stages, acc_stride, gain_stride);
      DDS_CHECK_CUDA(ctx, cudaFuncSetAttribute(
                              pe->fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              int(smem)));
      int occ = 0;
      DDS_CHECK_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                              &occ, pe->fn, kPipeThreads, smem));
      if (occ >= 1) {
        ctx->use_pipe = true;
        ctx->pipe_fn = pe->fn;
        ctx->pipe_smem = smem;
        ctx->pipe_stages = stages;
        ctx->acc_stride = acc_stride;
        ctx->gain_stride = gain_stride;
        ctx->dmax = uint32_t(pe->dmax);
        ctx->ng = 1;
      }
    }
  }
  int occ = 1;
  size_t slot_floats = 0;
  uint32_t runs_per_block = 0;
  if (ctx->use_pipe) {
    runs_per_block = kPipeRuns;
    slot_floats = size_t(ctx->n_ant) * ctx->acc_stride;
  } else {
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
    if (smem > size_t(max_optin))
      return ctx->Fail(DDSOLVE_E_UNSUPPORTED,
                       "antenna x direction accumulators exceed shared memory");
    DDS_CHECK_CUDA(ctx, cudaFuncSetAttribute(ke->fn,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             int(smem)));
    DDS_CHECK_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                            &occ, ke->fn, kThreads, smem));
    if (occ < 1) return ctx->Fail(DDSOLVE_E_UNSUPPORTED, "stream kernel cannot launch");
    ctx->stream_smem = smem;
    runs_per_block = kThreads / ng;
    slot_floats = acc_n;
  }

  // Global slab list and steps.
  struct GSlab {
    uint32_t cb, idx;
  };
  std::vector<GSlab> gslabs;
  std::vector<SlabDesc> descs;
  std::vector<uint32_t> slab_sol;
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
      sd.vis = cb.vis.as<char>() + s.elem_off * (1 + ctx->n_dir) * ctx->elem_bytes;
      sd.W = s.W;
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
  if (ctx->use_pipe) return BuildPipePlan(ctx, descs, slab_sol, max_optin);
  ctx->pipe_ng = 1;
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

  // Finalisation blocks: each covers items (cb, antenna, sub-solution) of one
  // interval only, so that its norm partial belongs to that interval.
  const uint32_t per_cb_items = ctx->n_ant * ctx->n_sub;
  std::vector<uint32_t> block_group, block_item0, block_item_end, group_blocks(1, 0);
  std::vector<uint32_t> cb_group(ctx->n_cb, 0);
  for (uint32_t g = 0; g < ctx->n_groups; ++g) {
    const uint32_t cb0 = ctx->n_groups == 1 ? 0 : ctx->group_first_cb[g];
    const uint32_t cb1 = ctx->n_groups == 1 ? ctx->n_cb : ctx->group_first_cb[g + 1];
    for (uint32_t cb = cb0; cb < cb1; ++cb) cb_group[cb] = g;
    const uint32_t i0 = cb0 * per_cb_items, i1 = cb1 * per_cb_items;
    for (uint32_t i = i0; i < i1; i += kThreads) {
      block_group.push_back(g);
      block_item0.push_back(i);
      block_item_end.push_back(std::min(i1, i + kThreads));
    }
    group_blocks.push_back(uint32_t(block_group.size()));
  }
  ctx->fin_blocks = uint32_t(block_group.size());

  auto upload = [&](DevBuf& b, const void* src, size_t bytes) -> int {
    DDS_CHECK_CUDA(ctx, b.Reserve(bytes));
    if (bytes)
      DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(b.ptr, src, bytes, cudaMemcpyHostToDevice,
                                          ctx->stream));
    return DDSOLVE_OK;
  };
  int rc;
  if ((rc = upload(ctx->d_block_group, block_group.data(), block_group.size() * 4))) return rc;
  if ((rc = upload(ctx->d_block_item0, block_item0.data(), block_item0.size() * 4))) return rc;
  if ((rc = upload(ctx->d_block_item_end, block_item_end.data(), block_item_end.size() * 4)))
    return rc;
  if ((rc = upload(ctx->d_group_blocks, group_blocks.data(), group_blocks.size() * 4))) return rc;
  if ((rc = upload(ctx->d_cb_group, cb_group.data(), cb_group.size() * 4))) return rc;
  if ((rc = upload(ctx->d_slabs, descs.data(), descs.size() * sizeof(SlabDesc)))) return rc;
  if ((rc = upload(ctx->d_visits, visits.data(), visits.size() * sizeof(Visit)))) return rc;
  if ((rc = upload(ctx->d_cta_off, cta_off.data(), cta_off.size() * 4))) return rc;
  if ((rc = upload(ctx->d_slab_sol, slab_sol.data(), slab_sol.size() * 4))) return rc;
  if ((rc = upload(ctx->d_fin_off, fin_off.data(), fin_off.size() * 4))) return rc;
  if ((rc = upload(ctx->d_fin_visits, fin_visits.data(), fin_visits.size() * 4))) return rc;
  if ((rc = upload(ctx->d_dir_of_sub, ctx->dir_of_sub.data(), ctx->dir_of_sub.size() * 4)))
    return rc;
  DDS_CHECK_CUDA(ctx, ctx->d_cb_done.Reserve(size_t(ctx->n_cb) * 4));
  DDS_CHECK_CUDA(ctx, ctx->d_cb_flag.Reserve(size_t(ctx->n_cb) * 4));
  DDS_CHECK_CUDA(ctx, ctx->d_cb_avg.Reserve(size_t(ctx->n_cb) * 8));
  DDS_CHECK_CUDA(ctx, ctx->d_counters.Reserve(16));
  DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_cb_done.ptr, 0, size_t(ctx->n_cb) * 4,
                                      ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_cb_flag.ptr, 0, size_t(ctx->n_cb) * 4,
                                      ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_counters.ptr, 0, 16, ctx->stream));
  DDS_CHECK_CUDA(ctx, ctx->d_partials.Reserve(
                          std::max<size_t>(1, size_t(ctx->n_visits) * slot_floats) * 4));
  const size_t n_block_partials = std::max<size_t>(ctx->fin_blocks, ctx->n_ctas);
  DDS_CHECK_CUDA(ctx, ctx->d_block_sum.Reserve(n_block_partials * 8));
  DDS_CHECK_CUDA(ctx, ctx->d_block_cnt.Reserve(n_block_partials * 4));
  // Plan arrays are small host vectors: wait so they can be released.
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->plan_dirty = false;
  ctx->DestroyGraph();
  return DDSOLVE_OK;
}

// The pipelined plan when it applies (a lane-group pipe_kernel needs every
// tile to take the direct reduction), else the stream_kernel plan.
int BuildPlan(ddsolve_ctx* ctx) {
  const int rc = BuildPlanImpl(ctx, true);
  if (rc != kPlanNoPipe) return rc;
  ctx->use_pipe = false;
  return BuildPlanImpl(ctx, false);
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
  f.fin_mode = kFinFused;
  f.settings = ctx->d_settings.as<DevSettings>();
  f.block_sum = ctx->d_block_sum.as<double>();
  f.block_cnt = ctx->d_block_cnt.as<uint32_t>();
  f.state = ctx->d_state.as<LoopState>();
  f.nonfinite = ctx->d_nonfinite.as<uint32_t>();
  f.step_magnitudes = ctx->d_mags.as<double>();
  f.handle = ctx->handle;
  f.use_handle = 0;
  f.block_group = ctx->d_block_group.as<uint32_t>();
  f.block_item0 = ctx->d_block_item0.as<uint32_t>();
  f.block_item_end = ctx->d_block_item_end.as<uint32_t>();
  f.group_blocks = ctx->d_group_blocks.as<uint32_t>();
  f.n_groups = ctx->n_groups;
  f.mags_stride = ctx->mags_stride;
  return f;
}

PipeParams MakePipeParams(ddsolve_ctx* ctx, bool host_mode, bool use_handle) {
  PipeParams p;
  p.slabs = ctx->d_slabs.as<SlabDesc>();
  p.frags = ctx->d_frags.as<Frag>();
  p.cta_frag_off = ctx->d_cta_frag_off.as<uint32_t>();
  p.slab_sol = ctx->d_slab_sol.as<uint32_t>();
  p.solutions = ctx->d_sol.as<double2>();
  p.partials = ctx->d_partials.as<float>();
  p.tables = ctx->d_tables.as<float2>();
  p.table_f2 = ctx->table_f2;
  p.tab_off = ctx->d_tab_off.as<uint32_t>();
  p.tab_ent = ctx->d_tab_ent.as<uint32_t>();
  p.n_ant = ctx->n_ant;
  p.n_dir = ctx->n_dir;
  p.n_sub = ctx->n_sub;
  p.n_cb = ctx->n_cb;
  p.acc_stride = ctx->acc_stride;
  p.gain_stride = ctx->gain_stride;
  p.stages = ctx->pipe_stages;
  p.acc_floats = ctx->n_ant * ctx->acc_stride;
  p.owner_groups = ctx->owner_groups;
  p.n_gbuf = ctx->n_gbuf;
  p.powers = ctx->use_powers ? ctx->d_powers.as<float>() : nullptr;
  p.power_floats = ctx->power_floats;
  p.off_acc = ctx->off_acc;
  p.off_gtab = ctx->off_gtab;
  p.off_stg = ctx->off_stg;
  p.off_cnt = ctx->off_cnt;
  p.off_off = ctx->off_off;
  p.off_pair = ctx->off_pair;
  p.off_ent = ctx->off_ent;
  p.off_wsum = ctx->off_wsum;
  p.off_stages = ctx->off_stages;
  p.fin_off = ctx->d_fin_off.as<uint32_t>();
  p.fin_visits = ctx->d_fin_visits.as<uint32_t>();
  p.fin_first = ctx->fin_ranges ? ctx->d_fin_first.as<uint32_t>() : nullptr;
  p.n_groups = ctx->n_groups;
  p.cb_group = ctx->d_cb_group.as<uint32_t>();
  p.group_cb = ctx->d_group_cb.as<uint32_t>();
  p.mags_stride = ctx->mags_stride;
  p.dir_of_sub = ctx->d_dir_of_sub.as<uint32_t>();
  p.cb_flag = ctx->d_cb_flag.as<uint32_t>();
  p.cb_avg = ctx->d_cb_avg.as<double>();
  p.cb_newflag = ctx->d_cb_done.as<uint32_t>();
  p.block_sum = ctx->d_block_sum.as<double>();
  p.block_cnt = ctx->d_block_cnt.as<uint32_t>();
  p.counters = ctx->d_counters.as<uint32_t>();
  p.next_out = ctx->d_next.as<double2>();
  p.host_mode = host_mode ? 1 : 0;
  p.fin_mode = kFinFused;
  p.settings = ctx->d_settings.as<DevSettings>();
  p.state = ctx->d_state.as<LoopState>();
  p.step_magnitudes = ctx->d_mags.as<double>();
  p.handle = ctx->handle;
  p.use_handle = use_handle ? 1 : 0;
  return p;
}

// Gain tables of the pipelined path from the current solutions.
int LaunchBuildTables(ddsolve_ctx* ctx) {
  if (!ctx->use_pipe) return DDSOLVE_OK;
  const uint32_t n = ctx->n_tables * ctx->n_ant * ctx->n_dir;
  if (n == 0) return DDSOLVE_OK;
  const uint32_t blocks = (n + 255) / 256;
  if (ctx->n_pol == 2)
    build_tables_kernel<2><<<blocks, 256, 0, ctx->stream>>>(
        ctx->d_sol.as<double2>(), ctx->d_tables.as<float2>(), ctx->d_tab_cb.as<uint32_t>(),
        ctx->d_tab_sol.as<uint32_t>(), ctx->n_tables, ctx->n_ant, ctx->n_dir, ctx->n_sub,
        ctx->gain_stride, ctx->table_f2);
  else
    build_tables_kernel<1><<<blocks, 256, 0, ctx->stream>>>(
        ctx->d_sol.as<double2>(), ctx->d_tables.as<float2>(), ctx->d_tab_cb.as<uint32_t>(),
        ctx->d_tab_sol.as<uint32_t>(), ctx->n_tables, ctx->n_ant, ctx->n_dir, ctx->n_sub,
        ctx->gain_stride, ctx->table_f2);
  DDS_CHECK_CUDA(ctx, cudaGetLastError());
  return DDSOLVE_OK;
}

// Model powers of the pipelined path, when the plan uses them and they are
// stale (new data, or a solve used them since), or `force`.
int LaunchPowers(ddsolve_ctx* ctx, bool force) {
  if (!ctx->use_pipe || !ctx->use_powers || (!ctx->powers_dirty && !force)) return DDSOLVE_OK;
  const uint32_t blocks = ctx->n_power_tiles * ctx->n_dir;
  if (blocks) {
    if (ctx->n_corr == 2)
      power_kernel<2><<<blocks, kPipeRuns, 0, ctx->stream>>>(
          ctx->d_slabs.as<SlabDesc>(), ctx->d_power_tiles.as<PowerTile>(), ctx->n_dir,
          ctx->power_floats, ctx->d_powers.as<float>());
    else
      power_kernel<4><<<blocks, kPipeRuns, 0, ctx->stream>>>(
          ctx->d_slabs.as<SlabDesc>(), ctx->d_power_tiles.as<PowerTile>(), ctx->n_dir,
          ctx->power_floats, ctx->d_powers.as<float>());
    DDS_CHECK_CUDA(ctx, cudaGetLastError());
  }
  ctx->powers_dirty = false;
  return DDSOLVE_OK;
}

int LaunchMakeFinite(ddsolve_ctx* ctx, bool use_handle) {
  const uint32_t per_cb = ctx->n_ant * ctx->n_sub * ctx->n_pol;
  if (ctx->n_pol == 2)
    make_finite_kernel<2><<<ctx->n_cb, kThreads, 0, ctx->stream>>>(
        ctx->d_sol.as<double2>(), ctx->d_nonfinite.as<uint32_t>(), per_cb,
        ctx->handle, use_handle ? 1 : 0,
        ctx->n_groups > 1 ? ctx->d_cb_group.as<uint32_t>() : nullptr,
        ctx->d_state.as<LoopState>());
  else
    make_finite_kernel<1><<<ctx->n_cb, kThreads, 0, ctx->stream>>>(
        ctx->d_sol.as<double2>(), ctx->d_nonfinite.as<uint32_t>(), per_cb,
        ctx->handle, use_handle ? 1 : 0,
        ctx->n_groups > 1 ? ctx->d_cb_group.as<uint32_t>() : nullptr,
        ctx->d_state.as<LoopState>());
  DDS_CHECK_CUDA(ctx, cudaGetLastError());
  return DDSOLVE_OK;
}

// Launches the device constraints, in order, on the stepped next solutions
// (d_next); *result = the buffer that then holds the constrained ones (the
// smoothing writes to the other buffer of the pair).
int LaunchConstraints(ddsolve_ctx* ctx, bool use_handle, double2** result) {
  double2* cur = ctx->d_next.as<double2>();
  const uint32_t n_series = ctx->n_ant * ctx->n_sub * ctx->n_pol;
  const int uh = use_handle ? 1 : 0;
  const LoopState* state = ctx->d_state.as<LoopState>();
  for (const ddsolve_ctx::DeviceConstraint& c : ctx->constraints) {
    const char* b = c.buf.as<const char>();
    if (c.kind == DDSOLVE_CONSTRAINT_SMOOTHNESS) {
      double2* dst = cur == ctx->d_next.as<double2>() ? ctx->d_cons.as<double2>()
                                                      : ctx->d_next.as<double2>();
      SmoothParams sp;
      sp.in = cur;
      sp.out = dst;
      sp.n_cb = ctx->n_cb;
      sp.n_series = n_series;
      sp.n_ant = ctx->n_ant;
      sp.n_sub = ctx->n_sub;
      sp.n_pol = ctx->n_pol;
      sp.freq = reinterpret_cast<const double*>(b + c.off[0]);
      sp.fcorr = reinterpret_cast<const double*>(b + c.off[1]);
      sp.band = reinterpret_cast<const uint32_t*>(b + c.off[2]);
      sp.weights = reinterpret_cast<const double*>(b + c.off[3]);
      sp.per_sub_weights = c.per_sub_weights;
      sp.factor = reinterpret_cast<const double*>(b + c.off[4]);
      sp.bandwidth = c.bandwidth;
      sp.truncate = c.truncate;
      sp.state = state;
      sp.use_handle = uh;
      const uint64_t n = uint64_t(ctx->n_cb) * n_series;
      smooth_kernel<<<uint32_t((n + 255) / 256), 256, 0, ctx->stream>>>(sp);
      cur = dst;
    } else if (c.kind == DDSOLVE_CONSTRAINT_ANTENNA) {
      const uint64_t n = uint64_t(ctx->n_cb) * ctx->n_sub * ctx->n_pol;
      antenna_constraint_kernel<<<uint32_t((n + 255) / 256), 256, 0, ctx->stream>>>(
          cur, ctx->n_cb, ctx->n_ant, ctx->n_sub, ctx->n_pol,
          reinterpret_cast<const uint32_t*>(b + c.off[0]),
          reinterpret_cast<const uint32_t*>(b + c.off[1]), c.n_sets, state, uh);
    } else {
      reference_antenna_select_kernel<<<1, 32, 0, ctx->stream>>>(
          cur, ctx->n_cb, ctx->n_ant, ctx->n_sub, ctx->n_pol, ctx->d_ref_ant.as<uint32_t>(),
          state, uh);
      const uint32_t n = ctx->n_cb * ctx->n_pol;
      reference_antenna_apply_kernel<<<(n + 255) / 256, 256, 0, ctx->stream>>>(
          cur, ctx->n_cb, ctx->n_ant, ctx->n_sub, ctx->n_pol, ctx->d_ref_ant.as<uint32_t>(),
          state, uh);
    }
    DDS_CHECK_CUDA(ctx, cudaGetLastError());
  }
  *result = cur;
  return DDSOLVE_OK;
}

// Kernel launches of the device constraints per iteration.
uint32_t ConstraintLaunches(const ddsolve_ctx* ctx) {
  uint32_t n = 0;
  for (const ddsolve_ctx::DeviceConstraint& c : ctx->constraints)
    n += c.kind == DDSOLVE_CONSTRAINT_REFERENCE_ANTENNA ? 2u : 1u;
  return n;
}

// Launches one iteration's kernels on the context stream: pipe_kernel alone
// on the pipelined path (its fused finalisation repairs non-finite solutions
// lazily, so make_finite_kernel only runs once before the loop), else
// make_finite_kernel + stream_kernel + finalize_kernel. With device
// constraints (solve mode) the finalisation is split around them: the pass
// finalises in step-only mode, the constraints run, and an assignment pass
// (assign_kernel, or finalize_kernel again) finishes the iteration.
// One full-Jones iteration: MakeSolutionsFinite4Pol, the pass, the
// finalisation (or, in host mode, the next solutions only).
// Launches of the full-Jones streaming pass: one, or the residual and the
// accumulation.
uint32_t FjPassLaunches(const ddsolve_ctx* ctx) {
  return ctx->n_dir <= uint32_t(kFjMaxDirections) ? 1u : 2u;
}

int LaunchFullJones(ddsolve_ctx* ctx, bool host_mode, bool use_handle, bool with_make_finite) {
  if (with_make_finite) {
    make_finite4_kernel<<<ctx->n_cb, kThreads, 0, ctx->stream>>>(
        ctx->d_sol.as<double2>(), ctx->d_nonfinite.as<uint32_t>(), ctx->n_ant * ctx->n_sub * 4,
        ctx->handle, use_handle ? 1 : 0, ctx->d_state.as<LoopState>());
    DDS_CHECK_CUDA(ctx, cudaGetLastError());
  }
  FjPassParams pp;
  pp.slabs = ctx->d_slabs.as<SlabDesc>();
  pp.slab_sol = ctx->d_slab_sol.as<uint32_t>();
  pp.run_start = ctx->d_fj_run_start.as<uint32_t>();
  pp.solutions = ctx->d_sol.as<double2>();
  pp.partials = ctx->d_partials.as<float>();
  pp.n_slabs = ctx->fj_n_slabs;
  pp.n_runs = ctx->fj_n_runs;
  pp.n_ant = ctx->n_ant;
  pp.n_sub = ctx->n_sub;
  pp.n_dir = ctx->n_dir;
  pp.state = ctx->d_state.as<LoopState>();
  pp.use_handle = (use_handle && !host_mode) ? 1 : 0;
  pp.resid = nullptr;
  pp.resid_off = nullptr;
  pp.n_parts = ctx->fj_parts;
  const uint32_t blocks = std::max<uint32_t>(
      1, uint32_t((uint64_t(ctx->fj_n_runs) * ctx->fj_parts + kFjThreads - 1) / kFjThreads));
  const uint64_t units = uint64_t(ctx->fj_n_runs) * ctx->fj_parts;
  const uint32_t blocks2 = uint32_t(std::max<uint64_t>(1, (units * 2 + kFjThreads - 1) / kFjThreads));
  // two directions: two lanes per part (measured faster than one thread per
  // part); three or four: one thread per part (two lanes of two directions
  // and four lanes of one direction each measured slower: their extra loads
  // and shuffles cost more than their occupancy gives)
  switch (ctx->n_dir) {
    case 1: fj_pass_kernel<1><<<blocks, kFjThreads, 0, ctx->stream>>>(pp); break;
    case 2: fj_lane_kernel<2, 1><<<blocks2, kFjThreads, 0, ctx->stream>>>(pp); break;
    case 3: fj_pass_kernel<3><<<blocks, kFjThreads, 0, ctx->stream>>>(pp); break;
    case 4: fj_pass_kernel<4><<<blocks, kFjThreads, 0, ctx->stream>>>(pp); break;
    default:
      pp.resid = ctx->d_fj_resid.as<float2>();
      pp.resid_off = ctx->d_fj_resid_off.as<uint64_t>();
      {  // its own row split (R is stored per row)
        FjPassParams rp = pp;
        rp.n_parts = ctx->fj_resid_parts;
        const uint64_t rthreads = uint64_t(ctx->fj_n_runs) * rp.n_parts;
        const uint32_t rblocks =
            uint32_t(std::max<uint64_t>(1, (rthreads + kFjThreads - 1) / kFjThreads));
        fj_residual_kernel<<<rblocks, kFjThreads, 0, ctx->stream>>>(rp);
      }
      {
        const uint64_t threads = units * ctx->n_dir;
        const uint32_t blocks_acc =
            uint32_t(std::max<uint64_t>(1, (threads + kFjThreads - 1) / kFjThreads));
        fj_accumulate_kernel<<<blocks_acc, kFjThreads, 0, ctx->stream>>>(pp);
      }
  }
  DDS_CHECK_CUDA(ctx, cudaGetLastError());
  FjFinParams fp;
  fp.partials = ctx->d_partials.as<float>();
  fp.list_off = ctx->d_fj_list_off.as<uint32_t>();
  fp.list_ent = ctx->d_fj_list_ent.as<uint32_t>();
  fp.solutions = ctx->d_sol.as<double2>();
  fp.next_out = ctx->d_next.as<double2>();
  fp.n_items = ctx->n_cb * ctx->n_ant * ctx->n_sub;
  fp.n_dir = ctx->n_dir;
  fp.n_ant = ctx->n_ant;
  fp.n_sub = ctx->n_sub;
  fp.host_mode = host_mode ? 1 : 0;
  fp.settings = ctx->d_settings.as<DevSettings>();
  fp.block_sum = ctx->d_block_sum.as<double>();
  fp.block_cnt = ctx->d_block_cnt.as<uint32_t>();
  fp.state = ctx->d_state.as<LoopState>();
  fp.nonfinite = ctx->d_nonfinite.as<uint32_t>();
  fp.step_magnitudes = ctx->d_mags.as<double>();
  fp.handle = ctx->handle;
  fp.use_handle = use_handle ? 1 : 0;
  fp.blocks_done = &ctx->d_state.as<LoopState>()->blocks_done;
  fj_finalize_kernel<<<ctx->fj_blocks, kThreads, 0, ctx->stream>>>(fp);
  DDS_CHECK_CUDA(ctx, cudaGetLastError());
  return DDSOLVE_OK;
}

int LaunchIteration(ddsolve_ctx* ctx, bool host_mode, bool use_handle,
                    bool with_make_finite) {
  if (ctx->n_pol == 4) return LaunchFullJones(ctx, host_mode, use_handle, with_make_finite);
  const bool constrained = !host_mode && !ctx->constraints.empty();
  if (ctx->use_pipe) {
    // Cooperative launch: pipe_kernel has a grid barrier, so all CTAs must be
    // resident (the grid is #SM x occupancy).
    PipeParams pp = MakePipeParams(ctx, host_mode, use_handle);
    if (constrained) pp.fin_mode = kFinStepOnly;
    void* args[] = {&pp};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ctx->n_ctas);
    cfg.blockDim = dim3(kPipeThreads);
    cfg.dynamicSmemBytes = ctx->pipe_smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    DDS_CHECK_CUDA(ctx, cudaLaunchKernelExC(&cfg, ctx->pipe_fn, args));
    if (!constrained) return DDSOLVE_OK;
    double2* cons = nullptr;
    const int rc = LaunchConstraints(ctx, use_handle, &cons);
    if (rc != DDSOLVE_OK) return rc;
    PipeParams ap = pp;
    ap.fin_mode = kFinAssignOnly;
    ap.next_out = cons;
    if (ctx->n_pol == 2)
      assign_kernel<2><<<ctx->n_ctas, kPipeRuns, 0, ctx->stream>>>(ap);
    else
      assign_kernel<1><<<ctx->n_ctas, kPipeRuns, 0, ctx->stream>>>(ap);
    DDS_CHECK_CUDA(ctx, cudaGetLastError());
    return DDSOLVE_OK;
  }
  if (with_make_finite) {
    const int rc = LaunchMakeFinite(ctx, use_handle);
    if (rc != DDSOLVE_OK) return rc;
  }
  const StreamParams sp = MakeStreamParams(ctx);
  ctx->stream_fn<<<ctx->n_ctas, kThreads, ctx->stream_smem, ctx->stream>>>(sp);
  DDS_CHECK_CUDA(ctx, cudaGetLastError());
  FinParams fp = MakeFinParams(ctx, host_mode);
  fp.use_handle = use_handle ? 1 : 0;
  if (constrained) fp.fin_mode = kFinStepOnly;
  for (int pass = 0; pass < (constrained ? 2 : 1); ++pass) {
    if (pass == 1) {
      double2* cons = nullptr;
      const int rc = LaunchConstraints(ctx, use_handle, &cons);
      if (rc != DDSOLVE_OK) return rc;
      fp.fin_mode = kFinAssignOnly;
      fp.next_out = cons;
    }
    if (ctx->n_pol == 2)
      finalize_kernel<2><<<ctx->fin_blocks, kThreads, 0, ctx->stream>>>(fp);
    else
      finalize_kernel<1><<<ctx->fin_blocks, kThreads, 0, ctx->stream>>>(fp);
    DDS_CHECK_CUDA(ctx, cudaGetLastError());
  }
  return DDSOLVE_OK;
}

// Enqueues the copy of the device error counters into the pinned stage (read
// by CheckDeviceError after the call's synchronization).
int StageCounters(ddsolve_ctx* ctx) {
  if (!ctx->use_pipe) return DDSOLVE_OK;
  DDS_CHECK_CUDA(ctx, ctx->ReserveStage(0));
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->h_stage->counters, ctx->d_counters.ptr, 16,
                                      cudaMemcpyDeviceToHost, ctx->stream));
  return DDSOLVE_OK;
}

// After the stream was synchronized: `staged` = the counters were copied by
// StageCounters in this call; otherwise they are read here.
int CheckDeviceError(ddsolve_ctx* ctx, bool staged = false) {
  if (!ctx->use_pipe) return DDSOLVE_OK;
  uint32_t c[2] = {0, 0};
  if (staged) {
    c[1] = ctx->h_stage->counters[1];
  } else {
    DDS_CHECK_CUDA(ctx, cudaMemcpy(c, ctx->d_counters.ptr, 8, cudaMemcpyDeviceToHost));
  }
  if (c[1] != 0) {
    cudaMemsetAsync(ctx->d_counters.ptr, 0, 16, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    return ctx->Fail(DDSOLVE_E_TIMEOUT,
                     "a bounded device wait of pipe_kernel timed out; results are invalid");
  }
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
  // pipe_kernel: several iterations per loop test (launches after the loop
  // stopped return at once); one otherwise.
  int rc = DDSOLVE_OK;
  uint32_t unroll = ctx->use_pipe ? ctx->graph_unroll : 1u;
  if (const char* e = std::getenv("DDSOLVE_GRAPH_UNROLL"))
    if (ctx->use_pipe) unroll = uint32_t(std::max(1, std::atoi(e)));
  for (uint32_t u = 0; u < unroll && rc == DDSOLVE_OK; ++u)
    rc = LaunchIteration(ctx, false, true, true);
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
  ctx->mags_stride = ds.hard_cap;
  DDS_CHECK_CUDA(ctx, ctx->d_mags.Reserve(size_t(ds.hard_cap) * ctx->n_groups * 8));
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
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    g_last_error = std::string("ddsolve_create: ") + cudaGetErrorString(e);
    return DDSOLVE_E_CUDA;
  }
  ctx->blk_predict_in.resize(ctx->n_cb);
  ctx->blk_data_stage.resize(ctx->n_cb);
  ctx->blk_predict_host.assign(ctx->n_cb, nullptr);
  ctx->blk_predict_host_bytes.assign(ctx->n_cb, 0);
  ctx->blk_predict_copied.assign(ctx->n_cb, nullptr);
  ctx->blk_data_copied.assign(ctx->n_cb, nullptr);
  ctx->blk_packed.assign(ctx->n_cb, nullptr);
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

// The regular layout of ddsolve_set_channel_block_regular; `make_stage`
// returns the stager that fills the block's staging buffer (copies, GPU
// predict, GPU weighting) once the block's visibility count is set.
static int SetRegularBlock(ddsolve_ctx* ctx, uint32_t cbi, uint32_t n_times,
                           uint32_t n_baselines, uint32_t n_channels,
                           const uint32_t* antenna1, const uint32_t* antenna2,
                           const std::function<StageFn(const ChannelBlockStore&)>& make_stage,
                           bool models_in_place = false) {
  if (!ctx) return DDSOLVE_E_INVALID;
  if (cbi >= ctx->n_cb) return ctx->Fail(DDSOLVE_E_INVALID, "channel block out of range");
  if (n_times == 0 || n_baselines == 0 || n_channels == 0 || !antenna1 || !antenna2)
    return ctx->Fail(DDSOLVE_E_INVALID, "empty channel block or NULL pointer");
  // Runs in cyclic-diagonal order. Each baseline is oriented so that its
  // cyclic distance delta = (a2 - a1) mod n_ant is at most n_ant / 2 (a
  // swapped baseline is stored Hermitian-transposed by the repack, which does
  // not change the normal equations); runs are sorted by (delta, a1). A
  // cyclic diagonal is then a permutation (distinct first and distinct second
  // antennas), so windows of up to n_ant consecutive runs have distinct
  // antennas on each side: conflict-free shared-memory accumulation. The
  // order depends on the antenna arrays only, so it is computed once for the
  // channel blocks and intervals that repeat them.
  const uint32_t n_ant = ctx->n_ant;
  const bool same_order = ctx->order_a1.size() == n_baselines &&
                          std::equal(antenna1, antenna1 + n_baselines, ctx->order_a1.begin()) &&
                          std::equal(antenna2, antenna2 + n_baselines, ctx->order_a2.begin());
  if (!same_order) {
    for (uint32_t b = 0; b < n_baselines; ++b)
      if (antenna1[b] >= n_ant || antenna2[b] >= n_ant || antenna1[b] == antenna2[b])
        return ctx->Fail(DDSOLVE_E_INVALID, "bad antenna pair (or autocorrelation)");
    std::vector<uint32_t> o_a1(n_baselines), o_a2(n_baselines), o_delta(n_baselines);
    std::vector<uint8_t> o_flip(n_baselines);
    for (uint32_t b = 0; b < n_baselines; ++b) {
      const uint32_t a = antenna1[b], c = antenna2[b];
      const uint32_t d = (c + n_ant - a) % n_ant;
      bool flip = 2 * d > n_ant;
      if (2 * d == n_ant) flip = a > c;  // half-way diagonal: first antenna < n/2
      o_flip[b] = flip;
      o_a1[b] = flip ? c : a;
      o_a2[b] = flip ? a : c;
      o_delta[b] = flip ? n_ant - d : d;
    }
    std::vector<uint32_t> order(n_baselines);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) {
      return o_delta[x] != o_delta[y] ? o_delta[x] < o_delta[y] : o_a1[x] < o_a1[y];
    });
    ctx->order_a1.assign(antenna1, antenna1 + n_baselines);
    ctx->order_a2.assign(antenna2, antenna2 + n_baselines);
    ctx->order_bl = order;
    ctx->order_ant.resize(n_baselines);
    ctx->order_flip.resize(n_baselines);
    for (uint32_t r = 0; r < n_baselines; ++r) {
      const uint32_t b = order[r];
      ctx->order_ant[r] = o_a1[b] | (o_a2[b] << 16);
      ctx->order_flip[r] = o_flip[b];
    }
  }
  cudaSetDevice(ctx->device);
  ChannelBlockStore& cb = ctx->cbs[cbi];
  cb.n_vis = uint64_t(n_times) * n_baselines * n_channels;
  cb.slabs.clear();
  // Run arrays padded to whole 16-byte groups (pipe_kernel bulk-copies
  // them); padding runs have no antennas and no visibilities.
  const size_t n_run_pad = (size_t(n_baselines) + 3) & ~size_t(3);
  cb.run_ant.assign(n_run_pad, 0u);
  cb.run_src.assign(n_run_pad, 0u);
  cb.run_len.assign(n_run_pad, 0u);
  for (uint32_t r = 0; r < n_baselines; ++r) {
    cb.run_ant[r] = ctx->order_ant[r];
    cb.run_src[r] = ctx->order_bl[r] * n_channels;
    cb.run_len[r] = n_channels | (ctx->order_flip[r] ? kRunFlipped : 0u);
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
  // Time steps folded into one slab: all that share solution indices (the
  // pipelined kernel splits slabs along their rows for load balance).
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
  return UploadAndPack(ctx, cb, make_stage(cb), models_in_place,
                       models_in_place ? int(cbi) : -1);
}

int ddsolve_set_channel_block_regular(ddsolve_ctx* ctx, uint32_t cbi, uint32_t n_times,
                                      uint32_t n_baselines, uint32_t n_channels,
                                      const float* data, const float* model,
                                      const uint32_t* antenna1, const uint32_t* antenna2) {
  if (ctx && (!data || !model))
    return ctx->Fail(DDSOLVE_E_INVALID, "empty channel block or NULL pointer");
  return SetRegularBlock(ctx, cbi, n_times, n_baselines, n_channels, antenna1, antenna2,
                         [&](const ChannelBlockStore& cb) {
                           return StageCopy(ctx, cb, data, model);
                         });
}

int ddsolve_set_channel_block_regular_sky(ddsolve_ctx* ctx, uint32_t cbi, uint32_t n_times,
                                          uint32_t n_baselines, uint32_t n_channels,
                                          const float* data, const double* frequencies,
                                          const double* station_uvw,
                                          const uint32_t* antenna1, const uint32_t* antenna2,
                                          const ddsolve_sky_direction* sky) {
  if (!ctx) return DDSOLVE_E_INVALID;
  if (!data) return ctx->Fail(DDSOLVE_E_INVALID, "empty channel block or NULL pointer");
  const PredictJob job{n_times, n_baselines, n_channels, frequencies, station_uvw,
                       antenna1, antenna2, sky};
  const int rc = CheckPredictJob(ctx, job);
  if (rc != DDSOLVE_OK) return rc;
  return SetRegularBlock(ctx, cbi, n_times, n_baselines, n_channels, antenna1, antenna2,
                         [&](const ChannelBlockStore& cb) {
                           return StagePredict(ctx, cb, data, job, cbi);
                         },
                         true);
}

// A device address for a host-or-device input: device memory of the
// context's device is used in place, host memory is copied into `dst` at
// byte offset `off` (stream-ordered).
static int DeviceView(ddsolve_ctx* ctx, const void* src, size_t bytes, DevBuf& dst, size_t off,
                      const void** out) {
  cudaPointerAttributes attr{};
  const bool dev = cudaPointerGetAttributes(&attr, src) == cudaSuccess &&
                   attr.type == cudaMemoryTypeDevice && attr.device == ctx->device;
  cudaGetLastError();
  if (dev) {
    *out = src;
    return DDSOLVE_OK;
  }
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(dst.as<char>() + off, src, bytes, cudaMemcpyDefault,
                                      ctx->stream));
  *out = dst.as<char>() + off;
  return DDSOLVE_OK;
}

int ddsolve_set_interval_buffers(ddsolve_ctx* ctx, const ddsolve_interval_buffers* in) {
  if (!ctx) return DDSOLVE_E_INVALID;
  if (!in || !in->antenna1 || !in->antenna2 || !in->data || !in->weights ||
      in->n_times == 0 || in->n_baselines == 0 || in->n_channels < ctx->n_cb)
    return ctx->Fail(DDSOLVE_E_INVALID, "interval buffers: NULL pointer or empty interval");
  if (!in->model && (!in->sky || !in->frequencies || !in->station_uvw))
    return ctx->Fail(DDSOLVE_E_INVALID, "interval buffers: no model and no sky to predict it");
  cudaSetDevice(ctx->device);
  const uint32_t n_t = in->n_times, n_bl = in->n_baselines, n_ch = in->n_channels;
  // Cross baselines in buffer order (the regular SolveData constructor's).
  std::vector<uint32_t> bl_of_cross, a1x, a2x;
  for (uint32_t b = 0; b < n_bl; ++b) {
    if (in->antenna1[b] >= ctx->n_ant || in->antenna2[b] >= ctx->n_ant)
      return ctx->Fail(DDSOLVE_E_INVALID, "interval buffers: antenna index out of range");
    if (in->antenna1[b] == in->antenna2[b]) continue;
    bl_of_cross.push_back(b);
    a1x.push_back(in->antenna1[b]);
    a2x.push_back(in->antenna2[b]);
  }
  const uint32_t n_bx = uint32_t(bl_of_cross.size());
  if (n_bx == 0) return ctx->Fail(DDSOLVE_E_INVALID, "interval buffers: no cross baselines");
  const size_t n_raw = size_t(n_t) * n_bl * n_ch;
  const size_t b_data = n_raw * 32, b_w = n_raw * 16, b_f = in->flags ? n_raw * 4 : 0;
  const size_t b_m = in->model ? n_raw * 32 * ctx->n_dir : 0;
  auto align = [](size_t x) { return (x + 255) / 256 * 256; };
  const size_t o_w = align(b_data), o_f = o_w + align(b_w), o_m = o_f + align(b_f);
  const size_t o_x = o_m + align(b_m);
  DDS_CHECK_CUDA(ctx, ctx->raw_in.Reserve(o_x + align(size_t(n_bx) * 4)));
  const void *d_data = nullptr, *d_w = nullptr, *d_f = nullptr, *d_m = nullptr;
  int rc;
  if ((rc = DeviceView(ctx, in->data, b_data, ctx->raw_in, 0, &d_data)) != DDSOLVE_OK) return rc;
  if ((rc = DeviceView(ctx, in->weights, b_w, ctx->raw_in, o_w, &d_w)) != DDSOLVE_OK) return rc;
  if (in->flags &&
      (rc = DeviceView(ctx, in->flags, b_f, ctx->raw_in, o_f, &d_f)) != DDSOLVE_OK)
    return rc;
  if (in->model &&
      (rc = DeviceView(ctx, in->model, b_m, ctx->raw_in, o_m, &d_m)) != DDSOLVE_OK)
    return rc;
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->raw_in.as<char>() + o_x, bl_of_cross.data(),
                                      size_t(n_bx) * 4, cudaMemcpyHostToDevice, ctx->stream));
  const uint32_t* d_x = reinterpret_cast<const uint32_t*>(ctx->raw_in.as<char>() + o_x);
  for (uint32_t cbi = 0; cbi < ctx->n_cb; ++cbi) {
    const uint32_t c0 = uint32_t(uint64_t(cbi) * n_ch / ctx->n_cb);
    const uint32_t L = uint32_t(uint64_t(cbi + 1) * n_ch / ctx->n_cb) - c0;
    PredictJob job{n_t, n_bx, L, in->frequencies ? in->frequencies + c0 : nullptr,
                   in->station_uvw, a1x.data(), a2x.data(), in->sky};
    if (!in->model && (rc = CheckPredictJob(ctx, job)) != DDSOLVE_OK) return rc;
    rc = SetRegularBlock(ctx, cbi, n_t, n_bx, L, a1x.data(), a2x.data(),
                         [&](const ChannelBlockStore& cb) -> StageFn {
                           return [&, c0, L, job](char* st) {
                             WeighParams p;
                             p.data = static_cast<const float2*>(d_data);
                             p.weights = static_cast<const float*>(d_w);
                             p.flags = static_cast<const uint8_t*>(d_f);
                             p.model = static_cast<const float2*>(d_m);
                             p.model_predicted = in->model ? 0 : 1;
                             if (!in->model) {  // the unweighted 4-correlation model
                               DDS_CHECK_CUDA(ctx, ctx->raw_model.Reserve(
                                                       size_t(ctx->n_dir) * cb.n_vis * 32));
                               const int r2 =
                                   LaunchPredict(ctx, job, ctx->raw_model.as<float2>(), 4);
                               if (r2 != DDSOLVE_OK) return r2;
                               p.model = ctx->raw_model.as<float2>();
                             }
                             p.bl_of_cross = d_x;
                             p.out = reinterpret_cast<float2*>(st);
                             p.n_times = n_t;
                             p.n_bl = n_bl;
                             p.n_ch = n_ch;
                             p.n_bx = n_bx;
                             p.c0 = c0;
                             p.L = L;
                             p.n_dir = ctx->n_dir;
                             p.linear = in->linear_weighting ? 1 : 0;
                             const uint32_t blocks = uint32_t(std::min<uint64_t>(
                                 (cb.n_vis + 255) / 256, uint64_t(ctx->n_sm) * 16));
                             if (ctx->n_corr == 1)
                               weigh_kernel<1><<<blocks, 256, 0, ctx->stream>>>(p);
                             else if (ctx->n_corr == 2)
                               weigh_kernel<2><<<blocks, 256, 0, ctx->stream>>>(p);
                             else
                               weigh_kernel<4><<<blocks, 256, 0, ctx->stream>>>(p);
                             DDS_CHECK_CUDA(ctx, cudaGetLastError());
                             return DDSOLVE_OK;
                           };
                         });
    if (rc != DDSOLVE_OK) return rc;
  }
  // The kernels just enqueued read raw_in; returning after them lets the
  // caller reuse its buffers and keeps raw_in free for the next call.
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return DDSOLVE_OK;
}

int ddsolve_correct_and_subtract(ddsolve_ctx* ctx, const ddsolve_subtract_buffers* in,
                                 const double* solutions, float* data_out,
                                 float* const* models_out) {
  if (!ctx) return DDSOLVE_E_INVALID;
  if (!in || !in->antenna1 || !in->antenna2 || !solutions || in->n_times == 0 ||
      in->n_baselines == 0 || in->n_channels < ctx->n_cb)
    return ctx->Fail(DDSOLVE_E_INVALID, "correct and subtract: NULL pointer or empty interval");
  if (!data_out && !models_out) return DDSOLVE_OK;  // neither subtract nor keepmodel
  if (data_out && !in->data)
    return ctx->Fail(DDSOLVE_E_INVALID, "correct and subtract: subtracting needs the data");
  if (!in->models && (!in->sky || !in->frequencies || !in->station_uvw))
    return ctx->Fail(DDSOLVE_E_INVALID,
                     "correct and subtract: no model and no sky to predict it");
  const uint32_t n_dir = ctx->n_dir;
  for (uint32_t d = 0; d < n_dir; ++d)
    if ((in->models && !in->models[d]) || (models_out && !models_out[d]))
      return ctx->Fail(DDSOLVE_E_INVALID, "correct and subtract: NULL model pointer");
  // DDECal.cc:1085-1090
  if (ctx->n_sub != n_dir)
    return ctx->Fail(DDSOLVE_E_UNSUPPORTED,
                     "Model correction is not implemented for DDECal with direction "
                     "dependent solution intervals");
  for (uint32_t b = 0; b < in->n_baselines; ++b)
    if (in->antenna1[b] >= ctx->n_ant || in->antenna2[b] >= ctx->n_ant)
      return ctx->Fail(DDSOLVE_E_INVALID, "correct and subtract: antenna index out of range");
  cudaSetDevice(ctx->device);
  const uint32_t n_t = in->n_times, n_bl = in->n_baselines, n_ch = in->n_channels;
  const uint64_t n_vis = uint64_t(n_t) * n_bl * n_ch;
  const size_t b_data = n_vis * 32, b_dir = n_vis * 32, b_m = b_dir * n_dir;
  const size_t b_sol = size_t(ctx->n_cb) * ctx->n_ant * n_dir * ctx->n_pol * 16;
  const size_t b_a = size_t(n_bl) * 4, b_ptr = size_t(n_dir) * 8;
  auto align = [](size_t x) { return (x + 255) / 256 * 256; };
  const size_t o_sol = data_out ? align(b_data) : 0, o_a1 = o_sol + align(b_sol);
  const size_t o_a2 = o_a1 + align(b_a), o_pin = o_a2 + align(b_a), o_pout = o_pin + align(b_ptr);
  DDS_CHECK_CUDA(ctx, ctx->raw_in.Reserve(o_pout + align(b_ptr)));
  DDS_CHECK_CUDA(ctx, ctx->raw_model.Reserve(b_m));
  char* base = ctx->raw_in.as<char>();
  char* staged_m = ctx->raw_model.as<char>();
  int rc;
  auto on_device = [&](const void* ptr) {
    cudaPointerAttributes a{};
    const bool dev = cudaPointerGetAttributes(&a, ptr) == cudaSuccess &&
                     a.type == cudaMemoryTypeDevice && a.device == ctx->device;
    cudaGetLastError();
    return dev;
  };
  const void* d_data = nullptr;
  if (data_out && (rc = DeviceView(ctx, in->data, b_data, ctx->raw_in, 0, &d_data)) != DDSOLVE_OK)
    return rc;
  // host solutions travel in the pinned image of the small inputs below
  const bool sol_on_device = on_device(solutions);
  const void* d_sol = sol_on_device ? static_cast<const void*>(solutions) : base + o_sol;
  // Every direction's model: used in place when it is device memory, else
  // staged (or predicted) into direction d's slice of raw_model.
  std::vector<const void*> m_in(n_dir);
  if (in->models) {
    for (uint32_t d = 0; d < n_dir; ++d)
      if ((rc = DeviceView(ctx, in->models[d], b_dir, ctx->raw_model, d * b_dir, &m_in[d])) !=
          DDSOLVE_OK)
        return rc;
  } else {  // the unweighted 4-correlation model of every baseline and channel
    const PredictJob job{n_t, n_bl, n_ch, in->frequencies, in->station_uvw,
                         in->antenna1, in->antenna2, in->sky};
    if ((rc = CheckPredictJob(ctx, job)) != DDSOLVE_OK) return rc;
    if ((rc = LaunchPredict(ctx, job, ctx->raw_model.as<float2>(), 4)) != DDSOLVE_OK) return rc;
    for (uint32_t d = 0; d < n_dir; ++d) m_in[d] = staged_m + d * b_dir;
  }
  // Outputs in device memory are written in place; host outputs go through
  // device memory of the context (the staged data or model slice when that
  // input was staged, else cs_out) and one copy back each.
  const bool data_dev = data_out && on_device(data_out);
  float4* k_data = nullptr;
  if (data_out) {
    if (data_dev)
      k_data = reinterpret_cast<float4*>(data_out);
    else if (d_data == base)
      k_data = reinterpret_cast<float4*>(base);
  }
  std::vector<void*> m_out(models_out ? n_dir : 0, nullptr);
  std::vector<bool> m_out_dev(m_out.size(), false);
  size_t cs_bytes = (data_out && !k_data) ? align(b_data) : 0;
  for (size_t d = 0; d < m_out.size(); ++d) {
    m_out_dev[d] = on_device(models_out[d]);
    if (m_out_dev[d])
      m_out[d] = models_out[d];
    else if (m_in[d] == staged_m + d * b_dir)
      m_out[d] = staged_m + d * b_dir;
    else
      cs_bytes += b_dir;
  }
  if (cs_bytes) {
    DDS_CHECK_CUDA(ctx, ctx->cs_out.Reserve(cs_bytes));
    size_t o = 0;
    if (data_out && !k_data) {
      k_data = ctx->cs_out.as<float4>();
      o = align(b_data);
    }
    for (size_t d = 0; d < m_out.size(); ++d)
      if (!m_out[d]) {
        m_out[d] = ctx->cs_out.as<char>() + o;
        o += b_dir;
      }
  }
  // The small inputs (host solutions, antennas, the per-direction pointer
  // tables) in one pinned image and one copy; the call synchronises before
  // it returns, so the image is free again for the next call.
  const size_t img_lo = sol_on_device ? o_a1 : o_sol, img_hi = o_pout + align(b_ptr);
  DDS_CHECK_CUDA(ctx, ctx->ReserveSmallHost(img_hi - img_lo));
  char* img = static_cast<char*>(ctx->small_host) - img_lo;
  if (!sol_on_device) std::memcpy(img + o_sol, solutions, b_sol);
  std::memcpy(img + o_a1, in->antenna1, b_a);
  std::memcpy(img + o_a2, in->antenna2, b_a);
  std::memcpy(img + o_pin, m_in.data(), b_ptr);
  if (models_out) std::memcpy(img + o_pout, m_out.data(), b_ptr);
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(base + img_lo, img + img_lo, img_hi - img_lo,
                                      cudaMemcpyHostToDevice, ctx->stream));
  CorrectParams p;
  p.data = static_cast<const float4*>(d_data);
  p.model = reinterpret_cast<const float4* const*>(base + o_pin);
  p.data_out = k_data;
  p.model_out = models_out ? reinterpret_cast<float4* const*>(base + o_pout) : nullptr;
  p.solutions = static_cast<const double2*>(d_sol);
  p.a1 = reinterpret_cast<const uint32_t*>(base + o_a1);
  p.a2 = reinterpret_cast<const uint32_t*>(base + o_a2);
  p.n_vis = n_vis;
  p.n_bl = n_bl;
  p.n_ch = n_ch;
  p.n_cb = ctx->n_cb;
  p.n_ant = ctx->n_ant;
  p.n_dir = n_dir;
  const uint32_t blocks =
      uint32_t(std::min<uint64_t>((n_vis + 255) / 256, uint64_t(ctx->n_sm) * 8));
  if (ctx->n_pol == 4)
    correct_subtract_kernel<4><<<blocks, 256, 0, ctx->stream>>>(p);
  else if (ctx->n_pol == 2)
    correct_subtract_kernel<2><<<blocks, 256, 0, ctx->stream>>>(p);
  else
    correct_subtract_kernel<1><<<blocks, 256, 0, ctx->stream>>>(p);
  DDS_CHECK_CUDA(ctx, cudaGetLastError());
  if (data_out && !data_dev)
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(data_out, k_data, b_data, cudaMemcpyDeviceToHost,
                                        ctx->stream));
  for (size_t d = 0; d < m_out.size(); ++d)
    if (!m_out_dev[d])
      DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(models_out[d], m_out[d], b_dir,
                                          cudaMemcpyDeviceToHost, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return DDSOLVE_OK;
}

int ddsolve_predict_regular(ddsolve_ctx* ctx, uint32_t n_times, uint32_t n_baselines,
                            uint32_t n_channels, const double* frequencies,
                            const double* station_uvw, const uint32_t* antenna1,
                            const uint32_t* antenna2, const ddsolve_sky_direction* sky,
                            float* model) {
  if (!ctx) return DDSOLVE_E_INVALID;
  if (n_times == 0 || n_baselines == 0 || n_channels == 0 || !model)
    return ctx->Fail(DDSOLVE_E_INVALID, "predict: empty block or NULL model");
  const PredictJob job{n_times, n_baselines, n_channels, frequencies, station_uvw,
                       antenna1, antenna2, sky};
  int rc = CheckPredictJob(ctx, job);
  if (rc != DDSOLVE_OK) return rc;
  cudaSetDevice(ctx->device);
  const size_t bytes =
      size_t(ctx->n_dir) * n_times * n_baselines * n_channels * ctx->elem_bytes;
  cudaPointerAttributes attr{};
  const bool on_device = cudaPointerGetAttributes(&attr, model) == cudaSuccess &&
                         attr.type == cudaMemoryTypeDevice && attr.device == ctx->device;
  cudaGetLastError();  // a host pointer may leave an error state behind
  float2* out = reinterpret_cast<float2*>(model);
  if (!on_device) {
    DDS_CHECK_CUDA(ctx, ctx->staging.Reserve(bytes));
    out = ctx->staging.as<float2>();
  }
  if ((rc = LaunchPredict(ctx, job, out)) != DDSOLVE_OK) return rc;
  if (!on_device)
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(model, out, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return DDSOLVE_OK;
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
  // put in baseline-diagonal order (see the regular upload); the sums do not
  // depend on the order.
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
    auto diag = [&](uint32_t x) {
      const uint32_t a1 = runs[x].ant & 0xFFFFu, a2 = runs[x].ant >> 16;
      return (a2 + ctx->n_ant - a1) % ctx->n_ant;
    };
    std::stable_sort(members.begin(), members.end(), [&](uint32_t x, uint32_t y) {
      const uint32_t dx = diag(x), dy = diag(y);
      return dx != dy ? dx < dy : (runs[x].ant & 0xFFFFu) < (runs[y].ant & 0xFFFFu);
    });
    HostSlab s;
    s.T = 1;
    s.L = kv.first[0];
    s.R = uint32_t(members.size());
    s.elem_off = off;
    s.src_base = 0;
    s.tstride = 0;
    PadRuns(cb);  // every slab's runs start on a 16-byte boundary
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
  PadRuns(cb);
  if (cb.run_ant.empty()) {
    cb.run_ant.assign(4, 0u);
    cb.run_src.assign(4, 0u);
    cb.run_len.assign(4, 0u);
  }
  return UploadAndPack(ctx, cb, StageCopy(ctx, cb, data, model));
}

}  // extern "C"

namespace {

// The solve of ddsolve_solve (one interval) and ddsolve_solve_batch (every
// interval of the context): results[g] and step_magnitudes[g * cap] per
// interval g.
int SolveImpl(ddsolve_ctx* ctx, double* solutions, ddsolve_result* results,
              double* step_magnitudes) {
  cudaSetDevice(ctx->device);
  int rc;
  bool solve_powers = false;
  if (ctx->n_groups > 1 && !ctx->constraints.empty())
    return ctx->Fail(DDSOLVE_E_UNSUPPORTED,
                     "device constraints apply to single-interval contexts");
  if (ctx->n_pol == 4 && (ctx->n_groups > 1 || !ctx->constraints.empty()))
    return ctx->Fail(DDSOLVE_E_UNSUPPORTED,
                     "the full-Jones solver runs single intervals without device constraints");
  if (ctx->plan_dirty && (rc = BuildPlan(ctx)) != DDSOLVE_OK) return rc;
  const uint32_t n_groups = ctx->n_groups;
  const size_t n_sol = size_t(ctx->n_cb) * ctx->n_ant * ctx->n_sub * ctx->n_pol;
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->d_sol.ptr, solutions, n_sol * sizeof(double2),
                                      cudaMemcpyDefault, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_state.ptr, 0, sizeof(LoopState) * n_groups,
                                      ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_nonfinite.ptr, 1, size_t(ctx->n_cb) * 4,
                                      ctx->stream));
  if (ctx->use_pipe) {
    // Initial MakeSolutionsFinite; later ones are fused into pipe_kernel.
    DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_cb_flag.ptr, 0, size_t(ctx->n_cb) * 4,
                                        ctx->stream));
    DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_cb_done.ptr, 0, size_t(ctx->n_cb) * 4,
                                        ctx->stream));
    DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_counters.ptr, 0, 16, ctx->stream));
    if ((rc = LaunchMakeFinite(ctx, false)) != DDSOLVE_OK) return rc;
    if ((rc = LaunchBuildTables(ctx)) != DDSOLVE_OK) return rc;
    // The model powers are part of solving the interval: a solve recomputes
    // them unless a ddsolve_perform_iteration[s] call computed them on the
    // same data since the last solve, and leaves them stale for the next.
    solve_powers = ctx->use_powers && ctx->powers_dirty;
    if ((rc = LaunchPowers(ctx, false)) != DDSOLVE_OK) return rc;
  }
  // DDSOLVE_NO_GRAPH: host-driven launches, one per kernel (for profilers
  // that do not see kernels inside conditional graph nodes).
  if (!ctx->graph_ok && !std::getenv("DDSOLVE_NO_GRAPH")) {
    rc = BuildGraph(ctx);
    if (rc != DDSOLVE_OK) {
      // Conditional graphs unavailable: fall back to host-driven launches.
      ctx->DestroyGraph();
      cudaGetLastError();
    }
  }
  LoopState ls{};
  std::vector<LoopState> states(n_groups);
  const size_t n_mags = std::max(std::max(ctx->settings.max_iterations,
                                          ctx->settings.min_iterations), 1u);
  DDS_CHECK_CUDA(ctx, ctx->ReserveStage(n_mags));
  bool staged = false;
  if (ctx->graph_ok && n_groups == 1) {
    DDS_CHECK_CUDA(ctx, cudaGraphLaunch(ctx->graph_exec, ctx->stream));
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(&ctx->h_stage->ls, ctx->d_state.ptr, sizeof(ls),
                                        cudaMemcpyDeviceToHost, ctx->stream));
    if (step_magnitudes)
      DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->h_stage->mags, ctx->d_mags.ptr, n_mags * 8,
                                          cudaMemcpyDeviceToHost, ctx->stream));
    if ((rc = StageCounters(ctx)) != DDSOLVE_OK) return rc;
    staged = true;
  } else if (ctx->graph_ok) {
    DDS_CHECK_CUDA(ctx, cudaGraphLaunch(ctx->graph_exec, ctx->stream));
  } else {
    const uint32_t cap = std::max(std::max(ctx->settings.max_iterations,
                                           ctx->settings.min_iterations), 1u);
    for (uint32_t it = 0; it < cap; ++it) {
      if ((rc = LaunchIteration(ctx, false, false, true)) != DDSOLVE_OK) return rc;
      DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(states.data(), ctx->d_state.ptr,
                                          sizeof(LoopState) * n_groups,
                                          cudaMemcpyDeviceToHost, ctx->stream));
      DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
      bool all_done = true;
      for (const LoopState& st : states) all_done = all_done && st.done;
      if (all_done) break;
    }
  }
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(solutions, ctx->d_sol.ptr, n_sol * sizeof(double2),
                                      cudaMemcpyDefault, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (staged) {
    states[0] = ctx->h_stage->ls;
  } else {
    DDS_CHECK_CUDA(ctx, cudaMemcpy(states.data(), ctx->d_state.ptr,
                                   sizeof(LoopState) * n_groups, cudaMemcpyDeviceToHost));
  }
  uint32_t max_it = 0;
  for (uint32_t g = 0; g < n_groups; ++g) {
    const LoopState& st = states[g];
    max_it = std::max(max_it, st.iteration);
    if (!step_magnitudes || st.iteration == 0) continue;
    const size_t n = std::min<size_t>(st.iteration, n_mags);
    if (staged) {
      memcpy(step_magnitudes, ctx->h_stage->mags, n * 8);
    } else {
      DDS_CHECK_CUDA(ctx, cudaMemcpy(step_magnitudes + g * n_mags,
                                     ctx->d_mags.as<double>() + size_t(g) * ctx->mags_stride,
                                     n * 8, cudaMemcpyDeviceToHost));
    }
  }
  // pipe path: make_finite + build_tables (+ power_kernel) + one pipe_kernel
  // per iteration; else three kernels per iteration (full-Jones: make_finite,
  // the pass launches and the finalisation); with device constraints also
  // their kernels and the assignment pass, every iteration
  const uint64_t per_it_cons =
      ctx->constraints.empty() ? 0u : uint64_t(ConstraintLaunches(ctx)) + 1u;
  const uint64_t per_it = ctx->n_pol == 4 ? 2u + FjPassLaunches(ctx) : 3u;
  ctx->last_launches = ctx->use_pipe
                           ? uint64_t(max_it) * (1 + per_it_cons) + 2 + (solve_powers ? 1 : 0)
                           : uint64_t(max_it) * (per_it + per_it_cons);
  // the model powers are fresh for one solve only (see LaunchPowers)
  ctx->powers_dirty = true;
  if ((rc = CheckDeviceError(ctx, staged)) != DDSOLVE_OK) return rc;
  if (results)
    for (uint32_t g = 0; g < n_groups; ++g) {
      // SolverBase::MakeResult (SolverBase.cc:192-213), constraints satisfied.
      const LoopState& st = states[g];
      results[g].iterations = st.has_converged ? st.iteration : st.iteration + 1;
      results[g].constraint_iterations = 0;
      results[g].has_converged = st.has_converged;
      results[g].has_stalled = st.has_stalled;
    }
  return DDSOLVE_OK;
}

}  // namespace

extern "C" {

int ddsolve_solve(ddsolve_ctx* ctx, double* solutions, ddsolve_result* result,
                  double* step_magnitudes) {
  if (!ctx || !solutions) return DDSOLVE_E_INVALID;
  if (ctx->n_groups != 1)
    return ctx->Fail(DDSOLVE_E_STATE,
                     "the context holds several intervals: use ddsolve_solve_batch");
  return SolveImpl(ctx, solutions, result, step_magnitudes);
}

int ddsolve_solve_batch(ddsolve_ctx* ctx, double* solutions, ddsolve_result* results,
                        double* step_magnitudes) {
  if (!ctx || !solutions) return DDSOLVE_E_INVALID;
  return SolveImpl(ctx, solutions, results, step_magnitudes);
}

int ddsolve_set_intervals(ddsolve_ctx* ctx, uint32_t n_intervals,
                          const uint32_t* first_channel_block) {
  if (!ctx || n_intervals == 0) return DDSOLVE_E_INVALID;
  if (n_intervals > 1) {
    if (!first_channel_block || first_channel_block[0] != 0 ||
        first_channel_block[n_intervals] != ctx->n_cb)
      return ctx->Fail(DDSOLVE_E_INVALID, "intervals must cover channel blocks 0..n_cb");
    for (uint32_t g = 0; g < n_intervals; ++g)
      if (first_channel_block[g + 1] <= first_channel_block[g])
        return ctx->Fail(DDSOLVE_E_INVALID, "every interval needs at least one channel block");
  }
  cudaSetDevice(ctx->device);
  ctx->n_groups = n_intervals;
  if (n_intervals > 1)
    ctx->group_first_cb.assign(first_channel_block, first_channel_block + n_intervals + 1);
  else
    ctx->group_first_cb = {0u, ctx->n_cb};
  DDS_CHECK_CUDA(ctx, ctx->d_state.Reserve(sizeof(LoopState) * n_intervals));
  ctx->plan_dirty = true;
  ctx->DestroyGraph();
  return UploadSettings(ctx);
}

int ddsolve_add_smoothness_constraint(ddsolve_ctx* ctx, const ddsolve_smoothness* s) {
  if (!ctx || !s || !s->frequencies) return DDSOLVE_E_INVALID;
  if (!s->weights && !s->sub_solution_weights)
    return ctx->Fail(DDSOLVE_E_INVALID, "smoothness constraint: no weights");
  if (!(s->bandwidth_hz > 0.0) || !std::isfinite(s->bandwidth_hz))
    return ctx->Fail(DDSOLVE_E_INVALID, "smoothness constraint: bandwidth must be positive");
  const uint32_t n = ctx->n_cb, n_ant = ctx->n_ant, n_sub = ctx->n_sub;
  const std::vector<double> f(s->frequencies, s->frequencies + n);
  for (uint32_t i = 1; i < n; ++i)
    if (!(f[i] >= f[i - 1]))
      return ctx->Fail(DDSOLVE_E_INVALID, "smoothness constraint: frequencies must ascend");
  // The band and frequency correction of each output channel block, as
  // KernelSmoother::Smooth (KernelSmoother.h:108-160) walks them.
  const double bw = s->bandwidth_hz;
  std::vector<double> fcorr(n);
  std::vector<uint32_t> band(2 * size_t(n));
  size_t band_left = 0;
  const size_t lbound =
      size_t(std::lower_bound(f.begin(), f.end(), f[0] + bw * 0.5) - f.begin());
  size_t band_right = std::min(lbound + 1, size_t(n));
  for (size_t i = 0; i < n; ++i) {
    size_t start = 0, end = n;
    const double local = s->bandwidth_ref_frequency_hz == 0.0
                             ? bw
                             : bw * f[i] / s->bandwidth_ref_frequency_hz;
    if (s->kernel_truncation) {
      while (band_left < n && f[band_left] < f[i] - local * 0.5) ++band_left;
      while (band_right != n && f[band_right] < f[i] + local * 0.5) ++band_right;
      start = band_left > 0 ? band_left - 1 : 0;
      end = band_right < n ? band_right + 1 : n;
    }
    band[2 * i] = uint32_t(start);
    band[2 * i + 1] = uint32_t(end);
    fcorr[i] = std::pow(local / bw, s->spectral_exponent);
  }
  // Kernel size factor of each (antenna, sub-solution): dd factor / antenna
  // factor (SmoothnessConstraint.cc:82-92).
  std::vector<double> factor(size_t(n_ant) * n_sub);
  for (uint32_t a = 0; a < n_ant; ++a)
    for (uint32_t k = 0; k < n_sub; ++k) {
      const double dd = s->dd_factors ? 1.0 / s->dd_factors[k] : 1.0;
      factor[size_t(a) * n_sub + k] = dd / (s->antenna_factors ? s->antenna_factors[a] : 1.0);
    }
  const bool per_sub = s->sub_solution_weights != nullptr;
  const size_t n_w = size_t(per_sub ? n_sub : 1) * n_ant * n;
  const double* w = per_sub ? s->sub_solution_weights : s->weights;
  ddsolve_ctx::DeviceConstraint c;
  c.kind = DDSOLVE_CONSTRAINT_SMOOTHNESS;
  c.per_sub_weights = per_sub ? 1u : 0u;
  c.bandwidth = bw;
  c.truncate = s->kernel_truncation ? 1 : 0;
  const size_t sizes[5] = {n * 8ull, n * 8ull, 2ull * n * 4, n_w * 8, factor.size() * 8};
  const void* src[5] = {f.data(), fcorr.data(), band.data(), w, factor.data()};
  size_t total = 0;
  for (int k = 0; k < 5; ++k) {
    c.off[k] = total;
    total += (sizes[k] + 15) / 16 * 16;
  }
  cudaSetDevice(ctx->device);
  DDS_CHECK_CUDA(ctx, c.buf.Reserve(total));
  for (int k = 0; k < 5; ++k)
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(c.buf.as<char>() + c.off[k], src[k], sizes[k],
                                        cudaMemcpyHostToDevice, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // pageable sources
  const size_t n_sol = size_t(n) * n_ant * n_sub * ctx->n_pol;
  DDS_CHECK_CUDA(ctx, ctx->d_cons.Reserve(n_sol * sizeof(double2)));
  ctx->constraints.push_back(std::move(c));
  ctx->DestroyGraph();
  return DDSOLVE_OK;
}

int ddsolve_add_antenna_constraint(ddsolve_ctx* ctx, uint32_t n_sets, const uint32_t* set_offsets,
                                   const uint32_t* antennas) {
  if (!ctx || (n_sets > 0 && !set_offsets)) return DDSOLVE_E_INVALID;
  // each set as a std::set: ascending, without repeats
  std::vector<uint32_t> off{0}, members;
  for (uint32_t k = 0; k < n_sets; ++k) {
    if (set_offsets[k + 1] < set_offsets[k] || (set_offsets[k + 1] > set_offsets[k] && !antennas))
      return ctx->Fail(DDSOLVE_E_INVALID, "antenna constraint: bad set offsets");
    std::vector<uint32_t> set(antennas + set_offsets[k], antennas + set_offsets[k + 1]);
    for (uint32_t a : set)
      if (a >= ctx->n_ant) return ctx->Fail(DDSOLVE_E_INVALID, "antenna constraint: bad antenna");
    std::sort(set.begin(), set.end());
    set.erase(std::unique(set.begin(), set.end()), set.end());
    members.insert(members.end(), set.begin(), set.end());
    off.push_back(uint32_t(members.size()));
  }
  ddsolve_ctx::DeviceConstraint c;
  c.kind = DDSOLVE_CONSTRAINT_ANTENNA;
  c.n_sets = n_sets;
  c.off[0] = 0;
  c.off[1] = (off.size() * 4 + 15) / 16 * 16;
  cudaSetDevice(ctx->device);
  DDS_CHECK_CUDA(ctx, c.buf.Reserve(c.off[1] + members.size() * 4 + 16));
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(c.buf.ptr, off.data(), off.size() * 4,
                                      cudaMemcpyHostToDevice, ctx->stream));
  if (!members.empty())
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(c.buf.as<char>() + c.off[1], members.data(),
                                        members.size() * 4, cudaMemcpyHostToDevice,
                                        ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // pageable sources
  ctx->constraints.push_back(std::move(c));
  ctx->DestroyGraph();
  return DDSOLVE_OK;
}

int ddsolve_add_reference_antenna_constraint(ddsolve_ctx* ctx) {
  if (!ctx) return DDSOLVE_E_INVALID;
  cudaSetDevice(ctx->device);
  DDS_CHECK_CUDA(ctx, ctx->d_ref_ant.Reserve(2 * sizeof(uint32_t)));
  ddsolve_ctx::DeviceConstraint c;
  c.kind = DDSOLVE_CONSTRAINT_REFERENCE_ANTENNA;
  ctx->constraints.push_back(std::move(c));
  ctx->DestroyGraph();
  return DDSOLVE_OK;
}

int ddsolve_clear_constraints(ddsolve_ctx* ctx) {
  if (!ctx) return DDSOLVE_E_INVALID;
  ctx->constraints.clear();
  ctx->DestroyGraph();
  return DDSOLVE_OK;
}

int ddsolve_perform_iteration(ddsolve_ctx* ctx, const double* solutions,
                              double* next_solutions) {
  if (!ctx || !solutions || !next_solutions) return DDSOLVE_E_INVALID;
  cudaSetDevice(ctx->device);
  int rc;
  if (ctx->plan_dirty && (rc = BuildPlan(ctx)) != DDSOLVE_OK) return rc;
  bool powers_launched = false;
  const size_t n_sol = size_t(ctx->n_cb) * ctx->n_ant * ctx->n_sub * ctx->n_pol;
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->d_sol.ptr, solutions, n_sol * sizeof(double2),
                                      cudaMemcpyDefault, ctx->stream));
  if (ctx->use_pipe) {
    DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_cb_flag.ptr, 0, size_t(ctx->n_cb) * 4,
                                        ctx->stream));
    DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_cb_done.ptr, 0, size_t(ctx->n_cb) * 4,
                                        ctx->stream));
    DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_counters.ptr, 0, 16, ctx->stream));
    if ((rc = LaunchBuildTables(ctx)) != DDSOLVE_OK) return rc;
    powers_launched = ctx->use_powers && ctx->powers_dirty;
    if ((rc = LaunchPowers(ctx, false)) != DDSOLVE_OK) return rc;
  }
  if ((rc = LaunchIteration(ctx, true, false, false)) != DDSOLVE_OK) return rc;
  DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(next_solutions, ctx->d_next.ptr,
                                      n_sol * sizeof(double2), cudaMemcpyDefault,
                                      ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  // pipe path: build_tables (+ power_kernel) + pipe_kernel; else
  // stream_kernel + finalize_kernel (full-Jones: the pass launches +
  // fj_finalize_kernel)
  ctx->last_launches = ctx->n_pol == 4 ? 1 + FjPassLaunches(ctx)
                       : ctx->use_pipe  ? 2 + (powers_launched ? 1 : 0)
                                        : 2;
  return CheckDeviceError(ctx);
}

int ddsolve_perform_iterations(ddsolve_ctx* ctx, const double* start, uint32_t n_passes,
                               double* outputs) {
  if (!ctx || !start || !outputs || n_passes == 0) return DDSOLVE_E_INVALID;
  cudaSetDevice(ctx->device);
  int rc;
  if (ctx->plan_dirty && (rc = BuildPlan(ctx)) != DDSOLVE_OK) return rc;
  const size_t n_sol = size_t(ctx->n_cb) * ctx->n_ant * ctx->n_sub * ctx->n_pol;
  const size_t bytes = n_sol * sizeof(double2);
  auto on_device = [&](const void* ptr) {
    cudaPointerAttributes attr{};
    const bool dev = cudaPointerGetAttributes(&attr, ptr) == cudaSuccess &&
                     (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) &&
                     attr.device == ctx->device;
    cudaGetLastError();  // unregistered host memory is not an error here
    return dev;
  };
  const bool dev_out = on_device(outputs);
  // Device arrays on this GPU are used in place: the first pass reads `start`
  // (passes never write their input) and every pass writes its slot of
  // `outputs`, unless the two overlap.
  const char* s0 = reinterpret_cast<const char*>(start);
  const char* o0 = reinterpret_cast<const char*>(outputs);
  const bool overlap = s0 < o0 + bytes * n_passes && o0 < s0 + bytes;
  const bool dev_in = !overlap && on_device(start);
  const bool in_place_out = dev_out && !overlap;
  if (!in_place_out) DDS_CHECK_CUDA(ctx, ctx->d_chain.Reserve(bytes * n_passes));
  char* chain = in_place_out ? reinterpret_cast<char*>(outputs) : ctx->d_chain.as<char>();
  if (!dev_in)
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->d_sol.ptr, start, bytes, cudaMemcpyDefault,
                                        ctx->stream));
  uint64_t launches = 0;
  // Pass k reads its solutions from the previous pass's slot of the chain
  // buffer and writes its own slot: the solver's solution buffers are
  // pointed there for the duration of the call (no copies between passes).
  struct Restore {
    ddsolve_ctx* c;
    void *sol, *next;
    ~Restore() {
      c->d_sol.ptr = sol;
      c->d_next.ptr = next;
    }
  } restore{ctx, ctx->d_sol.ptr, ctx->d_next.ptr};
  if (ctx->use_pipe) {
    // Once per call (every pipe_kernel launch leaves its counters at zero;
    // next-solutions passes use none of the solve's non-finite flags).
    DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_counters.ptr, 0, 16, ctx->stream));
  }
  if (dev_in) ctx->d_sol.ptr = const_cast<double*>(start);
  for (uint32_t k = 0; k < n_passes; ++k) {
    if (k > 0) ctx->d_sol.ptr = chain + bytes * (k - 1);
    ctx->d_next.ptr = chain + bytes * k;
    if (ctx->use_pipe) {
      // pass k > 0 uses the gain tables that pass k - 1 wrote from its output
      if (k == 0) {
        if ((rc = LaunchBuildTables(ctx)) != DDSOLVE_OK) return rc;
        if (ctx->use_powers && ctx->powers_dirty) ++launches;
        if ((rc = LaunchPowers(ctx, false)) != DDSOLVE_OK) return rc;
        ++launches;
      }
      ++launches;
    } else {
      launches += 2;
    }
    if ((rc = LaunchIteration(ctx, true, false, false)) != DDSOLVE_OK) return rc;
  }
  if (!in_place_out)
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(outputs, ctx->d_chain.ptr, bytes * n_passes,
                                        cudaMemcpyDefault, ctx->stream));
  ctx->last_launches = launches;
  if (dev_out) return DDSOLVE_OK;  // device outputs: no wait (see the header)
  if ((rc = StageCounters(ctx)) != DDSOLVE_OK) return rc;
  DDS_CHECK_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->last_launches = launches;
  return CheckDeviceError(ctx, true);
}

int ddsolve_time_stream_kernel(ddsolve_ctx* ctx, uint32_t n_launches, float* mean_ms) {
  if (!ctx || !mean_ms || n_launches == 0) return DDSOLVE_E_INVALID;
  cudaSetDevice(ctx->device);
  int rc;
  if (ctx->plan_dirty && (rc = BuildPlan(ctx)) != DDSOLVE_OK) return rc;
  cudaEvent_t a, b;
  DDS_CHECK_CUDA(ctx, cudaEventCreate(&a));
  DDS_CHECK_CUDA(ctx, cudaEventCreate(&b));
  // warm-up launch, then n_launches timed launches of the streaming pass
  // (pipe_kernel in next-solutions mode, stream_kernel alone, or the
  // full-Jones pass and its finalisation).
  if (ctx->n_pol == 4) {
    if ((rc = LaunchIteration(ctx, true, false, false)) != DDSOLVE_OK) return rc;
    DDS_CHECK_CUDA(ctx, cudaEventRecord(a, ctx->stream));
    for (uint32_t i = 0; i < n_launches; ++i)
      if ((rc = LaunchIteration(ctx, true, false, false)) != DDSOLVE_OK) return rc;
  } else if (ctx->use_pipe) {
    DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_cb_flag.ptr, 0, size_t(ctx->n_cb) * 4,
                                        ctx->stream));
    if ((rc = LaunchBuildTables(ctx)) != DDSOLVE_OK) return rc;
    if ((rc = LaunchPowers(ctx, false)) != DDSOLVE_OK) return rc;
    if ((rc = LaunchIteration(ctx, true, false, false)) != DDSOLVE_OK) return rc;
    DDS_CHECK_CUDA(ctx, cudaEventRecord(a, ctx->stream));
    for (uint32_t i = 0; i < n_launches; ++i)
      if ((rc = LaunchIteration(ctx, true, false, false)) != DDSOLVE_OK) return rc;
  } else {
    const StreamParams sp = MakeStreamParams(ctx);
    ctx->stream_fn<<<ctx->n_ctas, kThreads, ctx->stream_smem, ctx->stream>>>(sp);
    DDS_CHECK_CUDA(ctx, cudaEventRecord(a, ctx->stream));
    for (uint32_t i = 0; i < n_launches; ++i)
      ctx->stream_fn<<<ctx->n_ctas, kThreads, ctx->stream_smem, ctx->stream>>>(sp);
  }
  DDS_CHECK_CUDA(ctx, cudaEventRecord(b, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaEventSynchronize(b));
  float ms = 0;
  DDS_CHECK_CUDA(ctx, cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *mean_ms = ms / float(n_launches);
  return CheckDeviceError(ctx);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Autotuner: times the plan variants of the streaming pass on the uploaded
// data and keeps the fastest, cached per process by problem shape (stations,
// directions, correlations, polarizations, and per channel block its
// visibilities, channels and slabs, and the solutions per direction).
// ---------------------------------------------------------------------------
namespace {

struct TuneKey {
  std::vector<uint64_t> v;
  bool operator<(const TuneKey& o) const { return v < o.v; }
};

std::mutex g_tune_mu;
std::map<TuneKey, std::pair<ddsolve_tuning, float>> g_tune_cache;

TuneKey MakeTuneKey(const ddsolve_ctx* ctx) {
  TuneKey k;
  k.v = {ctx->n_ant, ctx->n_dir, ctx->n_corr, ctx->n_pol, ctx->n_cb};
  for (const ChannelBlockStore& cb : ctx->cbs) {
    k.v.push_back(cb.n_elems);
    k.v.push_back(cb.slabs.empty() ? 0 : cb.slabs[0].L);
    k.v.push_back(cb.slabs.size());
  }
  for (uint32_t d = 0; d < ctx->n_dir; ++d) k.v.push_back(ctx->n_sol_per_dir[d]);
  return k;
}

void ApplyTuning(ddsolve_ctx* ctx, const ddsolve_tuning& t) {
  ctx->tune_pipe = t.use_pipe;
  ctx->tune_ng = t.direction_groups;
  ctx->tune_stages = t.stages;
  ctx->tune_powers = t.model_powers;
  ctx->tune_gbuf = t.gain_buffers;
  ctx->plan_dirty = true;
}

ddsolve_tuning CurrentTuning(const ddsolve_ctx* ctx) {
  ddsolve_tuning t;
  t.use_pipe = ctx->tune_pipe;
  t.direction_groups = ctx->tune_ng;
  t.stages = ctx->tune_stages;
  t.model_powers = ctx->tune_powers;
  t.gain_buffers = ctx->tune_gbuf;
  return t;
}

// Mean time of one iteration's kernels in next-solutions mode (pipe_kernel,
// or stream_kernel + finalize_kernel), plus the once-per-solve model powers
// spread over the iteration cap; the plan must be built.
int TimeIteration(ddsolve_ctx* ctx, uint32_t n, float* ms_out) {
  int rc;
  cudaEvent_t a, b, c;
  DDS_CHECK_CUDA(ctx, cudaEventCreate(&a));
  DDS_CHECK_CUDA(ctx, cudaEventCreate(&b));
  DDS_CHECK_CUDA(ctx, cudaEventCreate(&c));
  if (ctx->use_pipe) {
    DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_cb_flag.ptr, 0, size_t(ctx->n_cb) * 4,
                                        ctx->stream));
    DDS_CHECK_CUDA(ctx, cudaMemsetAsync(ctx->d_counters.ptr, 0, 16, ctx->stream));
    if ((rc = LaunchBuildTables(ctx)) != DDSOLVE_OK) return rc;
  }
  DDS_CHECK_CUDA(ctx, cudaEventRecord(c, ctx->stream));
  if ((rc = LaunchPowers(ctx, true)) != DDSOLVE_OK) return rc;
  if ((rc = LaunchIteration(ctx, true, false, false)) != DDSOLVE_OK) return rc;  // warm-up
  DDS_CHECK_CUDA(ctx, cudaEventRecord(a, ctx->stream));
  for (uint32_t i = 0; i < n; ++i)
    if ((rc = LaunchIteration(ctx, true, false, false)) != DDSOLVE_OK) return rc;
  DDS_CHECK_CUDA(ctx, cudaEventRecord(b, ctx->stream));
  DDS_CHECK_CUDA(ctx, cudaEventSynchronize(b));
  float ms = 0.f, first = 0.f;
  DDS_CHECK_CUDA(ctx, cudaEventElapsedTime(&ms, a, b));
  DDS_CHECK_CUDA(ctx, cudaEventElapsedTime(&first, c, a));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaEventDestroy(c);
  if ((rc = CheckDeviceError(ctx)) != DDSOLVE_OK) return rc;
  const float per_it = ms / float(n);
  // `first` = model powers (when used) + one warm-up iteration
  const float powers = std::max(0.f, first - per_it);
  const float cap = float(std::max(ctx->settings.max_iterations, 1u));
  *ms_out = per_it + (ctx->use_pipe && ctx->use_powers ? powers / cap : 0.f);
  return DDSOLVE_OK;
}

}  // namespace

extern "C" {

int ddsolve_get_tuning(const ddsolve_ctx* ctx, ddsolve_tuning* tuning) {
  if (!ctx || !tuning) return DDSOLVE_E_INVALID;
  *tuning = CurrentTuning(ctx);
  return DDSOLVE_OK;
}

int ddsolve_set_plan_tuning(ddsolve_ctx* ctx, const ddsolve_tuning* t) {
  if (!ctx || !t) return DDSOLVE_E_INVALID;
  if (t->use_pipe < -1 || t->use_pipe > 1 || t->model_powers < -1 || t->model_powers > 1 ||
      t->gain_buffers > 2 || t->stages == 1 ||
      (t->direction_groups != 0 &&
       (t->direction_groups > 32 || (t->direction_groups & (t->direction_groups - 1)))))
    return ctx->Fail(DDSOLVE_E_INVALID, "invalid tuning");
  ApplyTuning(ctx, *t);
  return DDSOLVE_OK;
}

int ddsolve_autotune(ddsolve_ctx* ctx, uint32_t launches, ddsolve_tuning* chosen,
                     float* iteration_ms) {
  if (!ctx || launches == 0) return DDSOLVE_E_INVALID;
  cudaSetDevice(ctx->device);
  int rc;
  for (uint32_t c = 0; c < ctx->n_cb; ++c)
    if (!ctx->cbs[c].set) return ctx->Fail(DDSOLVE_E_STATE, "autotune needs uploaded data");
  if (ctx->n_pol == 4) {  // the full-Jones path has one plan: time it
    if ((rc = BuildPlan(ctx)) != DDSOLVE_OK) return rc;
    float ms = 0.f;
    if ((rc = TimeIteration(ctx, launches, &ms)) != DDSOLVE_OK) return rc;
    if (chosen) *chosen = CurrentTuning(ctx);
    if (iteration_ms) *iteration_ms = ms;
    return DDSOLVE_OK;
  }
  const TuneKey key = MakeTuneKey(ctx);
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      ApplyTuning(ctx, it->second.first);
      if ((rc = BuildPlan(ctx)) != DDSOLVE_OK) return rc;
      if (chosen) *chosen = it->second.first;
      if (iteration_ms) *iteration_ms = it->second.second;
      return DDSOLVE_OK;
    }
  }
  // candidates: pipe_kernel plan variants, then stream_kernel lane groups
  std::vector<ddsolve_tuning> cands;
  const bool pipe_ok = (ctx->n_corr == 2 || ctx->n_corr == 4) &&
                       FindPipeKernel(int(ctx->n_corr), int(ctx->n_pol), int(ctx->n_dir));
  if (pipe_ok)
    for (int32_t powers : {0, 1})
      for (uint32_t gbuf : {1u, 2u})
        for (uint32_t stages : {0u, 3u}) cands.push_back({1, 0, stages, powers, gbuf});
  for (uint32_t ng = 1; ng <= 32; ng <<= 1)
    if (FindKernel(int(ctx->n_corr), int(ctx->n_pol), int((ctx->n_dir + ng - 1) / ng)))
      cands.push_back({0, ng, 0, -1, 0});
  // defined solutions for the timed passes
  const size_t n_sol = size_t(ctx->n_cb) * ctx->n_ant * ctx->n_sub * ctx->n_pol;
  std::vector<double> ones(2 * n_sol, 0.0);
  for (size_t i = 0; i < n_sol; ++i) ones[2 * i] = 1.0;
  const ddsolve_tuning before = CurrentTuning(ctx);
  ddsolve_tuning best = before;
  float best_ms = -1.f;
  for (const ddsolve_tuning& c : cands) {
    ApplyTuning(ctx, c);
    if (BuildPlan(ctx) != DDSOLVE_OK) continue;  // variant not applicable
    if (c.use_pipe == 1 && !ctx->use_pipe) continue;
    DDS_CHECK_CUDA(ctx, cudaMemcpyAsync(ctx->d_sol.ptr, ones.data(), n_sol * 16,
                                        cudaMemcpyHostToDevice, ctx->stream));
    float ms = 0.f;
    if ((rc = TimeIteration(ctx, launches, &ms)) != DDSOLVE_OK) return rc;
    if (best_ms < 0.f || ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  if (best_ms < 0.f) {
    ApplyTuning(ctx, before);
    return ctx->Fail(DDSOLVE_E_UNSUPPORTED, "no plan variant could be built");
  }
  ApplyTuning(ctx, best);
  if ((rc = BuildPlan(ctx)) != DDSOLVE_OK) return rc;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[key] = {best, best_ms};
  }
  if (chosen) *chosen = best;
  if (iteration_ms) *iteration_ms = best_ms;
  return DDSOLVE_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free entry point: one direction-iterative pass over regular
// data that the caller already holds in device memory, with the per-antenna
// accumulators in a fixed-size array that lives in the library's own device
// image. Some callers cannot let a library allocate device memory:
// frameworks that hand all device memory out of their own pool or arena (a
// library cudaMalloc would bypass the pool's accounting and could fail once
// the pool holds the device), and hosts whose device memory is already fully
// budgeted. This variant only uses that static array; it never calls
// cudaMalloc, cudaFree or an allocating library routine.
// ---------------------------------------------------------------------------
namespace {

constexpr size_t kNoAllocScratchFloats = size_t(1) << 20;  // 4 MiB
constexpr uint32_t kNoAllocMaxChannelBlocks = 256;
constexpr uint32_t kNoAllocMaxDirections = 64;
constexpr uint32_t kNoAllocMaxChannels = 16;  // channels per block
constexpr uint32_t kNoAllocMaxTimes = 65535;   // grid y dimension
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
  // Invalid pairs are ignored; autocorrelations are dropped, as the regular
  // SolveData constructor drops them (SolveData.cc:100,137).
  if (a1 >= p.n_ant || a2 >= p.n_ant || a1 == a2) return;
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
// device current) and cached for the life of the process. The cache assumes
// the device's primary context is never reset: after cudaDeviceReset the
// cached address is stale.
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
  if (n_times > kNoAllocMaxTimes) {
    // the launch grid's y dimension runs over the time steps
    g_last_error = std::string(who) + "more than 65535 time steps";
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
