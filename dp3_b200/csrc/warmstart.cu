// Learned warm start: a three-layer perceptron trained and evaluated on the
// B200 tensor cores. The C ABI is in include/ddwarm_b200.h.
//
// Every matrix product is one launch of gemm_kernel<NT>: C = A . B^T for
// A (M x K) and B (N x K), BF16 operands, FP32 accumulation. A CTA owns a
// 128-row tile of C (the 128 lanes of tensor memory) and NT columns; its four
// warps stage 64-wide K chunks of A and B into shared memory in the canonical
// K-major layout without swizzle (8 x 16-byte core matrices, 128 B apart
// along K, 1024 B apart along M/N), double-buffered; one thread issues four
// tcgen05.mma (kind::f16, M = 128, N = NT, K = 16) per chunk and commits them
// to the chunk's mbarrier; the epilogue reads the accumulator with
// tcgen05.ld (32 lanes x 32 columns per warp and instruction) and applies the
// bias / ReLU / ReLU-derivative in FP32. Operands are read through either
// orientation (A(m, k) = a[m * lda + k] or a[k * lda + m]), so the training
// products (dW = dZ^T . H, dH = dZ . W) need no transposed copies.
//
// Waits on mbarriers are bounded (2 s of %globaltimer); a wait that runs out
// sets an error flag, the kernel still waits (bounded) for its in-flight MMAs
// and frees its tensor memory, and the host reports DDSOLVE_E_TIMEOUT.

#include "ddwarm_b200.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <vector>

namespace {

constexpr int kGemmThreads = 128;  // four warps: one quarter of the TMEM lanes each
constexpr int kMTile = 128;        // rows per CTA = tensor-memory lanes
constexpr int kKChunk = 64;        // K per shared-memory stage: four MMAs of K = 16
constexpr unsigned long long kWaitNs = 2000000000ull;

enum Epilogue : int {
  kEpiF32 = 0,       // C fp32 = acc (+ bias)
  kEpiBf16Relu = 1,  // C bf16 = relu(acc + bias)
  kEpiBf16Mask = 2,  // C bf16 = acc where mask > 0, else 0 (ReLU derivative)
};

struct GemmParams {
  const uint16_t* a;  // BF16 bits
  const uint16_t* b;
  void* c;
  const float* bias;     // [N] or null
  const uint16_t* mask;  // [M][ldc] BF16 bits (kEpiBf16Mask)
  unsigned int* error;
  int lda, ldb, ldc;
  int a_trans, b_trans;
  int M, N, K;
  int epilogue;
};

__device__ __forceinline__ uint32_t SmemAddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long GlobalTimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void MbarInit(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(SmemAddr(bar)), "r"(count)
               : "memory");
}

// Bounded wait for the completion of phase `parity` of `bar`.
__device__ __forceinline__ bool MbarWait(uint64_t* bar, uint32_t parity, unsigned int* error) {
  const uint32_t addr = SmemAddr(bar);
  const unsigned long long t0 = GlobalTimer();
  while (true) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(addr), "r"(parity)
        : "memory");
    if (ok) return true;
    if (GlobalTimer() - t0 > kWaitNs) {
      atomicExch(error, 1u);
      return false;
    }
  }
}

// Shared-memory matrix descriptor (tcgen05 format): start address, leading
// (K-direction core matrix) and stride (8-row group) byte offsets, all in
// 16-byte units; bits 46-47 = 1 (descriptor version of sm_100); base offset
// 0; layout type 0 = no swizzle.
__device__ __forceinline__ uint64_t SmemDesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), A
// and B BF16 (bits 7-9 = 1, 10-12 = 1), both K-major (bits 15, 16 = 0),
// N / 8 in bits 17-22, M / 16 in bits 24-28.
__host__ __device__ constexpr uint32_t InstrDesc(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(m >> 4) << 24);
}

// Loads an R x 64 (rows x K) chunk starting at (row0, k0) into the canonical
// K-major layout: element (r, k) at ((r / 8) * 8 + k / 8) * 128 + (r % 8) * 16
// + (k % 8) * 2 bytes. Out-of-range elements are zero. All of a thread's
// 16-byte groups are loaded into registers before any is stored, so that
// their global-memory latencies overlap.
template <int R>
__host__ __device__ constexpr int ChunkGroups() {
  return R * (kKChunk / 8) / kGemmThreads;  // 16-byte groups per thread
}

// Global reads of a chunk (R rows x kKChunk of K) into registers, all of a
// thread's 16-byte groups issued before any is used.
template <int R>
__device__ __forceinline__ void LoadChunkRegs(uint4 (&q)[ChunkGroups<R>()], const uint16_t* src,
                                              int ld, int trans, int rows, int K, int row0,
                                              int k0) {
  static_assert((R * (kKChunk / 8)) % kGemmThreads == 0, "chunk groups must split evenly");
  const bool fast = !trans && (ld & 7) == 0;
#pragma unroll
  for (int i = 0; i < ChunkGroups<R>(); ++i) {
    const int g = threadIdx.x + i * kGemmThreads;
    const int r = g >> 3, kc = g & 7;
    const int row = row0 + r, k = k0 + kc * 8;
    if (fast && row < rows && k + 8 <= K) {
      q[i] = __ldg(reinterpret_cast<const uint4*>(src + size_t(row) * ld + k));
    } else {
      uint16_t v[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const bool in = row < rows && k + j < K;
        v[j] = in ? (trans ? src[size_t(k + j) * ld + row] : src[size_t(row) * ld + k + j]) : 0;
      }
      memcpy(&q[i], v, 16);
    }
  }
}

// The chunk into shared memory in the canonical K-major no-swizzle layout:
// 8x8 core matrices of 128 contiguous bytes, K-adjacent cores 128 B apart,
// 8-row groups 1024 B apart.
template <int R>
__device__ __forceinline__ void StoreChunkRegs(unsigned char* dst,
                                               const uint4 (&q)[ChunkGroups<R>()]) {
#pragma unroll
  for (int i = 0; i < ChunkGroups<R>(); ++i) {
    const int g = threadIdx.x + i * kGemmThreads;
    const int r = g >> 3, kc = g & 7;
    *reinterpret_cast<uint4*>(dst + ((r >> 3) * 8 + kc) * 128 + (r & 7) * 16) = q[i];
  }
}

__device__ __forceinline__ uint16_t ToBf16(float x) {
  const __nv_bfloat16 h = __float2bfloat16_rn(x);
  uint16_t u;
  memcpy(&u, &h, 2);
  return u;
}

__device__ __forceinline__ float FromBf16(uint16_t u) {
  return __uint_as_float(uint32_t(u) << 16);
}

__device__ __forceinline__ void StoreEpilogueRow(const GemmParams& p, int row, int nb,
                                                 bool vec_out, bool vec_mask, float (&v)[32]);

template <int NT>
__global__ void __launch_bounds__(kGemmThreads) gemm_kernel(const GemmParams p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  constexpr uint32_t kABytes = kMTile * kKChunk * 2;  // 16 KB
  constexpr uint32_t kBBytes = NT * kKChunk * 2;
  unsigned char* a_buf = smem;
  unsigned char* b_buf = smem + 2 * kABytes;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + 2 * kABytes + 2 * kBBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kMTile, n0 = blockIdx.y * NT;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     SmemAddr(tmem_slot)),
                 "r"(uint32_t(NT))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    MbarInit(&mbar[0], 1);
    MbarInit(&mbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  const int n_chunks = (p.K + kKChunk - 1) / kKChunk;
  // Chunk c uses buffer c & 1; its MMAs commit to mbar[c & 1], whose phase
  // (c >> 1) & 1 completes when they are done. Every commit is waited for
  // exactly once: before chunk c + 2 reuses the buffer, or after the loop.
  constexpr uint32_t kIdesc = InstrDesc(kMTile, NT);
  // Chunk c + 1's global reads are issued before chunk c's MMAs, so that their
  // latency overlaps the barrier, the MMA issue and the buffer wait.
  uint4 qa[ChunkGroups<kMTile>()], qb[ChunkGroups<NT>()];
  if (n_chunks > 0) {
    LoadChunkRegs<kMTile>(qa, p.a, p.lda, p.a_trans, p.M, p.K, m0, 0);
    LoadChunkRegs<NT>(qb, p.b, p.ldb, p.b_trans, p.N, p.K, n0, 0);
  }
  for (int c = 0; c < n_chunks; ++c) {
    const int b = c & 1;
    if (c >= 2) MbarWait(&mbar[b], uint32_t((c - 2) >> 1) & 1u, p.error);  // chunk c - 2
    StoreChunkRegs<kMTile>(a_buf + b * kABytes, qa);
    StoreChunkRegs<NT>(b_buf + b * kBBytes, qb);
    if (c + 1 < n_chunks) {
      LoadChunkRegs<kMTile>(qa, p.a, p.lda, p.a_trans, p.M, p.K, m0, (c + 1) * kKChunk);
      LoadChunkRegs<NT>(qb, p.b, p.ldb, p.b_trans, p.N, p.K, n0, (c + 1) * kKChunk);
    }
    // generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a_addr = SmemAddr(a_buf + b * kABytes);
      const uint32_t b_addr = SmemAddr(b_buf + b * kBBytes);
#pragma unroll
      for (int s = 0; s < kKChunk / 16; ++s) {
        const uint64_t ad = SmemDesc(a_addr + s * 256, 128, 1024);
        const uint64_t bd = SmemDesc(b_addr + s * 256, 128, 1024);
        const uint32_t acc = (c > 0 || s > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n"
            " setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(kIdesc), "r"(acc)
            : "memory");
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              SmemAddr(&mbar[b]))
          : "memory");
    }
  }
  // All MMAs done (also before freeing tensor memory after a timeout).
  for (int c = n_chunks >= 2 ? n_chunks - 2 : 0; c < n_chunks; ++c)
    MbarWait(&mbar[c & 1], uint32_t(c >> 1) & 1u, p.error);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  // Epilogue: warp w reads TMEM lanes 32w..32w+31 = rows m0 + 32w + lane.
  // 16-byte output (and mask) accesses where every row start is 16-byte
  // aligned: column groups start at multiples of 32 elements.
  const int row = m0 + warp * 32 + lane;
  const int esz = p.epilogue == kEpiF32 ? 4 : 2;
  const bool vec_out = (reinterpret_cast<uintptr_t>(p.c) & 15u) == 0 &&
                       (size_t(p.ldc) * esz) % 16 == 0;
  const bool vec_mask = p.epilogue == kEpiBf16Mask &&
                        (reinterpret_cast<uintptr_t>(p.mask) & 15u) == 0 &&
                        (size_t(p.ldc) * 2) % 16 == 0;
  // Every lane of the warp runs every column group's tcgen05.ld (a
  // .sync.aligned warp-collective): rows beyond M only skip their stores,
  // inside the group, and the warp reconverges before the next load.
  for (int col = 0; col < NT; col += 32) {
    __syncwarp();
    uint32_t r[32];
    const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16) + uint32_t(col);
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
        "%28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    // The group's biases (and masks) are read before any output is written,
    // so that the reads are not serialised behind the stores.
    const int nb = n0 + col;
    float v[32];
#pragma unroll
    for (int j = 0; j < 32; ++j)
      v[j] = __uint_as_float(r[j]) + (p.bias && nb + j < p.N ? __ldg(p.bias + nb + j) : 0.f);
    if (row < p.M) StoreEpilogueRow(p, row, nb, vec_out, vec_mask, v);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(uint32_t(NT))
                 : "memory");
}

// One row's 32-column group of the epilogue: bias already added in v; applies
// the ReLU or the ReLU-derivative mask and stores FP32 or BF16.
__device__ __forceinline__ void StoreEpilogueRow(const GemmParams& p, int row, int nb,
                                                 bool vec_out, bool vec_mask, float (&v)[32]) {
  {  // one output row, columns nb .. nb + 31
    const size_t o0 = size_t(row) * p.ldc + nb;
    const bool full = vec_out && nb + 32 <= p.N;
    if (p.epilogue == kEpiF32) {
      float* out = static_cast<float*>(p.c) + o0;
      if (full) {
#pragma unroll
        for (int j = 0; j < 32; j += 4)
          *reinterpret_cast<float4*>(out + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (nb + j < p.N) out[j] = v[j];
      }
      return;
    }
    if (p.epilogue == kEpiBf16Mask) {  // v = 0 where the mask (ReLU output) is not > 0
      const uint16_t* mk = p.mask + o0;
      if (vec_mask && nb + 32 <= p.N) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const uint4 mv = __ldg(reinterpret_cast<const uint4*>(mk) + q);
          const uint32_t w[4] = {mv.x, mv.y, mv.z, mv.w};
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const uint16_t m = uint16_t(w[e >> 1] >> (16 * (e & 1)));
            if (!(FromBf16(m) > 0.f)) v[q * 8 + e] = 0.f;
          }
        }
      } else {
#pragma unroll
        for (int j = 0; j < 32; ++j)
          if (!(nb + j < p.N && FromBf16(mk[j]) > 0.f)) v[j] = 0.f;
      }
    } else {  // kEpiBf16Relu
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = fmaxf(v[j], 0.f);
    }
    uint16_t* out = static_cast<uint16_t*>(p.c) + o0;
    if (full) {
#pragma unroll
      for (int j = 0; j < 32; j += 8) {
        uint4 w;
        w.x = uint32_t(ToBf16(v[j + 0])) | (uint32_t(ToBf16(v[j + 1])) << 16);
        w.y = uint32_t(ToBf16(v[j + 2])) | (uint32_t(ToBf16(v[j + 3])) << 16);
        w.z = uint32_t(ToBf16(v[j + 4])) | (uint32_t(ToBf16(v[j + 5])) << 16);
        w.w = uint32_t(ToBf16(v[j + 6])) | (uint32_t(ToBf16(v[j + 7])) << 16);
        *reinterpret_cast<uint4*>(out + j) = w;
      }
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (nb + j < p.N) out[j] = ToBf16(v[j]);
    }
  }
}

template <int NT>
constexpr size_t GemmSmem() {
  return 2 * size_t(kMTile) * kKChunk * 2 + 2 * size_t(NT) * kKChunk * 2 + 64;
}

// ---------------------------------------------------------------------------
// Fused forward pass: all three products of the network in one kernel, one
// CTA per 128-row tile. Operands live in global memory pre-tiled in the
// canonical K-major layout of the tensor cores, chunk by chunk:
//   tiled(r, k) = (((k / 64) * (R / 8) + r / 8) * 8 + (k % 64) / 8) * 64
//                 + (r % 8) * 8 + k % 8        (BF16 elements, R rows)
// so that one K-chunk of a 128-row tile (16 KB) or of a whole weight matrix
// (N x 64, N * 128 bytes) is one contiguous block that a single bulk copy
// (cp.async.bulk, no multicast) moves into shared memory in the layout the
// MMA descriptors read. One thread of warp 4 streams the chunks of all three
// layers through a 3-stage ring (layer 1: the input tile and W1; layers 2
// and 3: W2 and W3) and issues tcgen05.mma (M = 128, K = 16) into tensor
// memory: layer 1 at columns 0.., layer 2 at 256.., layer 3 at 0.. again.
// Warps 0-3 run the epilogues: each reads its 32 accumulator lanes
// (tcgen05.ld), adds the bias, applies the ReLU and writes the BF16 hidden
// activations into shared memory in the canonical layout, where the next
// layer's MMAs read them as their A operand; the last epilogue writes the
// FP32 output. Every wait is bounded (kWaitNs) and sets the error flag.
// ---------------------------------------------------------------------------
constexpr int kFusedThreads = 160;  // warps 0-3 epilogue, warp 4 producer / MMA
constexpr int kFusedStages = 3;
constexpr uint32_t kFusedABytes = kMTile * kKChunk * 2;                 // 16 KB input chunk
constexpr uint32_t kFusedStageBytes = kFusedABytes + 256 * kKChunk * 2;  // + 32 KB weights
constexpr uint32_t kFusedHBytes = kMTile * 256 * 2;                     // 64 KB hidden tile
constexpr size_t kFusedSmem = size_t(kFusedStages) * kFusedStageBytes + kFusedHBytes + 128;

__host__ __device__ inline size_t TiledIndex(uint32_t r, uint32_t k, uint32_t rows) {
  return ((size_t(k / 64) * (rows / 8) + r / 8) * 8 + (k % 64) / 8) * 64 + (r % 8) * 8 + k % 8;
}

// The first `rows` rows of a row-major BF16 [..][ld] matrix -> a tiled one of
// layout_rows rows (layout_rows >= rows, a multiple of 8; ld of 64).
__global__ void tile_kernel(const uint16_t* __restrict__ src, uint32_t rows, uint32_t ld,
                            uint16_t* __restrict__ dst, uint32_t layout_rows) {
  const size_t total = size_t(rows) * ld;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += size_t(gridDim.x) * blockDim.x) {
    const uint32_t r = uint32_t(i / ld), k = uint32_t(i % ld);
    dst[TiledIndex(r, k, layout_rows)] = src[i];
  }
}

struct FusedParams {
  const uint16_t* xt;   // input, tiled with rows_pad rows, k1_chunks * 64 columns
  const uint16_t* w1t;  // [dh][k1 * 64] tiled
  const uint16_t* w2t;  // [dh][dh] tiled
  const uint16_t* w3t;  // [dout][dh] tiled
  const float* b1;
  const float* b2;
  const float* b3;
  float* y;  // [M][dout]
  unsigned int* error;
  uint32_t rows_pad, M, k1_chunks, dh, dout;
};

__device__ __forceinline__ void FusedBulkCopy(void* dst, const void* src, uint32_t bytes,
                                              uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
          "r"(SmemAddr(dst)),
      "l"(src), "r"(bytes), "r"(SmemAddr(bar))
      : "memory");
}

__device__ __forceinline__ void MbarArrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(SmemAddr(bar)) : "memory");
}

__device__ __forceinline__ void FusedExpectTx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(SmemAddr(bar)),
               "r"(bytes)
               : "memory");
}

__global__ void __launch_bounds__(kFusedThreads, 1) mlp_forward_kernel(const FusedParams p) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* stages = smem;
  unsigned char* hbuf = smem + size_t(kFusedStages) * kFusedStageBytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(hbuf + kFusedHBytes);
  uint64_t* empty = full + kFusedStages;
  uint64_t* done = empty + kFusedStages;  // one phase per layer's MMAs
  uint64_t* hready = done + 1;            // one phase per hidden tile written
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(hready + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t tile = blockIdx.x;
  const uint32_t h_chunks = p.dh / kKChunk;
  const uint32_t n_steps = p.k1_chunks + 2 * h_chunks;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     SmemAddr(tmem_slot)),
                 "r"(512u)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 128) {
    for (int s = 0; s < kFusedStages; ++s) {
      MbarInit(&full[s], 1);
      MbarInit(&empty[s], 1);
    }
    MbarInit(done, 1);
    MbarInit(hready, 128);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  if (warp == 4) {
    if (lane == 0) {
      // Step j: layer 1 chunks 0..k1-1, then layer 2 and layer 3 chunks.
      auto issue = [&](uint32_t j) {
        unsigned char* st = stages + size_t(j % kFusedStages) * kFusedStageBytes;
        uint64_t* bar = &full[j % kFusedStages];
        if (j < p.k1_chunks) {
          const uint32_t wb = p.dh * kKChunk * 2;
          FusedExpectTx(bar, kFusedABytes + wb);
          // 8-row group g of chunk j starts at element (j * rows_pad / 8 + g) * 512
          FusedBulkCopy(st, p.xt + (size_t(j) * (p.rows_pad / 8) + 16 * tile) * 512,
                        kFusedABytes, bar);
          FusedBulkCopy(st + kFusedABytes, p.w1t + size_t(j) * p.dh * kKChunk, wb, bar);
        } else if (j < p.k1_chunks + h_chunks) {
          const uint32_t c = j - p.k1_chunks, wb = p.dh * kKChunk * 2;
          FusedExpectTx(bar, wb);
          FusedBulkCopy(st + kFusedABytes, p.w2t + size_t(c) * p.dh * kKChunk, wb, bar);
        } else {
          const uint32_t c = j - p.k1_chunks - h_chunks, wb = p.dout * kKChunk * 2;
          FusedExpectTx(bar, wb);
          FusedBulkCopy(st + kFusedABytes, p.w3t + size_t(c) * p.dout * kKChunk, wb, bar);
        }
      };
      for (uint32_t j = 0; j < n_steps && j < uint32_t(kFusedStages); ++j) issue(j);
      bool ok = true;
      for (uint32_t i = 0; i < n_steps && ok; ++i) {
        const uint32_t layer = i < p.k1_chunks ? 1u : (i < p.k1_chunks + h_chunks ? 2u : 3u);
        const uint32_t c = layer == 1 ? i : (layer == 2 ? i - p.k1_chunks
                                                        : i - p.k1_chunks - h_chunks);
        const uint32_t n_chunks = layer == 1 ? p.k1_chunks : h_chunks;
        if (layer > 1 && c == 0) ok = MbarWait(hready, layer - 2, p.error);
        ok = ok && MbarWait(&full[i % kFusedStages], (i / kFusedStages) & 1u, p.error);
        if (!ok) break;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        const unsigned char* st = stages + size_t(i % kFusedStages) * kFusedStageBytes;
        const uint32_t a_addr = layer == 1 ? SmemAddr(st) : SmemAddr(hbuf) + c * kFusedABytes;
        const uint32_t b_addr = SmemAddr(st + kFusedABytes);
        const uint32_t d = tmem + (layer == 2 ? 256u : 0u);
        const uint32_t idesc = InstrDesc(kMTile, int(layer == 3 ? p.dout : p.dh));
#pragma unroll
        for (int s = 0; s < kKChunk / 16; ++s) {
          const uint64_t ad = SmemDesc(a_addr + s * 256, 128, 1024);
          const uint64_t bd = SmemDesc(b_addr + s * 256, 128, 1024);
          const uint32_t acc = (c > 0 || s > 0) ? 1u : 0u;
          asm volatile(
              "{\n .reg .pred p;\n"
              " setp.ne.b32 p, %4, 0;\n"
              " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
              "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
              : "memory");
        }
        asm volatile(
            "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                SmemAddr(&empty[i % kFusedStages]))
            : "memory");
        if (c + 1 == n_chunks)
          asm volatile(
              "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                  SmemAddr(done))
              : "memory");
        if (i + kFusedStages < n_steps) {
          ok = MbarWait(&empty[i % kFusedStages], (i / kFusedStages) & 1u, p.error);
          if (ok) issue(i + kFusedStages);
        }
      }
      // Before returning (also after a timeout): the MMAs already issued
      // have finished, so that tensor memory can be freed.
      for (uint32_t i = n_steps > kFusedStages ? n_steps - kFusedStages : 0; i < n_steps; ++i)
        MbarWait(&empty[i % kFusedStages], (i / kFusedStages) & 1u, p.error);
    }
    __syncwarp();
  } else {
    // Epilogues: warp w owns accumulator lanes / tile rows 32w .. 32w + 31.
    const uint32_t row_in = uint32_t(warp * 32 + lane);
    const uint32_t row = tile * kMTile + row_in;
    for (uint32_t layer = 1; layer <= 3; ++layer) {
      if (!MbarWait(done, (layer - 1) & 1u, p.error)) break;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t ncols = layer == 3 ? p.dout : p.dh;
      const float* bias = layer == 1 ? p.b1 : (layer == 2 ? p.b2 : p.b3);
      const uint32_t base = layer == 2 ? 256u : 0u;
      for (uint32_t col = 0; col < ncols; col += 32) {
        __syncwarp();
        uint32_t r[32];
        const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16) + base + col;
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
            "%10, %11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, "
            "%26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
              "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
              "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
              "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
              "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
              "=r"(r[30]), "=r"(r[31])
            : "r"(taddr)
            : "memory");
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        float v[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]) + __ldg(bias + col + j);
        if (layer < 3) {
          // BF16 ReLU activations into the canonical layout of the next A.
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            uint4 w;
            const int j = q * 8;
            w.x = uint32_t(ToBf16(fmaxf(v[j], 0.f))) |
                  (uint32_t(ToBf16(fmaxf(v[j + 1], 0.f))) << 16);
            w.y = uint32_t(ToBf16(fmaxf(v[j + 2], 0.f))) |
                  (uint32_t(ToBf16(fmaxf(v[j + 3], 0.f))) << 16);
            w.z = uint32_t(ToBf16(fmaxf(v[j + 4], 0.f))) |
                  (uint32_t(ToBf16(fmaxf(v[j + 5], 0.f))) << 16);
            w.w = uint32_t(ToBf16(fmaxf(v[j + 6], 0.f))) |
                  (uint32_t(ToBf16(fmaxf(v[j + 7], 0.f))) << 16);
            const uint32_t k = col + uint32_t(j);
            *reinterpret_cast<uint4*>(hbuf + TiledIndex(row_in, k, kMTile) * 2) = w;
          }
        } else if (row < p.M) {
          float* out = p.y + size_t(row) * p.dout + col;
#pragma unroll
          for (int j = 0; j < 32; j += 4)
            *reinterpret_cast<float4*>(out + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
        }
      }
      if (layer < 3) {
        // generic-proxy writes -> visible to the tensor core; TMEM reads done
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        MbarArrive(hready);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512u)
                 : "memory");
}

// x fp32 [n][n_in] (rows idx[i] if idx) -> bf16 [n][ld] zero-padded; target
// fp32 [n][n_out] -> fp32 [n][ld_t] zero-padded.
__global__ void gather_rows_kernel(const float* __restrict__ x, uint32_t n_in, const uint32_t* idx,
                                   uint32_t n, uint16_t* __restrict__ xb, uint32_t ld,
                                   const float* __restrict__ t, uint32_t n_out,
                                   float* __restrict__ tb, uint32_t ld_t) {
  const uint32_t r = blockIdx.x;
  if (r >= n) return;
  const uint32_t src = idx ? idx[r] : r;
  for (uint32_t j = threadIdx.x; j < ld; j += blockDim.x)
    xb[size_t(r) * ld + j] = ToBf16(j < n_in ? x[size_t(src) * n_in + j] : 0.f);
  if (t)
    for (uint32_t j = threadIdx.x; j < ld_t; j += blockDim.x)
      tb[size_t(r) * ld_t + j] = j < n_out ? t[size_t(src) * n_out + j] : 0.f;
}

// dY = 2 (y - t) / (n * n_out) on the first n_out columns (0 elsewhere), as
// BF16; per-block partial sums of (y - t)^2.
__global__ void loss_grad_kernel(const float* __restrict__ y, const float* __restrict__ t,
                                 uint32_t n, uint32_t n_out, uint32_t ld,
                                 uint16_t* __restrict__ dy, double* __restrict__ partial) {
  __shared__ double s[256];
  double acc = 0.0;
  const float scale = 2.f / (float(n) * float(n_out));
  const size_t total = size_t(n) * ld;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += size_t(gridDim.x) * blockDim.x) {
    const uint32_t col = uint32_t(i % ld);
    float g = 0.f;
    if (col < n_out) {
      const float d = y[i] - t[i];
      acc += double(d) * d;
      g = scale * d;
    }
    dy[i] = ToBf16(g);
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (int(threadIdx.x) < w) s[threadIdx.x] += s[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

__global__ void loss_sum_kernel(const double* __restrict__ partial, uint32_t n_part,
                                double denom, float* __restrict__ loss_out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double s = 0.0;
  for (uint32_t i = 0; i < n_part; ++i) s += partial[i];
  *loss_out = float(s / denom);
}

// Column sums of a BF16 matrix [n][ld] (first `cols` columns) into fp32.
__global__ void col_sum_kernel(const uint16_t* __restrict__ d, uint32_t n, uint32_t ld,
                               uint32_t cols, float* __restrict__ out) {
  const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (uint32_t r = 0; r < n; ++r) s += FromBf16(d[size_t(r) * ld + c]);
  out[c] = s;
}

// Adam on the FP32 masters; refreshes the BF16 copies (padded layouts).
struct AdamParams {
  float* w;
  const float* g;
  float* m;
  float* v;
  uint16_t* wb;  // BF16 copy, or null (biases)
  uint32_t rows, cols, ld;  // master/grad are [rows][ld] padded; bf16 copy same layout
  float lr, b1, b2, eps, c1, c2;  // c1 = 1 - b1^t, c2 = 1 - b2^t
};

__global__ void adam_kernel(const AdamParams a) {
  const size_t total = size_t(a.rows) * a.ld;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < total;
       i += size_t(gridDim.x) * blockDim.x) {
    if (uint32_t(i % a.ld) >= a.cols) continue;  // padding stays zero
    const float g = a.g[i];
    const float m = a.b1 * a.m[i] + (1.f - a.b1) * g;
    const float v = a.b2 * a.v[i] + (1.f - a.b2) * g * g;
    a.m[i] = m;
    a.v[i] = v;
    const float w = a.w[i] - a.lr * (m / a.c1) / (sqrtf(v / a.c2) + a.eps);
    a.w[i] = w;
    if (a.wb) a.wb[i] = ToBf16(w);
  }
}

__global__ void to_bf16_kernel(const float* __restrict__ w, size_t n, uint16_t* __restrict__ wb) {
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += size_t(gridDim.x) * blockDim.x)
    wb[i] = ToBf16(w[i]);
}

constexpr uint32_t kMaxSets = 16;
struct SetPtrs {
  const double2* p[kMaxSets];  // device addresses of the solution sets
};

// Network samples from solution sets (see ddwarm_features); one thread per
// (row, value, set >= 1). Writes FP32 features (x32, ld = n_feat) and / or
// BF16 features (xb: row-major with ld = ldb, or, with tiled_rows > 0, in the
// tiled layout of the fused forward pass with tiled_rows rows).
__global__ void features_kernel(const SetPtrs sets, uint32_t n_sets, uint32_t n_cb,
                                uint32_t n_ant, uint32_t n_sub, uint32_t n_pol, double scale,
                                float* __restrict__ x32, uint16_t* __restrict__ xb,
                                uint32_t ldb, uint32_t tiled_rows) {
  const uint32_t w_n = n_cb * n_pol;
  const uint32_t rows = n_ant * n_sub;
  const size_t total = size_t(rows) * w_n * (n_sets - 1);
  const uint32_t n_feat = 2 * w_n * (n_sets - 1);
  for (size_t t = size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
       t += size_t(gridDim.x) * blockDim.x) {
    const uint32_t w = uint32_t(t % w_n);
    const uint32_t row = uint32_t((t / w_n) % rows);
    const uint32_t k = 1 + uint32_t(t / (size_t(w_n) * rows));
    const uint32_t cb = w / n_pol, pol = w - cb * n_pol;
    const uint32_t ant = row / n_sub, sub = row - ant * n_sub;
    const size_t i = ((size_t(cb) * n_ant + ant) * n_sub + sub) * n_pol + pol;
    const double2 b = sets.p[0][i];
    const double2 v = sets.p[k][i];
    // r = v / b; log r = (log |r|, arg r)
    const double den = b.x * b.x + b.y * b.y;
    const double rr = (v.x * b.x + v.y * b.y) / den;
    const double ri = (v.y * b.x - v.x * b.y) / den;
    double lre = 0.5 * log(rr * rr + ri * ri);
    double lim = atan2(ri, rr);
    if (!isfinite(lre) || !isfinite(lim)) lre = lim = 0.0;
    const uint32_t c = (k - 1) * 2 * w_n + w;
    if (x32) {
      x32[size_t(row) * n_feat + c] = float(scale * lre);
      x32[size_t(row) * n_feat + c + w_n] = float(scale * lim);
    }
    if (xb) {
      const size_t i0 = tiled_rows ? TiledIndex(row, c, tiled_rows) : size_t(row) * ldb + c;
      const size_t i1 =
          tiled_rows ? TiledIndex(row, c + w_n, tiled_rows) : size_t(row) * ldb + c + w_n;
      xb[i0] = ToBf16(float(scale * lre));
      xb[i1] = ToBf16(float(scale * lim));
    }
  }
}

// start = base * exp((y_re + i y_im) / scale); base where not finite.
__global__ void apply_kernel(const double2* __restrict__ base, const float* __restrict__ y,
                             uint32_t ldy, uint32_t n_cb, uint32_t n_ant, uint32_t n_sub,
                             uint32_t n_pol, double scale, double2* __restrict__ start) {
  const uint32_t w_n = n_cb * n_pol;
  const size_t n_sol = size_t(n_cb) * n_ant * n_sub * n_pol;
  for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n_sol;
       i += size_t(gridDim.x) * blockDim.x) {
    const uint32_t pol = uint32_t(i % n_pol);
    const uint32_t sub = uint32_t((i / n_pol) % n_sub);
    const uint32_t ant = uint32_t((i / (size_t(n_pol) * n_sub)) % n_ant);
    const uint32_t cb = uint32_t(i / (size_t(n_pol) * n_sub * n_ant));
    const uint32_t row = ant * n_sub + sub, w = cb * n_pol + pol;
    const double lre = double(y[size_t(row) * ldy + w]) / scale;
    const double lim = double(y[size_t(row) * ldy + w + w_n]) / scale;
    const double m = exp(lre);
    double s, c;
    sincos(lim, &s, &c);
    const double2 b = base[i];
    double2 o = make_double2(m * (b.x * c - b.y * s), m * (b.x * s + b.y * c));
    if (!isfinite(o.x) || !isfinite(o.y)) o = b;
    start[i] = o;
  }
}

struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (ptr) cudaFree(ptr);
  }
  cudaError_t Reserve(size_t n) {
    if (n <= bytes && ptr) return cudaSuccess;
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

uint32_t RoundUp(uint32_t x, uint32_t m) { return (x + m - 1) / m * m; }

}  // namespace

// One layer's parameters in padded device layout: W [rows][ld] (rows = out,
// ld = padded in), b [rows].
struct Layer {
  uint32_t out, in, rows, ld;  // logical out/in, padded rows (out) and ld (in)
  DevBuf w, b, gw, gb, mw, vw, mb, vb, wb;
  DevBuf wt;  // wb in the tiled layout of the fused forward pass
};

struct ddwarm_ctx {
  int device = 0;
  std::string err;
  uint32_t n_in = 0, n_hidden = 0, n_out = 0;
  uint32_t di = 0, dh = 0, dout = 0;  // padded widths
  Layer L[3];
  cudaStream_t stream = nullptr;
  uint64_t adam_t = 0;
  // activations for up to `cap` rows
  uint32_t cap = 0;
  // rows of xb whose padding columns (n_in..di) are known to be zero: every
  // writer of xb either writes whole padded rows with zero padding (the row
  // gathers) or the feature columns only (features_kernel)
  uint32_t xb_zero_rows = 0;
  DevBuf xb, h1, h2, y, t, dy, dz2, dz1, partial, loss, error;
  DevBuf sets, start, x32;  // warm-start features / predictions
  // fused forward pass: the input in the tiled layout, rows padded to 128;
  // xt_zero_rows as xb_zero_rows (features_kernel writes feature columns only)
  DevBuf xt;
  uint32_t xt_rows = 0, xt_zero_rows = 0;
  // training data set
  DevBuf ds_x, ds_t, ds_idx;

  int Fail(int code, const std::string& m) {
    err = m;
    return code;
  }
  cudaStream_t own_stream = nullptr;  // created by the context; `stream` may be a caller's
  ~ddwarm_ctx() {
    if (own_stream) cudaStreamDestroy(own_stream);
  }
};

#define WARM_CHECK(ctx, expr)                                             \
  do {                                                                    \
    const cudaError_t e_ = (expr);                                        \
    if (e_ != cudaSuccess)                                                \
      return (ctx)->Fail(2, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

namespace {

int Reserve(ddwarm_ctx* ctx, uint32_t rows) {
  if (rows <= ctx->cap) return 0;
  const uint32_t r = RoundUp(rows, kMTile);
  WARM_CHECK(ctx, ctx->xb.Reserve(size_t(r) * ctx->di * 2));
  ctx->xb_zero_rows = 0;  // new memory
  WARM_CHECK(ctx, ctx->h1.Reserve(size_t(r) * ctx->dh * 2));
  WARM_CHECK(ctx, ctx->h2.Reserve(size_t(r) * ctx->dh * 2));
  WARM_CHECK(ctx, ctx->y.Reserve(size_t(r) * ctx->dout * 4));
  WARM_CHECK(ctx, ctx->t.Reserve(size_t(r) * ctx->dout * 4));
  WARM_CHECK(ctx, ctx->dy.Reserve(size_t(r) * ctx->dout * 2));
  WARM_CHECK(ctx, ctx->dz2.Reserve(size_t(r) * ctx->dh * 2));
  WARM_CHECK(ctx, ctx->dz1.Reserve(size_t(r) * ctx->dh * 2));
  WARM_CHECK(ctx, ctx->partial.Reserve(256 * 8));
  WARM_CHECK(ctx, ctx->loss.Reserve(8));
  ctx->cap = r;
  return 0;
}

int Gemm(ddwarm_ctx* ctx, const uint16_t* a, int lda, int a_trans, const uint16_t* b, int ldb,
         int b_trans, int M, int N, int K, void* c, int ldc, const float* bias,
         const uint16_t* mask, int epilogue) {
  GemmParams p;
  p.a = a;
  p.b = b;
  p.c = c;
  p.bias = bias;
  p.mask = mask;
  p.error = ctx->error.as<unsigned int>();
  p.lda = lda;
  p.ldb = ldb;
  p.ldc = ldc;
  p.a_trans = a_trans;
  p.b_trans = b_trans;
  p.M = M;
  p.N = N;
  p.K = K;
  p.epilogue = epilogue;
  const uint32_t gm = (uint32_t(M) + kMTile - 1) / kMTile;
  // Wide tiles when there are enough row tiles to fill the GPU; otherwise
  // 64-column tiles spread a small batch over more SMs.
  if (N % 256 == 0 && gm >= 32) {
    dim3 grid(gm, uint32_t(N) / 256);
    gemm_kernel<256><<<grid, kGemmThreads, GemmSmem<256>(), ctx->stream>>>(p);
  } else {
    dim3 grid(gm, (uint32_t(N) + 63) / 64);
    gemm_kernel<64><<<grid, kGemmThreads, GemmSmem<64>(), ctx->stream>>>(p);
  }
  WARM_CHECK(ctx, cudaGetLastError());
  return 0;
}

// Forward pass on the first n rows of ctx->xb: h1, h2 (BF16), y (FP32).
int Forward(ddwarm_ctx* ctx, uint32_t n) {
  int rc;
  Layer& l1 = ctx->L[0];
  Layer& l2 = ctx->L[1];
  Layer& l3 = ctx->L[2];
  if ((rc = Gemm(ctx, ctx->xb.as<uint16_t>(), ctx->di, 0, l1.wb.as<uint16_t>(), l1.ld, 0, n,
                 ctx->dh, ctx->di, ctx->h1.ptr, ctx->dh, l1.b.as<float>(), nullptr,
                 kEpiBf16Relu)))
    return rc;
  if ((rc = Gemm(ctx, ctx->h1.as<uint16_t>(), ctx->dh, 0, l2.wb.as<uint16_t>(), l2.ld, 0, n,
                 ctx->dh, ctx->dh, ctx->h2.ptr, ctx->dh, l2.b.as<float>(), nullptr,
                 kEpiBf16Relu)))
    return rc;
  return Gemm(ctx, ctx->h2.as<uint16_t>(), ctx->dh, 0, l3.wb.as<uint16_t>(), l3.ld, 0, n,
              ctx->dout, ctx->dh, ctx->y.ptr, ctx->dout, l3.b.as<float>(), nullptr, kEpiF32);
}

// Tiled input buffer of the fused forward pass for `rows` rows (padded to
// whole 128-row tiles).
int ReserveTiled(ddwarm_ctx* ctx, uint32_t rows) {
  const uint32_t r = RoundUp(std::max<uint32_t>(rows, 1), kMTile);
  if (r <= ctx->xt_rows) return 0;
  WARM_CHECK(ctx, ctx->xt.Reserve(size_t(r) * ctx->di * 2));
  ctx->xt_rows = r;
  ctx->xt_zero_rows = 0;  // new memory
  return 0;
}

// The BF16 weights in the tiled layout of the fused forward pass (after
// every change of the weights that inference will use).
int RefreshTiled(ddwarm_ctx* ctx) {
  for (Layer& l : ctx->L) {
    WARM_CHECK(ctx, l.wt.Reserve(size_t(l.rows) * l.ld * 2));
    tile_kernel<<<64, 256, 0, ctx->stream>>>(l.wb.as<uint16_t>(), l.rows, l.ld,
                                             l.wt.as<uint16_t>(), l.rows);
  }
  WARM_CHECK(ctx, cudaGetLastError());
  return 0;
}

// Forward pass on the first n rows of ctx->xt (tiled input): y (FP32), one
// launch of mlp_forward_kernel.
int ForwardFused(ddwarm_ctx* ctx, uint32_t n) {
  FusedParams p;
  p.xt = ctx->xt.as<uint16_t>();
  p.w1t = ctx->L[0].wt.as<uint16_t>();
  p.w2t = ctx->L[1].wt.as<uint16_t>();
  p.w3t = ctx->L[2].wt.as<uint16_t>();
  p.b1 = ctx->L[0].b.as<float>();
  p.b2 = ctx->L[1].b.as<float>();
  p.b3 = ctx->L[2].b.as<float>();
  p.y = ctx->y.as<float>();
  p.error = ctx->error.as<unsigned int>();
  p.rows_pad = ctx->xt_rows;
  p.M = n;
  p.k1_chunks = ctx->di / kKChunk;
  p.dh = ctx->dh;
  p.dout = ctx->dout;
  mlp_forward_kernel<<<(n + kMTile - 1) / kMTile, kFusedThreads, kFusedSmem, ctx->stream>>>(p);
  WARM_CHECK(ctx, cudaGetLastError());
  return 0;
}

// Loss and gradients for the first n rows of xb / t (after Forward).
int Backward(ddwarm_ctx* ctx, uint32_t n) {
  int rc;
  Layer& l1 = ctx->L[0];
  Layer& l2 = ctx->L[1];
  Layer& l3 = ctx->L[2];
  const uint32_t blocks = 128;
  loss_grad_kernel<<<blocks, 256, 0, ctx->stream>>>(ctx->y.as<float>(), ctx->t.as<float>(), n,
                                                    ctx->n_out, ctx->dout, ctx->dy.as<uint16_t>(),
                                                    ctx->partial.as<double>());
  loss_sum_kernel<<<1, 32, 0, ctx->stream>>>(ctx->partial.as<double>(), blocks,
                                             double(n) * ctx->n_out, ctx->loss.as<float>());
  WARM_CHECK(ctx, cudaGetLastError());
  // dW3 = dY^T . H2   [dout x dh]
  if ((rc = Gemm(ctx, ctx->dy.as<uint16_t>(), ctx->dout, 1, ctx->h2.as<uint16_t>(), ctx->dh, 1,
                 ctx->dout, ctx->dh, n, l3.gw.ptr, l3.ld, nullptr, nullptr, kEpiF32)))
    return rc;
  // dZ2 = (dY . W3) * [H2 > 0]   [n x dh]
  if ((rc = Gemm(ctx, ctx->dy.as<uint16_t>(), ctx->dout, 0, l3.wb.as<uint16_t>(), l3.ld, 1, n,
                 ctx->dh, ctx->dout, ctx->dz2.ptr, ctx->dh, nullptr, ctx->h2.as<uint16_t>(),
                 kEpiBf16Mask)))
    return rc;
  // dW2 = dZ2^T . H1
  if ((rc = Gemm(ctx, ctx->dz2.as<uint16_t>(), ctx->dh, 1, ctx->h1.as<uint16_t>(), ctx->dh, 1,
                 ctx->dh, ctx->dh, n, l2.gw.ptr, l2.ld, nullptr, nullptr, kEpiF32)))
    return rc;
  // dZ1 = (dZ2 . W2) * [H1 > 0]
  if ((rc = Gemm(ctx, ctx->dz2.as<uint16_t>(), ctx->dh, 0, l2.wb.as<uint16_t>(), l2.ld, 1, n,
                 ctx->dh, ctx->dh, ctx->dz1.ptr, ctx->dh, nullptr, ctx->h1.as<uint16_t>(),
                 kEpiBf16Mask)))
    return rc;
  // dW1 = dZ1^T . X
  if ((rc = Gemm(ctx, ctx->dz1.as<uint16_t>(), ctx->dh, 1, ctx->xb.as<uint16_t>(), ctx->di, 1,
                 ctx->dh, ctx->di, n, l1.gw.ptr, l1.ld, nullptr, nullptr, kEpiF32)))
    return rc;
  col_sum_kernel<<<(ctx->dout + 127) / 128, 128, 0, ctx->stream>>>(
      ctx->dy.as<uint16_t>(), n, ctx->dout, ctx->dout, l3.gb.as<float>());
  col_sum_kernel<<<(ctx->dh + 127) / 128, 128, 0, ctx->stream>>>(
      ctx->dz2.as<uint16_t>(), n, ctx->dh, ctx->dh, l2.gb.as<float>());
  col_sum_kernel<<<(ctx->dh + 127) / 128, 128, 0, ctx->stream>>>(
      ctx->dz1.as<uint16_t>(), n, ctx->dh, ctx->dh, l1.gb.as<float>());
  WARM_CHECK(ctx, cudaGetLastError());
  return 0;
}

int AdamStep(ddwarm_ctx* ctx, float lr) {
  ++ctx->adam_t;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - std::pow(b1, float(ctx->adam_t));
  const float c2 = 1.f - std::pow(b2, float(ctx->adam_t));
  for (Layer& l : ctx->L) {
    AdamParams a{l.w.as<float>(), l.gw.as<float>(), l.mw.as<float>(), l.vw.as<float>(),
                 l.wb.as<uint16_t>(), l.rows, l.in, l.ld, lr, b1, b2, 1e-8f, c1, c2};
    adam_kernel<<<256, 256, 0, ctx->stream>>>(a);
    AdamParams ab{l.b.as<float>(), l.gb.as<float>(), l.mb.as<float>(), l.vb.as<float>(),
                  nullptr, 1, l.out, l.rows, lr, b1, b2, 1e-8f, c1, c2};
    adam_kernel<<<4, 256, 0, ctx->stream>>>(ab);
  }
  WARM_CHECK(ctx, cudaGetLastError());
  return 0;
}

int CheckError(ddwarm_ctx* ctx) {
  unsigned int e = 0;
  WARM_CHECK(ctx, cudaMemcpyAsync(&e, ctx->error.ptr, 4, cudaMemcpyDeviceToHost, ctx->stream));
  WARM_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  if (e) return ctx->Fail(5, "a bounded tensor-core wait timed out; results are invalid");
  return 0;
}

// Host packed (logical) <-> device padded parameter copies.
int CopyParams(ddwarm_ctx* ctx, float* host, bool to_host, bool grads) {
  size_t off = 0;
  std::vector<float> tmp;
  for (Layer& l : ctx->L) {
    DevBuf& w = grads ? l.gw : l.w;
    DevBuf& b = grads ? l.gb : l.b;
    tmp.assign(size_t(l.rows) * l.ld, 0.f);
    if (to_host) {
      WARM_CHECK(ctx, cudaMemcpyAsync(tmp.data(), w.ptr, tmp.size() * 4, cudaMemcpyDeviceToHost,
                                      ctx->stream));
      WARM_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
      for (uint32_t r = 0; r < l.out; ++r)
        memcpy(host + off + size_t(r) * l.in, tmp.data() + size_t(r) * l.ld, size_t(l.in) * 4);
    } else {
      for (uint32_t r = 0; r < l.out; ++r)
        memcpy(tmp.data() + size_t(r) * l.ld, host + off + size_t(r) * l.in, size_t(l.in) * 4);
      WARM_CHECK(ctx, cudaMemcpyAsync(w.ptr, tmp.data(), tmp.size() * 4, cudaMemcpyHostToDevice,
                                      ctx->stream));
      WARM_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
    }
    off += size_t(l.out) * l.in;
    std::vector<float> tb(l.rows, 0.f);
    if (to_host) {
      WARM_CHECK(ctx, cudaMemcpyAsync(tb.data(), b.ptr, tb.size() * 4, cudaMemcpyDeviceToHost,
                                      ctx->stream));
      WARM_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
      memcpy(host + off, tb.data(), size_t(l.out) * 4);
    } else {
      memcpy(tb.data(), host + off, size_t(l.out) * 4);
      WARM_CHECK(ctx, cudaMemcpyAsync(b.ptr, tb.data(), tb.size() * 4, cudaMemcpyHostToDevice,
                                      ctx->stream));
      WARM_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
    }
    off += l.out;
    if (!to_host && !grads) {
      to_bf16_kernel<<<64, 256, 0, ctx->stream>>>(l.w.as<float>(), size_t(l.rows) * l.ld,
                                                  l.wb.as<uint16_t>());
      WARM_CHECK(ctx, cudaGetLastError());
    }
  }
  if (!to_host && !grads) return RefreshTiled(ctx);
  return 0;
}

int Upload(ddwarm_ctx* ctx, DevBuf& dst, const void* src, size_t bytes) {
  WARM_CHECK(ctx, dst.Reserve(bytes));
  WARM_CHECK(ctx, cudaMemcpyAsync(dst.ptr, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
  return 0;
}

}  // namespace

extern "C" {

int ddwarm_create(uint32_t n_in, uint32_t n_hidden, uint32_t n_out, uint64_t seed, int device,
                  ddwarm_ctx** out) {
  if (!out) return 1;
  *out = nullptr;
  if (n_in == 0 || n_in > 1024 || n_out == 0 || n_out > 256 || n_hidden < 64 ||
      n_hidden > 256 || n_hidden % 64)
    return 1;
  int n_dev = 0;
  if (cudaGetDeviceCount(&n_dev) != cudaSuccess || device < 0 || device >= n_dev) return 2;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return 2;
  if (prop.major != 10) return 4;  // tcgen05 needs an sm_100-class device
  auto* ctx = new ddwarm_ctx();
  ctx->device = device;
  cudaSetDevice(device);
  ctx->n_in = n_in;
  ctx->n_hidden = n_hidden;
  ctx->n_out = n_out;
  ctx->di = RoundUp(n_in, 64);
  ctx->dh = n_hidden;
  ctx->dout = RoundUp(n_out, 64);
  const uint32_t outs[3] = {n_hidden, n_hidden, n_out};
  const uint32_t ins[3] = {n_in, n_hidden, n_hidden};
  const uint32_t rows[3] = {ctx->dh, ctx->dh, ctx->dout};
  const uint32_t lds[3] = {ctx->di, ctx->dh, ctx->dh};
  int rc = 0;
  auto fail = [&](int code) {
    delete ctx;
    return code;
  };
  if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(2);
  ctx->stream = ctx->own_stream;
  if (cudaFuncSetAttribute(gemm_kernel<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           int(GemmSmem<256>())) != cudaSuccess ||
      cudaFuncSetAttribute(gemm_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           int(GemmSmem<64>())) != cudaSuccess ||
      cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           int(kFusedSmem)) != cudaSuccess)
    return fail(2);
  std::mt19937_64 rng(seed);
  for (int i = 0; i < 3; ++i) {
    Layer& l = ctx->L[i];
    l.out = outs[i];
    l.in = ins[i];
    l.rows = rows[i];
    l.ld = lds[i];
    const size_t nw = size_t(l.rows) * l.ld;
    for (DevBuf* b : {&l.w, &l.gw, &l.mw, &l.vw})
      if (b->Reserve(nw * 4) != cudaSuccess) return fail(2);
    if (l.wb.Reserve(nw * 2) != cudaSuccess) return fail(2);
    for (DevBuf* b : {&l.b, &l.gb, &l.mb, &l.vb})
      if (b->Reserve(size_t(l.rows) * 4) != cudaSuccess) return fail(2);
    for (DevBuf* b : {&l.w, &l.gw, &l.mw, &l.vw, &l.b, &l.gb, &l.mb, &l.vb})
      cudaMemsetAsync(b->ptr, 0, b->bytes, ctx->stream);
    cudaMemsetAsync(l.wb.ptr, 0, l.wb.bytes, ctx->stream);
  }
  // He-uniform weights (bound sqrt(6 / fan_in)), last layer scaled by 0.1 so
  // that the untrained network predicts small corrections.
  std::vector<float> params(ddwarm_param_count(ctx), 0.f);
  size_t off = 0;
  for (int i = 0; i < 3; ++i) {
    const Layer& l = ctx->L[i];
    const double bound = std::sqrt(6.0 / l.in) * (i == 2 ? 0.1 : 1.0);
    for (size_t k = 0; k < size_t(l.out) * l.in; ++k) {
      const double u = double(rng() >> 11) * (1.0 / 9007199254740992.0);  // [0, 1)
      params[off + k] = float((2.0 * u - 1.0) * bound);
    }
    off += size_t(l.out) * l.in + l.out;
  }
  if (ctx->error.Reserve(16) != cudaSuccess) return fail(2);
  cudaMemsetAsync(ctx->error.ptr, 0, 16, ctx->stream);
  if ((rc = CopyParams(ctx, params.data(), false, false))) return fail(rc);
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return fail(2);
  *out = ctx;
  return 0;
}

void ddwarm_destroy(ddwarm_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  delete ctx;
}

const char* ddwarm_last_error(const ddwarm_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

uint64_t ddwarm_param_count(const ddwarm_ctx* ctx) {
  if (!ctx) return 0;
  uint64_t n = 0;
  for (const Layer& l : ctx->L) n += uint64_t(l.out) * l.in + l.out;
  return n;
}

int ddwarm_get_params(ddwarm_ctx* ctx, float* params) {
  if (!ctx || !params) return 1;
  cudaSetDevice(ctx->device);
  return CopyParams(ctx, params, true, false);
}

int ddwarm_set_params(ddwarm_ctx* ctx, const float* params) {
  if (!ctx || !params) return 1;
  cudaSetDevice(ctx->device);
  ctx->adam_t = 0;
  for (Layer& l : ctx->L)
    for (DevBuf* b : {&l.mw, &l.vw, &l.mb, &l.vb}) cudaMemsetAsync(b->ptr, 0, b->bytes, ctx->stream);
  return CopyParams(ctx, const_cast<float*>(params), false, false);
}

int ddwarm_predict(ddwarm_ctx* ctx, uint32_t n, const float* x, float* y) {
  if (!ctx || (n && (!x || !y))) return 1;
  if (n == 0) return 0;
  cudaSetDevice(ctx->device);
  int rc;
  if ((rc = Reserve(ctx, n))) return rc;
  if ((rc = Upload(ctx, ctx->ds_x, x, size_t(n) * ctx->n_in * 4))) return rc;
  gather_rows_kernel<<<n, 128, 0, ctx->stream>>>(ctx->ds_x.as<float>(), ctx->n_in, nullptr, n,
                                                 ctx->xb.as<uint16_t>(), ctx->di, nullptr, 0,
                                                 nullptr, 0);
  WARM_CHECK(ctx, cudaGetLastError());
  // The fused forward pass (one launch): the input rows tiled first.
  if ((rc = ReserveTiled(ctx, n))) return rc;
  tile_kernel<<<64, 256, 0, ctx->stream>>>(ctx->xb.as<uint16_t>(), n, ctx->di,
                                           ctx->xt.as<uint16_t>(), ctx->xt_rows);
  WARM_CHECK(ctx, cudaGetLastError());
  if ((rc = ForwardFused(ctx, n))) return rc;
  std::vector<float> tmp(size_t(n) * ctx->dout);
  WARM_CHECK(ctx, cudaMemcpyAsync(tmp.data(), ctx->y.ptr, tmp.size() * 4, cudaMemcpyDeviceToHost,
                                  ctx->stream));
  if ((rc = CheckError(ctx))) return rc;
  for (uint32_t r = 0; r < n; ++r)
    memcpy(y + size_t(r) * ctx->n_out, tmp.data() + size_t(r) * ctx->dout, size_t(ctx->n_out) * 4);
  return 0;
}

int ddwarm_gradients(ddwarm_ctx* ctx, uint32_t n, const float* x, const float* target,
                     float* grads, float* loss) {
  if (!ctx || n == 0 || !x || !target || !grads) return 1;
  cudaSetDevice(ctx->device);
  int rc;
  if ((rc = Reserve(ctx, n))) return rc;
  if ((rc = Upload(ctx, ctx->ds_x, x, size_t(n) * ctx->n_in * 4))) return rc;
  if ((rc = Upload(ctx, ctx->ds_t, target, size_t(n) * ctx->n_out * 4))) return rc;
  gather_rows_kernel<<<n, 128, 0, ctx->stream>>>(ctx->ds_x.as<float>(), ctx->n_in, nullptr, n,
                                                 ctx->xb.as<uint16_t>(), ctx->di,
                                                 ctx->ds_t.as<float>(), ctx->n_out,
                                                 ctx->t.as<float>(), ctx->dout);
  WARM_CHECK(ctx, cudaGetLastError());
  if ((rc = Forward(ctx, n))) return rc;
  if ((rc = Backward(ctx, n))) return rc;
  if ((rc = CheckError(ctx))) return rc;
  if ((rc = CopyParams(ctx, grads, true, true))) return rc;
  if (loss) {
    WARM_CHECK(ctx, cudaMemcpyAsync(loss, ctx->loss.ptr, 4, cudaMemcpyDeviceToHost, ctx->stream));
    WARM_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return 0;
}

int ddwarm_trace(ddwarm_ctx* ctx, uint32_t n, const float* x, const float* target,
                 const ddwarm_trace_out* out) {
  if (!ctx || n == 0 || !x || !out) return 1;
  cudaSetDevice(ctx->device);
  int rc;
  if ((rc = Reserve(ctx, n))) return rc;
  if ((rc = Upload(ctx, ctx->ds_x, x, size_t(n) * ctx->n_in * 4))) return rc;
  if (target && (rc = Upload(ctx, ctx->ds_t, target, size_t(n) * ctx->n_out * 4))) return rc;
  gather_rows_kernel<<<n, 128, 0, ctx->stream>>>(
      ctx->ds_x.as<float>(), ctx->n_in, nullptr, n, ctx->xb.as<uint16_t>(), ctx->di,
      target ? ctx->ds_t.as<float>() : nullptr, ctx->n_out, ctx->t.as<float>(), ctx->dout);
  WARM_CHECK(ctx, cudaGetLastError());
  if ((rc = Forward(ctx, n))) return rc;
  if (target && (rc = Backward(ctx, n))) return rc;
  if ((rc = CheckError(ctx))) return rc;
  // Padded device rows [n][ld] -> host [n][cols] FP32.
  auto fetch = [&](const DevBuf& src, bool bf16, uint32_t ld, uint32_t cols, float* dst) {
    if (!dst) return 0;
    const size_t esz = bf16 ? 2 : 4;
    std::vector<unsigned char> tmp(size_t(n) * ld * esz);
    WARM_CHECK(ctx, cudaMemcpyAsync(tmp.data(), src.ptr, tmp.size(), cudaMemcpyDeviceToHost,
                                    ctx->stream));
    WARM_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
    for (uint32_t r = 0; r < n; ++r)
      for (uint32_t c = 0; c < cols; ++c) {
        const size_t i = size_t(r) * ld + c;
        if (bf16) {
          uint16_t u;
          memcpy(&u, tmp.data() + i * 2, 2);
          const uint32_t w = uint32_t(u) << 16;
          memcpy(dst + size_t(r) * cols + c, &w, 4);
        } else {
          memcpy(dst + size_t(r) * cols + c, tmp.data() + i * 4, 4);
        }
      }
    return 0;
  };
  if ((rc = fetch(ctx->xb, true, ctx->di, ctx->n_in, out->xb))) return rc;
  if ((rc = fetch(ctx->h1, true, ctx->dh, ctx->n_hidden, out->h1))) return rc;
  if ((rc = fetch(ctx->h2, true, ctx->dh, ctx->n_hidden, out->h2))) return rc;
  if ((rc = fetch(ctx->y, false, ctx->dout, ctx->n_out, out->y))) return rc;
  if (!target) return 0;
  if ((rc = fetch(ctx->dy, true, ctx->dout, ctx->n_out, out->dy))) return rc;
  if ((rc = fetch(ctx->dz2, true, ctx->dh, ctx->n_hidden, out->dz2))) return rc;
  if ((rc = fetch(ctx->dz1, true, ctx->dh, ctx->n_hidden, out->dz1))) return rc;
  if (out->grads && (rc = CopyParams(ctx, out->grads, true, true))) return rc;
  if (out->loss) {
    WARM_CHECK(ctx, cudaMemcpyAsync(out->loss, ctx->loss.ptr, 4, cudaMemcpyDeviceToHost,
                                    ctx->stream));
    WARM_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return 0;
}

int ddwarm_train(ddwarm_ctx* ctx, uint32_t n, const float* x, const float* target,
                 uint32_t epochs, uint32_t batch, float lr, uint64_t seed, float* epoch_loss) {
  if (!ctx || n == 0 || !x || !target || batch == 0) return 1;
  cudaSetDevice(ctx->device);
  int rc;
  batch = std::min(batch, n);
  if ((rc = Reserve(ctx, batch))) return rc;
  if ((rc = Upload(ctx, ctx->ds_x, x, size_t(n) * ctx->n_in * 4))) return rc;
  if ((rc = Upload(ctx, ctx->ds_t, target, size_t(n) * ctx->n_out * 4))) return rc;
  WARM_CHECK(ctx, ctx->ds_idx.Reserve(size_t(n) * 4));
  DevBuf losses;
  const uint32_t steps_per_epoch = (n + batch - 1) / batch;
  WARM_CHECK(ctx, losses.Reserve(size_t(std::max<uint32_t>(epochs, 1)) * steps_per_epoch * 4));
  std::mt19937_64 rng(seed);
  std::vector<uint32_t> order(n);
  std::iota(order.begin(), order.end(), 0u);
  std::vector<uint32_t> all(size_t(epochs) * n);
  for (uint32_t e = 0; e < epochs; ++e) {
    // Fisher-Yates with explicit draws (no implementation-defined shuffle)
    for (uint32_t i = n - 1; i > 0; --i) {
      const uint32_t j = uint32_t(rng() % (uint64_t(i) + 1));
      std::swap(order[i], order[j]);
    }
    std::copy(order.begin(), order.end(), all.begin() + size_t(e) * n);
  }
  DevBuf idx_all;
  if ((rc = Upload(ctx, idx_all, all.data(), all.size() * 4))) return rc;
  for (uint32_t e = 0; e < epochs; ++e) {
    for (uint32_t s = 0; s < steps_per_epoch; ++s) {
      const uint32_t r0 = s * batch;
      const uint32_t nb = std::min(batch, n - r0);
      gather_rows_kernel<<<nb, 128, 0, ctx->stream>>>(
          ctx->ds_x.as<float>(), ctx->n_in, idx_all.as<uint32_t>() + size_t(e) * n + r0, nb,
          ctx->xb.as<uint16_t>(), ctx->di, ctx->ds_t.as<float>(), ctx->n_out,
          ctx->t.as<float>(), ctx->dout);
      WARM_CHECK(ctx, cudaGetLastError());
      if ((rc = Forward(ctx, nb))) return rc;
      if ((rc = Backward(ctx, nb))) return rc;
      WARM_CHECK(ctx, cudaMemcpyAsync(losses.as<float>() + size_t(e) * steps_per_epoch + s,
                                      ctx->loss.ptr, 4, cudaMemcpyDeviceToDevice, ctx->stream));
      if ((rc = AdamStep(ctx, lr))) return rc;
    }
  }
  if ((rc = RefreshTiled(ctx))) return rc;  // the trained weights for inference
  if ((rc = CheckError(ctx))) return rc;
  if (epoch_loss && epochs) {
    std::vector<float> l(size_t(epochs) * steps_per_epoch);
    WARM_CHECK(ctx, cudaMemcpyAsync(l.data(), losses.ptr, l.size() * 4, cudaMemcpyDeviceToHost,
                                    ctx->stream));
    WARM_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
    for (uint32_t e = 0; e < epochs; ++e) {
      double s = 0.0;
      for (uint32_t k = 0; k < steps_per_epoch; ++k) s += l[size_t(e) * steps_per_epoch + k];
      epoch_loss[e] = float(s / steps_per_epoch);
    }
  }
  return 0;
}

// Device addresses of the solution sets: device memory of this context's
// device is used in place, host memory is staged into ctx->sets.
static int ResolveSets(ddwarm_ctx* ctx, const ddwarm_layout* lay, uint32_t n_sets,
                       const double* const* sets, SetPtrs* out, size_t* n_sol_out) {
  const size_t n_sol = size_t(lay->n_channel_blocks) * lay->n_antennas * lay->n_sub * lay->n_pol;
  WARM_CHECK(ctx, ctx->sets.Reserve(n_sol * 16 * n_sets));
  for (uint32_t k = 0; k < n_sets; ++k) {
    cudaPointerAttributes attr{};
    const bool dev = cudaPointerGetAttributes(&attr, sets[k]) == cudaSuccess &&
                     (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) &&
                     attr.device == ctx->device;
    cudaGetLastError();  // unregistered host memory is not an error here
    if (dev) {
      out->p[k] = reinterpret_cast<const double2*>(sets[k]);
    } else {
      char* dst = ctx->sets.as<char>() + n_sol * 16 * k;
      WARM_CHECK(ctx, cudaMemcpyAsync(dst, sets[k], n_sol * 16, cudaMemcpyHostToDevice,
                                      ctx->stream));
      out->p[k] = reinterpret_cast<const double2*>(dst);
    }
  }
  *n_sol_out = n_sol;
  return 0;
}

static bool BadLayout(const ddwarm_layout* lay, uint32_t n_sets, const double* const* sets) {
  if (!lay || !sets || n_sets < 2 || n_sets > kMaxSets) return true;
  if (!lay->n_channel_blocks || !lay->n_antennas || !lay->n_sub || !lay->n_pol) return true;
  if (!(lay->scale > 0.0)) return true;
  for (uint32_t k = 0; k < n_sets; ++k)
    if (!sets[k]) return true;
  return false;
}

int ddwarm_features(ddwarm_ctx* ctx, const ddwarm_layout* lay, uint32_t n_sets,
                    const double* const* sets, float* x) {
  if (!ctx || !x || BadLayout(lay, n_sets, sets)) return 1;
  cudaSetDevice(ctx->device);
  int rc;
  size_t n_sol = 0;
  SetPtrs sp{};
  if ((rc = ResolveSets(ctx, lay, n_sets, sets, &sp, &n_sol))) return rc;
  const size_t rows = size_t(lay->n_antennas) * lay->n_sub;
  const size_t n_feat = size_t(2) * lay->n_channel_blocks * lay->n_pol * (n_sets - 1);
  WARM_CHECK(ctx, ctx->x32.Reserve(rows * n_feat * 4));
  features_kernel<<<256, 256, 0, ctx->stream>>>(sp, n_sets, lay->n_channel_blocks,
                                                lay->n_antennas, lay->n_sub, lay->n_pol,
                                                lay->scale, ctx->x32.as<float>(), nullptr, 0,
                                                0);
  WARM_CHECK(ctx, cudaGetLastError());
  WARM_CHECK(ctx, cudaMemcpyAsync(x, ctx->x32.ptr, rows * n_feat * 4, cudaMemcpyDefault,
                                  ctx->stream));
  WARM_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  return 0;
}

int ddwarm_predict_start(ddwarm_ctx* ctx, const ddwarm_layout* lay, uint32_t n_sets,
                         const double* const* sets, double* start) {
  if (!ctx || !start || BadLayout(lay, n_sets, sets)) return 1;
  const uint32_t w_n = lay->n_channel_blocks * lay->n_pol;
  if (ctx->n_in != 2 * w_n * (n_sets - 1) || ctx->n_out != 2 * w_n)
    return ctx->Fail(1, "network shape does not match the layout and the number of sets");
  cudaSetDevice(ctx->device);
  int rc;
  size_t n_sol = 0;
  const uint32_t rows = lay->n_antennas * lay->n_sub;
  if ((rc = Reserve(ctx, rows))) return rc;
  SetPtrs sp{};
  if ((rc = ResolveSets(ctx, lay, n_sets, sets, &sp, &n_sol))) return rc;
  if ((rc = ReserveTiled(ctx, rows))) return rc;
  if (rows > ctx->xt_zero_rows) {  // zero padding once per allocation
    WARM_CHECK(ctx, cudaMemsetAsync(ctx->xt.ptr, 0, ctx->xt.bytes, ctx->stream));
    ctx->xt_zero_rows = ctx->xt_rows;
  }
  features_kernel<<<256, 256, 0, ctx->stream>>>(sp, n_sets, lay->n_channel_blocks,
                                                lay->n_antennas, lay->n_sub, lay->n_pol,
                                                lay->scale, nullptr, ctx->xt.as<uint16_t>(),
                                                0, ctx->xt_rows);
  WARM_CHECK(ctx, cudaGetLastError());
  if ((rc = ForwardFused(ctx, rows))) return rc;
  cudaPointerAttributes attr{};
  const bool dev_out = cudaPointerGetAttributes(&attr, start) == cudaSuccess &&
                       (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged) &&
                       attr.device == ctx->device;
  cudaGetLastError();
  double2* out = reinterpret_cast<double2*>(start);
  if (!dev_out) {
    WARM_CHECK(ctx, ctx->start.Reserve(n_sol * 16));
    out = ctx->start.as<double2>();
  }
  apply_kernel<<<256, 256, 0, ctx->stream>>>(sp.p[0], ctx->y.as<float>(), ctx->dout,
                                             lay->n_channel_blocks, lay->n_antennas, lay->n_sub,
                                             lay->n_pol, lay->scale, out);
  WARM_CHECK(ctx, cudaGetLastError());
  if (!dev_out) {
    WARM_CHECK(ctx, cudaMemcpyAsync(start, out, n_sol * 16, cudaMemcpyDeviceToHost, ctx->stream));
    return CheckError(ctx);
  }
  return 0;  // device output: no wait (see the header)
}

int ddwarm_set_stream(ddwarm_ctx* ctx, void* stream) {
  if (!ctx) return 1;
  cudaSetDevice(ctx->device);
  WARM_CHECK(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
  return 0;
}

}  // extern "C"
