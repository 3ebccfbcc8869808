// Learned near-contact correction: a 4-layer MLP (16 -> 128 -> 128 -> 128 -> 16,
// SiLU) evaluated and trained with tcgen05 BF16 tensor-core MMAs (FP32
// accumulators in tensor memory).  The reference has no learned component;
// the network corrects the hydrodynamic force and torque that an
// under-resolved interface (a/dx ~ 5) gives a close pair of spheres, relative
// to a run at twice the resolution.
//
// One CTA of 128 threads processes a tile of 128 rows (samples or pairs).
// Every operand lives in shared memory in one "8x8 blocked" layout: a matrix
// of R rows and C columns (C a multiple of 8) is cut into 8x8 bf16 blocks of
// 128 contiguous bytes (8 rows of 16 bytes), blocks ordered row-group major:
//   byte(r, c) = ((r/8) * (C/8) + c/8) * 128 + (r%8) * 16 + (c%8) * 2.
// That is the canonical no-swizzle core-matrix layout of the UMMA
// descriptors, and the same bytes read as K-major when the row index is M/N
// and as MN-major when the row index is K.  So activations written once by
// the epilogue feed both the next layer (K-major A) and the weight gradient
// (MN-major A or B) with no transposed copies.
//
// Tensor memory: 512 columns x 128 lanes; lane = row of the tile.
//   fwd  Z1 [0,128)  Z2 [128,256)  Z3 [256,384)  O [384,400)
//   bwd  dA3 -> [384,512), dW4^T -> [256,272), dW3^T -> [256,384),
//        dA2 -> [384,512), dW2^T -> [256,384), dA1 -> [384,512), dW1 -> [256,272)
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "particle_kernels.cuh"

namespace kapsel {
namespace nc {

constexpr int IN = 16, HID = 128, OUT = 16, TILE = 128;
// packed FP32 parameter vector
constexpr int OW1 = 0, OB1 = OW1 + HID * IN, OW2 = OB1 + HID, OB2 = OW2 + HID * HID, OW3 = OB2 + HID,
              OB3 = OW3 + HID * HID, OW4 = OB3 + HID, OB4 = OW4 + OUT * HID, NPARAM = OB4 + OUT;
static_assert(NPARAM == 37264, "parameter count");

// shared-memory byte offsets: the 128-column operands first, so that every
// descriptor's reach (up to 60 KB past its start for a 128 x 128 operand)
// stays inside the allocation; the launch reserves the full 227 KB.
constexpr uint32_t S_G = 0, S_A1 = S_G + TILE * HID * 2, S_A2 = S_A1 + TILE * HID * 2, S_A3 = S_A2 + TILE * HID * 2,
                   S_W2 = S_A3 + TILE * HID * 2, S_W3 = S_W2 + HID * HID * 2, S_W1 = S_W3 + HID * HID * 2,
                   S_W4 = S_W1 + HID * IN * 2, S_X = S_W4 + OUT * HID * 2, S_D = S_X + TILE * IN * 2,
                   S_B = S_D + TILE * OUT * 2, S_DB = S_B + (3 * HID + OUT) * 4, S_BAR = S_DB + (3 * HID + OUT) * 4,
                   S_TADDR = S_BAR + 8, S_TOTAL = S_TADDR + 8;
constexpr uint32_t SMEM_ALLOC = 227 * 1024;
static_assert(S_TOTAL <= SMEM_ALLOC, "shared memory");
constexpr uint32_t TMEM_COLS = 512;

constexpr int NC_ETIMEOUT = -7;  // an MMA completion wait ran out (KAPSEL_ETIMEOUT)

__device__ __forceinline__ uint32_t blk(int r, int c, int ncols) {
  return (uint32_t)((((r >> 3) * (ncols >> 3) + (c >> 3)) << 7) + ((r & 7) << 4) + ((c & 7) << 1));
}

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, no swizzle (layout type 0), version 1.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Descriptor of K-slice j (16 deep) of an operand stored blocked with `cols`
// columns.  K-major: rows are M/N, columns K; core matrices 128 B apart along
// K (LBO) and (cols/8)*128 B apart along M/N (SBO).  MN-major: rows are K,
// columns M/N; 128 B apart along M/N (SBO) and (cols/8)*128 B along K (LBO).
__device__ __forceinline__ uint64_t opdesc(uint32_t base, int cols, bool mn_major, int j) {
  const uint32_t rowgrp = (uint32_t)(cols >> 3) * 128u;
  return mn_major ? sdesc(base + (uint32_t)j * 2u * rowgrp, rowgrp, 128u) : sdesc(base + (uint32_t)j * 256u, 128u, rowgrp);
}
// Instruction descriptor: kind::f16 with BF16 A and B, FP32 D, dense.
__device__ __forceinline__ uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ uint64_t gtimer() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait on an mbarrier phase (0.5 s); false when it ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const uint64_t t0 = gtimer();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
    if (gtimer() - t0 > 500000000ull) return false;
  }
}

// Self-check of the bounded wait: one thread waits on an mbarrier that
// nothing arrives at; when the wait gives up (0.5 s) it records
// NC_ETIMEOUT, as the network kernels do, and the kernel returns.
__global__ void k_wait_selfcheck(int *status) {
  __shared__ __align__(8) unsigned long long bar;
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(&bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait(a, 0)) atomicExch(status, NC_ETIMEOUT);
}

// 16 consecutive FP32 columns of this thread's lane.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t *>(&h);
}
// Store 16 FP32 values of row r, columns c0..c0+15, as bf16 into a blocked matrix.
__device__ __forceinline__ void st_row16(unsigned char *sm, uint32_t base, int r, int c0, int ncols, const float *v) {
  uint4 lo = {pack_bf16(v[0], v[1]), pack_bf16(v[2], v[3]), pack_bf16(v[4], v[5]), pack_bf16(v[6], v[7])};
  uint4 hi = {pack_bf16(v[8], v[9]), pack_bf16(v[10], v[11]), pack_bf16(v[12], v[13]), pack_bf16(v[14], v[15])};
  *reinterpret_cast<uint4 *>(sm + base + blk(r, c0, ncols)) = lo;
  *reinterpret_cast<uint4 *>(sm + base + blk(r, c0 + 8, ncols)) = hi;
}

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + __expf(-z)); }

// Convert an FP32 row-major [rows][cols] matrix to the blocked bf16 layout.
__device__ __forceinline__ void load_matrix(unsigned char *sm, uint32_t base, const float *__restrict__ src, int rows,
                                            int cols) {
  const int chunks = rows * cols / 8;
  for (int q = threadIdx.x; q < chunks; q += blockDim.x) {
    const int r = q / (cols / 8), c = (q % (cols / 8)) * 8;
    const float4 f0 = *reinterpret_cast<const float4 *>(src + r * cols + c);
    const float4 f1 = *reinterpret_cast<const float4 *>(src + r * cols + c + 4);
    const uint4 v = {pack_bf16(f0.x, f0.y), pack_bf16(f0.z, f0.w), pack_bf16(f1.x, f1.y), pack_bf16(f1.z, f1.w)};
    *reinterpret_cast<uint4 *>(sm + base + blk(r, c, cols)) = v;
  }
}

// Issue one GEMM D[M][N] (+)= sum_k A[m][k] B[n][k] from one thread.
__device__ __forceinline__ void gemm(uint32_t tmem_d, uint32_t sm0, uint32_t a_off, int a_cols, bool a_mn,
                                     uint32_t b_off, int b_cols, bool b_mn, int M, int N, int K) {
  const uint32_t id = idesc_bf16(M, N, a_mn, b_mn);
  for (int j = 0; j < K / 16; ++j)
    umma(tmem_d, opdesc(sm0 + a_off, a_cols, a_mn, j), opdesc(sm0 + b_off, b_cols, b_mn, j), id, j > 0 ? 1u : 0u);
}

// Column sums over the 128 rows of a tile: warp shuffles, then one shared
// atomic per warp and column.
__device__ __forceinline__ void col_sum16(float *dst, const float *v) {
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    float s = v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(dst + i, s);
  }
}

// Feature and output scaling of a trained network, and its gap range.
struct NcScale {
  float in_shift[IN], in_scale[IN], out_scale[OUT];
  double a;               // sphere radius the network was trained for
  double gap_lo, gap_hi;  // trained surface-gap range in units of a
};

// Pair frame: e1 along the centre line from sphere 1 to sphere 2, e2 =
// normalise(e1 x h) with h = z (or x when e1 is within ~26 deg of z), e3 = e1 x e2.
__host__ __device__ inline void nc_frame(const double d[3], double e[9]) {
  const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  for (int k = 0; k < 3; ++k) e[k] = d[k] / r;
  const double h[3] = {fabs(e[2]) > 0.9 ? 1.0 : 0.0, 0.0, fabs(e[2]) > 0.9 ? 0.0 : 1.0};
  double c[3] = {e[1] * h[2] - e[2] * h[1], e[2] * h[0] - e[0] * h[2], e[0] * h[1] - e[1] * h[0]};
  const double cn = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
  for (int k = 0; k < 3; ++k) e[3 + k] = c[k] / cn;
  e[6] = e[1] * e[5] - e[2] * e[4];
  e[7] = e[2] * e[3] - e[0] * e[5];
  e[8] = e[0] * e[4] - e[1] * e[3];
}

// Network input of a pair: log(gap/a), v2 - v1, omega1, omega2 in the pair
// frame, shifted and scaled; inputs 10..15 are zero.
__host__ __device__ inline void nc_features(const NcScale &sc, double gap, const double e[9], const double v1[3],
                                            const double v2[3], const double w1[3], const double w2[3], float *f) {
  double raw[10];
  raw[0] = log(gap / sc.a);
  for (int k = 0; k < 3; ++k) {
    const double *ek = e + 3 * k;
    raw[1 + k] = (v2[0] - v1[0]) * ek[0] + (v2[1] - v1[1]) * ek[1] + (v2[2] - v1[2]) * ek[2];
    raw[4 + k] = w1[0] * ek[0] + w1[1] * ek[1] + w1[2] * ek[2];
    raw[7 + k] = w2[0] * ek[0] + w2[1] * ek[1] + w2[2] * ek[2];
  }
  for (int i = 0; i < 10; ++i) f[i] = (float)((raw[i] - (double)sc.in_shift[i]) * (double)sc.in_scale[i]);
  for (int i = 10; i < IN; ++i) f[i] = 0.f;
}

// Rows of a tile: sample indices into x/y (optionally through idx), or the
// pair list of the step (count read on the device).
struct TileIO {
  const float *x;      // [n][IN]
  const float *y;      // [n][OUT] targets (training)
  const float *colw;   // [OUT] loss weights (training)
  const int *idx;      // optional row -> sample map
  int n;               // rows, or -1: read *n_dev
  const int *n_dev;
  int n_cap;           // upper bound of *n_dev
  float *out;          // [n][OUT] network output (inference), may be null
  float *grad;         // [NPARAM] accumulated gradient (training)
  float *loss;         // accumulated weighted squared error (training)
  float inv_n;         // 1 / (rows of the whole minibatch)
  int *status;
  // pair list of a step: output rows become force/torque corrections
  const int2 *pairs;   // [n_cap] (i, j)
  const float *frames; // [n_cap][9] e1, e2, e3
  double *corr;        // [Np][6] F, T accumulated per particle
  NcScale sc;
};

// Forward (TRAIN=false) or forward + backward with gradient accumulation.
// Loss = inv_n * sum_rows sum_c colw[c] (O[c] - y[c])^2.
// Inference runs 256 threads: two per row (TMEM lane), each taking half of
// the hidden columns in the epilogues (warps w and w+4 read the same 32
// tensor-memory lanes); training runs 128, one per row.
template <bool TRAIN>
__global__ void __launch_bounds__(TRAIN ? 128 : 256, 1) k_mlp_tile(const float *__restrict__ params, TileIO io) {
  extern __shared__ __align__(128) unsigned char sm[];
  const int t = threadIdx.x, w = t >> 5;
  const int r = t & (TILE - 1);             // row of the tile (TMEM lane)
  const int h = TRAIN ? 0 : t >> 7;          // column half of the epilogues
  constexpr int HC = TRAIN ? HID : HID / 2;  // hidden columns per thread
  const int n = io.n >= 0 ? io.n : min(*io.n_dev, io.n_cap);
  if (blockIdx.x * TILE >= n) return;
  const uint32_t sm0 = smem_u32(sm);
  const uint32_t bar = sm0 + S_BAR;
  float *sb = reinterpret_cast<float *>(sm + S_B);
  float *sdb = reinterpret_cast<float *>(sm + S_DB);

  // ---- weights, biases and the input tile into shared memory
  load_matrix(sm, S_W1, params + OW1, HID, IN);
  load_matrix(sm, S_W2, params + OW2, HID, HID);
  load_matrix(sm, S_W3, params + OW3, HID, HID);
  load_matrix(sm, S_W4, params + OW4, OUT, HID);
  for (int i = t; i < 3 * HID + OUT; i += blockDim.x) {
    const int off = i < HID ? OB1 + i : i < 2 * HID ? OB2 + i - HID : i < 3 * HID ? OB3 + i - 2 * HID : OB4 + i - 3 * HID;
    sb[i] = params[off];
    sdb[i] = 0.f;
  }
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sm0 + S_TADDR),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tm = *reinterpret_cast<volatile uint32_t *>(sm + S_TADDR);
  const uint32_t lane_tm = tm + ((uint32_t)((w & 3) * 32) << 16);  // this warp's 32 lanes
  uint32_t phase = 0;
  bool ok = true;

  // commit the MMAs issued so far and wait for them (all threads)
  auto sync_mma = [&]() -> bool {
    if (t == 0) umma_commit(bar);
    const bool done = mbar_wait(bar, phase & 1u);
    phase += 1;
    tc_fence_after();
    return __syncthreads_and(done) != 0;
  };
  // make generic smem writes and tcgen05.ld reads ordered before the next MMA
  auto to_mma = [&]() {
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  };
  // hidden-layer epilogue: A = silu(Z + b) -> blocked bf16
  auto fwd_hidden = [&](uint32_t zc, const float *b, uint32_t dst) {
    for (int c0 = h * HC; c0 < (h + 1) * HC; c0 += 16) {
      float v[16];
      tmem_ld16(lane_tm + zc + c0, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float z = v[i] + b[c0 + i];
        v[i] = z * sigm(z);
      }
      st_row16(sm, dst, r, c0, HID, v);
    }
  };

  // The CTA loops over row tiles (a grid smaller than the tile count keeps
  // the weights and the tensor memory of one CTA for several tiles): the
  // previous tile's MMAs and tensor-memory reads have all completed when the
  // next tile's input is staged.
  for (int tile = blockIdx.x; ok && tile * TILE < n; tile += gridDim.x) {
  const int row0 = tile * TILE;
  const int row = row0 + r;
  const bool valid = row < n;
  const int src = valid ? (io.idx ? io.idx[row] : row) : 0;
  if (h == 0) {
    float xv[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) xv[i] = valid ? io.x[(size_t)src * IN + i] : 0.f;
    st_row16(sm, S_X, r, 0, IN, xv);
  }
  to_mma();

  // ---- forward
  if (t == 0) { tc_fence_after(); gemm(tm + 0, sm0, S_X, IN, false, S_W1, IN, false, 128, HID, IN); }
  ok = sync_mma();
  if (ok) { fwd_hidden(0, sb, S_A1); to_mma(); }
  if (ok && t == 0) gemm(tm + 128, sm0, S_A1, HID, false, S_W2, HID, false, 128, HID, HID);
  if (ok) ok = sync_mma();
  if (ok) { fwd_hidden(128, sb + HID, S_A2); to_mma(); }
  if (ok && t == 0) gemm(tm + 256, sm0, S_A2, HID, false, S_W3, HID, false, 128, HID, HID);
  if (ok) ok = sync_mma();
  if (ok) { fwd_hidden(256, sb + 2 * HID, S_A3); to_mma(); }
  if (ok && t == 0) gemm(tm + 384, sm0, S_A3, HID, false, S_W4, HID, false, 128, OUT, HID);
  if (ok) ok = sync_mma();
  if (ok && h == 0) {
    float o[16];
    tmem_ld16(lane_tm + 384, o);
#pragma unroll
    for (int i = 0; i < 16; ++i) o[i] += sb[3 * HID + i];
    if (!TRAIN) {
      if (valid && io.out) {
#pragma unroll
        for (int i = 0; i < 16; i += 4)
          *reinterpret_cast<float4 *>(io.out + (size_t)row * OUT + i) = make_float4(o[i], o[i + 1], o[i + 2], o[i + 3]);
      }
      if (valid && io.corr) {
        // [F1, T1, F2, T2] in the pair frame -> box frame, added to both spheres
        const int2 pr = io.pairs[row];
        const float *e = io.frames + (size_t)row * 9;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          double *dst = io.corr + 6 * (size_t)(v < 2 ? pr.x : pr.y) + 3 * (v & 1);
          const double c0 = (double)(o[3 * v] * io.sc.out_scale[3 * v]);
          const double c1 = (double)(o[3 * v + 1] * io.sc.out_scale[3 * v + 1]);
          const double c2 = (double)(o[3 * v + 2] * io.sc.out_scale[3 * v + 2]);
#pragma unroll
          for (int k = 0; k < 3; ++k) atomicAdd(dst + k, c0 * e[k] + c1 * e[3 + k] + c2 * e[6 + k]);
        }
      }
    } else {
      float d[16], l = 0.f;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float e = valid ? o[i] - io.y[(size_t)src * OUT + i] : 0.f;
        l += io.colw[i] * e * e;
        d[i] = 2.f * io.colw[i] * e * io.inv_n;
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) l += __shfl_xor_sync(0xffffffffu, l, off);
      if ((t & 31) == 0) atomicAdd(io.loss, l * io.inv_n);
      col_sum16(sdb + 3 * HID, d);
      st_row16(sm, S_D, t, 0, OUT, d);
    }
  }

  if (TRAIN) {
    // backward epilogue: dZ = dA * silu'(Z + b) -> blocked bf16, bias grads
    auto bwd_hidden = [&](uint32_t dac, uint32_t zc, const float *b, float *db, uint32_t dst) {
      for (int c0 = 0; c0 < HID; c0 += 16) {
        float da[16], z[16];
        tmem_ld16(lane_tm + dac + c0, da);
        tmem_ld16(lane_tm + zc + c0, z);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const float a = z[i] + b[c0 + i], s = sigm(a);
          da[i] *= s * (1.f + a * (1.f - s));
        }
        col_sum16(db + c0, da);
        st_row16(sm, dst, t, c0, HID, da);
      }
    };
    // weight-gradient epilogue: lanes are the rows of the TMEM block
    auto grad_out = [&](uint32_t col, int ncols, float *g, int lane_stride, int col_stride) {
      for (int c0 = 0; c0 < ncols; c0 += 16) {
        float v[16];
        tmem_ld16(lane_tm + col + c0, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) atomicAdd(g + t * lane_stride + (c0 + i) * col_stride, v[i]);
      }
    };
    if (ok) to_mma();
    // dA3 = dO W4
    if (ok && t == 0) gemm(tm + 384, sm0, S_D, OUT, false, S_W4, HID, true, 128, HID, OUT);
    if (ok) ok = sync_mma();
    if (ok) { bwd_hidden(384, 256, sb + 2 * HID, sdb + 2 * HID, S_G); to_mma(); }
    // dW4^T = A3^T dO   (lane = input unit, column = output unit)
    if (ok && t == 0) gemm(tm + 256, sm0, S_A3, HID, true, S_D, OUT, true, 128, OUT, TILE);
    if (ok) ok = sync_mma();
    if (ok) { grad_out(256, OUT, io.grad + OW4, 1, HID); to_mma(); }
    // dW3^T = A2^T dZ3, dA2 = dZ3 W3
    if (ok && t == 0) {
      gemm(tm + 256, sm0, S_A2, HID, true, S_G, HID, true, 128, HID, TILE);
      gemm(tm + 384, sm0, S_G, HID, false, S_W3, HID, true, 128, HID, HID);
    }
    if (ok) ok = sync_mma();
    if (ok) {
      grad_out(256, HID, io.grad + OW3, 1, HID);
      bwd_hidden(384, 128, sb + HID, sdb + HID, S_A3);
      to_mma();
    }
    // dW2^T = A1^T dZ2, dA1 = dZ2 W2
    if (ok && t == 0) {
      gemm(tm + 256, sm0, S_A1, HID, true, S_A3, HID, true, 128, HID, TILE);
      gemm(tm + 384, sm0, S_A3, HID, false, S_W2, HID, true, 128, HID, HID);
    }
    if (ok) ok = sync_mma();
    if (ok) {
      grad_out(256, HID, io.grad + OW2, 1, HID);
      bwd_hidden(384, 0, sb, sdb, S_A2);
      to_mma();
    }
    // dW1 = dZ1^T X   (lane = output unit, column = input)
    if (ok && t == 0) gemm(tm + 256, sm0, S_A2, HID, true, S_X, IN, true, 128, IN, TILE);
    if (ok) ok = sync_mma();
    if (ok) grad_out(256, IN, io.grad + OW1, IN, 1);
    __syncthreads();
    if (ok)
      for (int i = t; i < 3 * HID + OUT; i += blockDim.x) {
        const int off =
            i < HID ? OB1 + i : i < 2 * HID ? OB2 + i - HID : i < 3 * HID ? OB3 + i - 2 * HID : OB4 + i - 3 * HID;
        atomicAdd(io.grad + off, sdb[i]);
        sdb[i] = 0.f;
      }
    __syncthreads();
  }
  }  // tiles

  if (!ok && t == 0) atomicExch(io.status, NC_ETIMEOUT);
  tc_fence_before();
  __syncthreads();
  if (w == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(TMEM_COLS) : "memory");
  }
}

// Near pairs of a step: every pair i < j whose surface gap lies in the
// trained range gets a slot with its features, frame and indices.  Pairs
// beyond `cap` are dropped and flagged with status -6.
__global__ void __launch_bounds__(128) k_nc_pairs(PPar p, const DPart *__restrict__ parts, NcScale sc,
                                                  float *__restrict__ feat, float *__restrict__ frames,
                                                  int2 *__restrict__ pairs, int *__restrict__ count, int cap,
                                                  int *__restrict__ status) {
  const int i = blockIdx.x;
  const DPart &a = parts[i];
  const double lo = sc.gap_lo * sc.a, hi = sc.gap_hi * sc.a;
  // candidates j > i: the neighbour list (sorted; it covers the trained gap
  // range) or all later particles
  const int *lst = p.nbl ? p.nbl + (size_t)i * (NBL_MAX + 1) : nullptr;
  const int ncand = lst ? lst[0] : p.Np - i - 1;
  const int lane = threadIdx.x & 31;
  // every lane of a warp takes the same number of turns, so that the pairs a
  // warp finds take their slots with one atomic per warp
  for (int base = 0; base < ncand; base += blockDim.x) {
    const int t = base + threadIdx.x;
    const int j = t < ncand ? (lst ? lst[1 + t] : i + 1 + t) : -1;
    double d[3], gap = -1.0;
    bool keep = false;
    if (j > i) {
      const DPart &b = parts[j];
      for (int k = 0; k < 3; ++k) {
        d[k] = b.x[k] - a.x[k];
        d[k] -= nint_d(d[k] * p.invL[k]) * p.L[k];
      }
      gap = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) - 2.0 * p.RADIUS;
      keep = gap >= lo && gap <= hi;
    }
    const unsigned found = __ballot_sync(0xffffffffu, keep);
    int first = 0;
    if (lane == 0 && found) first = atomicAdd(count, __popc(found));
    first = __shfl_sync(0xffffffffu, first, 0);
    if (!keep) continue;
    const int s = first + __popc(found & ((1u << lane) - 1u));
    if (s >= cap) {
      atomicExch(status, -6);
      continue;
    }
    const DPart &b = parts[j];
    double e[9];
    nc_frame(d, e);
    nc_features(sc, gap, e, a.v, b.v, a.omega, b.omega, feat + (size_t)s * IN);
    for (int k = 0; k < 9; ++k) frames[(size_t)s * 9 + k] = (float)e[k];
    pairs[s] = make_int2(i, j);
  }
}

// Adam on the packed parameters; clears the gradient.
__global__ void k_adam(float *__restrict__ p, float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       int n, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  g[i] = 0.f;
}

}  // namespace nc
}  // namespace kapsel
