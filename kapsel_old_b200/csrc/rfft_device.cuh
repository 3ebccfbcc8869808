// Two-level register FFT on tiles staged in shared memory.
//
// A line of N = N1*N2 points (N a power of two, 8..256) is transformed as
//   X[k1 + N1 k2] = sum_n2 w_N2^(n2 k2) [ w_N^(n2 k1) sum_n1 x[N2 n1 + n2] w_N1^(n1 k1) ]
// Phase 1: one thread per (line, n2) loads its N1 points into registers,
//          does the N1-point DFT and the twiddle, and writes the result to a
//          shared scratch tile.
// Phase 2: one thread per (line, k1) reads its N2 points back, does the
//          N2-point DFT and writes X in natural order over the input.
// The small DFTs (2, 4, 8, 16 points) are radix-2 networks in registers.
// Sign: w = exp(SIGN * 2 pi i / n); SIGN = +1 is the reference's forward
// transform (fftsg3d.c:108-119), -1 its inverse, both unscaled.
#pragma once

#include "fft_device.cuh"

namespace kapsel {

template <typename R, int SIGN>
__device__ __forceinline__ Cx<R> mul_si(Cx<R> a) {  // a * (SIGN i)
  return SIGN > 0 ? Cx<R>{-a.y, a.x} : Cx<R>{a.y, -a.x};
}

template <typename R, int SIGN>
__device__ __forceinline__ void dft2(Cx<R> *v) {
  const Cx<R> a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <typename R, int SIGN>
__device__ __forceinline__ void dft4(Cx<R> *v) {
  const Cx<R> t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
  const Cx<R> t2 = cadd(v[1], v[3]), t3 = mul_si<R, SIGN>(csub(v[1], v[3]));
  v[0] = cadd(t0, t2);
  v[2] = csub(t0, t2);
  v[1] = cadd(t1, t3);
  v[3] = csub(t1, t3);
}

// exp(SIGN 2 pi i k / 16), k = 0..7, from cos/sin of multiples of pi/8
template <typename R, int SIGN>
__device__ __forceinline__ Cx<R> w16(int k) {
  const R c1 = R(0.92387953251128675613), s1 = R(0.38268343236508977173), h = R(0.70710678118654752440);
  const R cs[8] = {R(1), c1, h, s1, R(0), -s1, -h, -c1};
  const R sn[8] = {R(0), s1, h, c1, R(1), c1, h, s1};
  return {cs[k], R(SIGN) * sn[k]};
}

template <typename R, int SIGN>
__device__ __forceinline__ void dft8(Cx<R> *v) {
  Cx<R> e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
  dft4<R, SIGN>(e);
  dft4<R, SIGN>(o);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const Cx<R> t = k == 0 ? o[0] : cmul(o[k], w16<R, SIGN>(2 * k));
    v[k] = cadd(e[k], t);
    v[k + 4] = csub(e[k], t);
  }
}

template <typename R, int SIGN>
__device__ __forceinline__ void dft16(Cx<R> *v) {
  Cx<R> e[8], o[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    e[i] = v[2 * i];
    o[i] = v[2 * i + 1];
  }
  dft8<R, SIGN>(e);
  dft8<R, SIGN>(o);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const Cx<R> t = k == 0 ? o[0] : cmul(o[k], w16<R, SIGN>(k));
    v[k] = cadd(e[k], t);
    v[k + 8] = csub(e[k], t);
  }
}

template <typename R, int SIGN>
__device__ __forceinline__ void dft_small(Cx<R> *v, int n) {
  switch (n) {
    case 2: dft2<R, SIGN>(v); break;
    case 4: dft4<R, SIGN>(v); break;
    case 8: dft8<R, SIGN>(v); break;
    case 16: dft16<R, SIGN>(v); break;
    default: break;
  }
}

// Factors of a line length: N1 = 2^ceil(log2(N)/2) (at most 16), N2 = N/N1;
// 128-point lines split 8 x 16 (against 16 x 8: the FP64 x passes -2 us
// each, FP32 unchanged).
__device__ __forceinline__ int fft2_n1(int logn) {
  if (logn == 7) return 8;
  const int l1 = (logn + 1) >> 1;
  return 1 << (l1 > 4 ? 4 : l1);
}

// SPLIT = 1 takes the other factorisation of the same length (both factors
// 2..16): 8 = 2 x 4, 16 = 8 x 2, 32 = 4 x 8, 64 = 16 x 4, 128 = 16 x 8;
// 256 has only 16 x 16.  Which one is faster depends on the line count and
// the precision; the batch autotuner times both.
template <int SPLIT>
__device__ __forceinline__ int fft2_n1_sel(int logn) {
  if (SPLIT == 0) return fft2_n1(logn);
  switch (logn) {
    case 3: return 2;
    case 4: return 8;
    case 5: return 4;
    default: return 16;
  }
}

template <int L, typename R, int SIGN>
__device__ __forceinline__ void phase1_item(const Cx<R> *data, Cx<R> *scr, int s, int t, int N, int N2, int nseq,
                                            int ss, int es, const Cx<R> *tw) {
  Cx<R> v[L];
#pragma unroll
  for (int n1 = 0; n1 < L; ++n1) v[n1] = data[s * ss + (N2 * n1 + t) * es];
  dft_small<R, SIGN>(v, L);
#pragma unroll
  for (int k1 = 0; k1 < L; ++k1) {
    Cx<R> x = v[k1];
    if (t * k1) x = cmul(x, twid(tw, t * k1, SIGN));
    scr[(k1 * N2 + t) * nseq + s] = x;
  }
}

template <int L, typename R, int SIGN>
__device__ __forceinline__ void phase2_item(Cx<R> *data, const Cx<R> *scr, int s, int k1, int N1, int nseq, int ss,
                                            int es) {
  Cx<R> y[L];
#pragma unroll
  for (int n2 = 0; n2 < L; ++n2) y[n2] = scr[(k1 * L + n2) * nseq + s];
  dft_small<R, SIGN>(y, L);
#pragma unroll
  for (int k2 = 0; k2 < L; ++k2) data[s * ss + (k1 + N1 * k2) * es] = y[k2];
}

// Transforms NSEQ lines of length 2^logn in place; element e of line s is at
// data[s*ss + e*es]; scr holds at least NSEQ*N values; tw[j] = exp(+2 pi i j/N).
// All threads of the block call it; it ends with a barrier.
// LOGN > 0 fixes the length at compile time (constant indexing and loop
// bounds); LOGN = 0 takes it from logn_rt.
template <typename R, int SIGN, int NSEQ, int LOGN = 0, int SPLIT = 0>
__device__ __forceinline__ void fft2_smem(Cx<R> *data, Cx<R> *scr, int logn_rt, int ss, int es, const Cx<R> *tw) {
  const int logn = LOGN > 0 ? LOGN : logn_rt;
  const int N = 1 << logn;
  const int N1 = fft2_n1_sel<SPLIT>(logn), N2 = N / N1;
  for (int it = threadIdx.x; it < NSEQ * N2; it += blockDim.x) {
    const int s = it % NSEQ, t = it / NSEQ;
    switch (N1) {
      case 2: phase1_item<2, R, SIGN>(data, scr, s, t, N, N2, NSEQ, ss, es, tw); break;
      case 4: phase1_item<4, R, SIGN>(data, scr, s, t, N, N2, NSEQ, ss, es, tw); break;
      case 8: phase1_item<8, R, SIGN>(data, scr, s, t, N, N2, NSEQ, ss, es, tw); break;
      default: phase1_item<16, R, SIGN>(data, scr, s, t, N, N2, NSEQ, ss, es, tw); break;
    }
  }
  __syncthreads();
  for (int it = threadIdx.x; it < NSEQ * N1; it += blockDim.x) {
    const int s = it % NSEQ, k1 = it / NSEQ;
    switch (N2) {
      case 1: phase2_item<1, R, SIGN>(data, scr, s, k1, N1, NSEQ, ss, es); break;
      case 2: phase2_item<2, R, SIGN>(data, scr, s, k1, N1, NSEQ, ss, es); break;
      case 4: phase2_item<4, R, SIGN>(data, scr, s, k1, N1, NSEQ, ss, es); break;
      case 8: phase2_item<8, R, SIGN>(data, scr, s, k1, N1, NSEQ, ss, es); break;
      default: phase2_item<16, R, SIGN>(data, scr, s, k1, N1, NSEQ, ss, es); break;
    }
  }
  __syncthreads();
}

}  // namespace kapsel
