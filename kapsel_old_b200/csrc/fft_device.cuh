// Shared-memory FFT building blocks for the pruned 3D real transforms.
//
// The reference transforms a whole NX*NY*NZ_ field with Ooura's row-column
// rdft3d (fftsg3d.c:560-642) behind A2a_k / A_k2a (fft_wrapper.h:432-631).
// Here a 3D transform is split into three batched 1D passes (x, y, z); each
// pass stages a tile of lines in shared memory and runs an in-place
// decimation-in-time FFT on it: bit-reversed load, one radix-2 stage when
// log2(N) is odd, then merged radix-2^2 (radix-4) stages, one barrier per
// stage.  The sign convention is the reference's: forward exp(+i theta),
// inverse exp(-i theta), no scaling (the 1/N of A_k2a is applied by the
// caller at the real-space end).
#pragma once

#include <cuda_runtime.h>

namespace kapsel {

template <typename R>
struct alignas(2 * sizeof(R)) Cx {
  R x, y;
};

template <typename R>
__device__ __forceinline__ Cx<R> cmul(Cx<R> a, Cx<R> b) {
  return {a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x};
}
template <typename R>
__device__ __forceinline__ Cx<R> cadd(Cx<R> a, Cx<R> b) { return {a.x + b.x, a.y + b.y}; }
template <typename R>
__device__ __forceinline__ Cx<R> csub(Cx<R> a, Cx<R> b) { return {a.x - b.x, a.y - b.y}; }
template <typename R>
__device__ __forceinline__ Cx<R> cconj(Cx<R> a) { return {a.x, -a.y}; }
template <typename R>
__device__ __forceinline__ Cx<R> cscale(Cx<R> a, R s) { return {a.x * s, a.y * s}; }
// multiply by -i
template <typename R>
__device__ __forceinline__ Cx<R> cmul_mi(Cx<R> a) { return {a.y, -a.x}; }
// multiply by +i
template <typename R>
__device__ __forceinline__ Cx<R> cmul_pi(Cx<R> a) { return {-a.y, a.x}; }

__device__ __forceinline__ int bitrev(int v, int logn) { return (int)(__brev((unsigned)v) >> (32 - logn)); }

// Twiddle w_N^j = exp(sign * 2 pi i j / N) from a table of exp(+2 pi i j/N).
template <typename R>
__device__ __forceinline__ Cx<R> twid(const Cx<R> *tw, int j, int sign) {
  Cx<R> w = tw[j];
  if (sign < 0) w.y = -w.y;
  return w;
}

// In-place DIT FFT of `ncols` sequences of length 2^logn held in shared
// memory in bit-reversed order.  Element e of sequence c is at
// buf[c*cstride + e*estride].  tw holds exp(+2 pi i j/N), j < N.  All
// threads of the block must call it; it ends with a barrier.
template <typename R, int NCOLS = 0>
__device__ void fft_inplace(Cx<R> *buf, int logn, int ncols_rt, int cstride, int estride, const Cx<R> *tw,
                            int sign) {
  const int ncols = NCOLS > 0 ? NCOLS : ncols_rt;
  const int N = 1 << logn;
  int s = 0;
  if (logn & 1) {
    const int items = ncols * (N >> 1);
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
      const int c = it % ncols, k = it / ncols;
      Cx<R> *p = buf + c * cstride + (2 * k) * estride;
      Cx<R> a = p[0], b = p[estride];
      p[0] = cadd(a, b);
      p[estride] = csub(a, b);
    }
    s = 1;
    __syncthreads();
  }
  for (; s < logn; s += 2) {
    const int h = 1 << s;
    const int items = ncols * (N >> 2);
    const int t2 = N >> (s + 1);  // table stride of w_{2h}
    const int t4 = N >> (s + 2);  // table stride of w_{4h}
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
      const int c = it % ncols, q = it / ncols;
      const int k = q & (h - 1);
      const int base = ((q >> s) << (s + 2)) + k;
      Cx<R> *p = buf + c * cstride;
      Cx<R> a = p[base * estride], b = p[(base + h) * estride];
      Cx<R> cc = p[(base + 2 * h) * estride], d = p[(base + 3 * h) * estride];
      const Cx<R> w1 = twid(tw, k * t2, sign);
      b = cmul(b, w1);
      d = cmul(d, w1);
      Cx<R> a1 = cadd(a, b), b1 = csub(a, b), c1 = cadd(cc, d), d1 = csub(cc, d);
      const Cx<R> w2 = twid(tw, k * t4, sign), w3 = twid(tw, (k + h) * t4, sign);
      c1 = cmul(c1, w2);
      d1 = cmul(d1, w3);
      p[base * estride] = cadd(a1, c1);
      p[(base + 2 * h) * estride] = csub(a1, c1);
      p[(base + h) * estride] = cadd(b1, d1);
      p[(base + 3 * h) * estride] = csub(b1, d1);
    }
    __syncthreads();
  }
}

// Asynchronous global -> shared copies (cp.async): every thread queues all of
// its copies before waiting once, so a tile load keeps many requests in flight.
__device__ __forceinline__ void cp_async_8(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_16(void *smem, const void *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most N of this thread's committed groups are still in flight
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
template <typename R>
__device__ __forceinline__ void cp_async_cx(Cx<R> *smem, const Cx<R> *gmem) {
  if (sizeof(Cx<R>) == 16)
    cp_async_16(smem, gmem);
  else
    cp_async_8(smem, gmem);
}

// Programmatic dependent launch: let the next kernel of the stream start its
// launch now, then wait until the previous kernel has finished and its
// writes are visible.  Both are no-ops when the kernel was launched without
// the programmatic-serialization attribute.
__device__ __forceinline__ void pdl_begin() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// Cooperative copy of a twiddle table (n entries) into shared memory.
template <typename R>
__device__ __forceinline__ void load_twiddles(Cx<R> *dst, const Cx<R> *src, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
}

}  // namespace kapsel
