// z and y passes with compile-time line length and warp-level transforms.
//
// The z passes of the step (the nonlinear-term centre, the inverse to u*,
// and the rigidity force) work on independent rows of NZ = 2M reals, so
// each warp owns a group of RW rows from staging to store and needs no
// block barrier.  The M-point complex transform is the two-level
// decomposition M = N1 * N2 of rfft_device.cuh, done by one warp on RW =
// 32/N2 lines at a time:
//   phase 1: lane (line, t) loads x[N2 n1 + t], n1 < N1, does the N1-point
//            DFT, multiplies by w_M^(t k1) (twiddles kept in registers: t is
//            fixed per lane) and stores the result over its own inputs;
//   phase 2: lane (line, k1) loads the N2 values of row k1, does the N2-point
//            DFT and stores X[k1 + N1 k2] in natural order.
// Lines live in a padded layout, element j at j + j/N2, which makes both
// phases' shared-memory accesses conflict-free and lets phase 1 work in
// place.  The real-to-complex packing (even/odd split) is the same as the
// block-level kernels; z lengths are M = 32, 64, 128 (NZ = 64..256), y
// lengths NY = 32..256.
#pragma once

#include "spectral_kernels.cuh"

namespace kapsel {

template <int LM>
struct ZL {
  static constexpr int M = 1 << LM, NZ = 2 * M, TZ = (NZ + 2) / 3, TS = (TZ + 3) & ~3;
  static constexpr int L1 = ((LM + 1) >> 1) > 4 ? 4 : ((LM + 1) >> 1);
  static constexpr int N1 = 1 << L1, L2 = LM - L1, N2 = 1 << L2;
  static constexpr int RW = 32 / N2;                         // lines per warp batch
  static constexpr int PL = M + M / N2;                      // padded line length
  static constexpr int LS = PL + ((8 - PL % 16) + 16) % 16;  // line stride, LS % 16 == 8
  static constexpr int IT2 = RW * N1 / 32;                   // phase-2 items per lane
  static constexpr int KW = M / 32;                          // k values per lane in pre/post
  static constexpr int LR = L2 > 5 ? 0 : 5 - L2;             // log2(RW)
  static_assert(LM >= 5 && LM <= 8, "line length");
};

template <int LM>
__device__ __forceinline__ int zpos(int j) {
  return j + (j >> ZL<LM>::L2);
}

// Placement of the RW lines of a warp batch in shared memory: line l starts
// at base(l).  The z passes use l*LS.  The y pass uses a stride and an order
// of the lines chosen for its element size so that its strided gather and
// scatter (four kz columns of consecutive rows per half warp) and the
// transform phases hit distinct banks (a search over strides and orders,
// counting wavefronts of every access of the pass: 268 -> 219 per work item
// for 128-point float lines, 684 -> 368 for double).
struct ZLines {
  template <int LM>
  __device__ __forceinline__ static int base(int l) { return l * ZL<LM>::LS; }
};
template <typename R, int LY>
struct YLines {
  static constexpr bool F = sizeof(R) == 4;
  static constexpr int LS = LY == 6 ? (F ? 76 : 74) : LY == 7 ? (F ? 148 : 146) : LY == 8 ? (F ? 280 : 276)
                                                                                        : ZL<LY>::LS;
  // line order as 4-bit fields: (1,3,2,0) for float, (3,2,1,0) for double
  static constexpr unsigned PERM = (LY == 6 || LY == 7) ? (F ? 0x0231u : 0x0123u) : 0x76543210u;
  template <int LM>
  __device__ __forceinline__ static int base(int l) { return (int)((PERM >> (4 * l)) & 15u) * LS; }
};

// Phase-1 twiddles of this lane: w_M^(SIGN t k1), t = lane mod N2.
template <typename R, int LM, int SIGN>
__device__ __forceinline__ void wfft_twiddles(const Cx<R> *__restrict__ twm, Cx<R> (&w)[ZL<LM>::N1]) {
  const int t = (threadIdx.x & 31) & (ZL<LM>::N2 - 1);
#pragma unroll
  for (int k1 = 0; k1 < ZL<LM>::N1; ++k1) w[k1] = twid(twm, t * k1, SIGN);
}

// In-place transform of RW lines (line l at buf + l*LS, padded layout),
// natural order in and out; ends with __syncwarp.
template <typename R, int LM, int SIGN, typename LB = ZLines>
__device__ __forceinline__ void wfft(Cx<R> *buf, const Cx<R> (&w)[ZL<LM>::N1]) {
  using Z = ZL<LM>;
  const int lane = threadIdx.x & 31;
  {
    const int l = lane >> Z::L2, t = lane & (Z::N2 - 1);
    Cx<R> *p = buf + LB::template base<LM>(l) + t;
    Cx<R> v[Z::N1];
#pragma unroll
    for (int n1 = 0; n1 < Z::N1; ++n1) v[n1] = p[n1 * (Z::N2 + 1)];
    dft_small<R, SIGN>(v, Z::N1);
#pragma unroll
    for (int k1 = 1; k1 < Z::N1; ++k1) v[k1] = cmul(v[k1], w[k1]);
#pragma unroll
    for (int k1 = 0; k1 < Z::N1; ++k1) p[k1 * (Z::N2 + 1)] = v[k1];
  }
  __syncwarp();
  Cx<R> y[Z::IT2][Z::N2];
#pragma unroll
  for (int q = 0; q < Z::IT2; ++q) {
    const int i = lane + 32 * q, l = i >> Z::L1, k1 = i & (Z::N1 - 1);
    const Cx<R> *p = buf + LB::template base<LM>(l) + k1 * (Z::N2 + 1);
#pragma unroll
    for (int n2 = 0; n2 < Z::N2; ++n2) y[q][n2] = p[n2];
  }
  __syncwarp();
#pragma unroll
  for (int q = 0; q < Z::IT2; ++q) {
    const int i = lane + 32 * q, l = i >> Z::L1, k1 = i & (Z::N1 - 1);
    dft_small<R, SIGN>(y[q], Z::N2);
    Cx<R> *p = buf + LB::template base<LM>(l);
#pragma unroll
    for (int k2 = 0; k2 < Z::N2; ++k2) p[zpos<LM>(k1 + Z::N1 * k2)] = y[q][k2];
  }
  __syncwarp();
}

// c2r packing of one line of A[k], k < TZ (stride 1, shared or global) into the padded
// line Z: Z[k] = (A[k] + conj A[M-k]) + i (A[k] - conj A[M-k]) w_NZ^{-k}.
// wk[j] = w_NZ^{-k} for this lane's k = lane + 32 j.
template <typename R, int LM>
__device__ __forceinline__ void wpack_c2r(const Cx<R> *A, Cx<R> *Zl, const Cx<R> (&wk)[ZL<LM>::KW]) {
  using Z = ZL<LM>;
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < Z::KW; ++j) {
    const int k = lane + 32 * j;
    const Cx<R> zero = {R(0), R(0)};
    const Cx<R> a = k < Z::TZ ? A[k] : zero;
    const Cx<R> b = (Z::M - k) < Z::TZ ? cconj(A[Z::M - k]) : zero;
    Zl[zpos<LM>(k)] = cadd(cadd(a, b), cmul_pi(cmul(csub(a, b), wk[j])));
  }
}

// r2c unpacking of a transformed line at index k < TZ: twz = w_NZ^{+j} table.
template <typename R, int LM>
__device__ __forceinline__ Cx<R> wunpack_r2c(const Cx<R> *Zl, int k, const Cx<R> *__restrict__ twz) {
  using Z = ZL<LM>;
  const Cx<R> zk = Zl[zpos<LM>(k)];
  const Cx<R> zm = cconj(Zl[zpos<LM>((Z::M - k) & (Z::M - 1))]);
  const Cx<R> e = cadd(zk, zm), d = csub(zk, zm);
  const Cx<R> t = cmul_mi(cmul(d, twz[k]));
  return cscale(cadd(e, t), R(0.5));
}

template <typename R, int LM>
__device__ __forceinline__ void wpre_twiddles(const Cx<R> *__restrict__ twz, Cx<R> (&wk)[ZL<LM>::KW]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int j = 0; j < ZL<LM>::KW; ++j) wk[j] = twid(twz, lane + 32 * j, -1);
}

template <typename R>
struct Vec2;
template <>
struct Vec2<float> {
  using T = float2;
};
template <>
struct Vec2<double> {
  using T = double2;
};

// ---------------------------------------------------------------------------
// Nonlinear-term centre (as k_z_products): per row group, inverse z of the
// three velocity components, the five products, forward z (kz < TZ kept).
// In place on I2.  Warps stride over row groups of RW rows.  FP32 fields:
// four line groups per warp, the fifth product waits in registers and
// reuses group 0 once the first four are stored.  The c2r packing reads the
// rows straight from global memory (no stage area): a row group's loads are
// then in flight together instead of behind a staging copy, which cut the
// long-scoreboard stalls per issue from 4.1 to 0.9 at the same 16 resident
// warps per SM.
template <typename R, int LM, int NW>
__global__ void __launch_bounds__(NW * 32) k_zw_products(Geo g, Twiddles<R> tw, Cx<R> *__restrict__ io) {
  using Z = ZL<LM>;
  constexpr int GL = Z::RW * Z::LS, KP = Z::RW * Z::M / 32;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_begin();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Cx<R> *buf = reinterpret_cast<Cx<R> *>(smem_raw) + (size_t)warp * 4 * GL;
  Cx<R> wi[Z::N1], wf[Z::N1], wk[Z::KW];
  wfft_twiddles<R, LM, -1>(tw.m, wi);
  wfft_twiddles<R, LM, 1>(tw.m, wf);
  wpre_twiddles<R, LM>(tw.z, wk);
  const size_t rows = (size_t)g.NX * g.NY;
  const size_t cstr = rows * Z::TS;
  const int ngroups = (int)(rows / Z::RW);
  const R sc = R(g.inv_n);
  for (int grp = blockIdx.x * NW + warp; grp < ngroups; grp += gridDim.x * NW) {
    const size_t row0 = (size_t)grp * Z::RW;
#pragma unroll
    for (int c = 0; c < 3; ++c)
      for (int rr = 0; rr < Z::RW; ++rr)
        wpack_c2r<R, LM>(io + c * cstr + (row0 + rr) * Z::TS, buf + c * GL + rr * Z::LS, wk);
    __syncwarp();
#pragma unroll
    for (int c = 0; c < 3; ++c) wfft<R, LM, -1>(buf + c * GL, wi);
    Cx<R> p4[KP];
#pragma unroll
    for (int jj = 0; jj < KP; ++jj) {
      const int i = lane + 32 * jj;
      const int rr = i >> LM, n = rr * Z::LS + zpos<LM>(i & (Z::M - 1));
      const Cx<R> U1 = buf[n], U2 = buf[GL + n], U3 = buf[2 * GL + n];
      const R u1a = U1.x * sc, u1b = U1.y * sc, u2a = U2.x * sc, u2b = U2.y * sc, u3a = U3.x * sc, u3b = U3.y * sc;
      buf[n] = {u2a * u3a, u2b * u3b};
      buf[GL + n] = {u3a * u1a, u3b * u1b};
      buf[2 * GL + n] = {u1a * u2a, u1b * u2b};
      buf[3 * GL + n] = {(u2a - u3a) * (u2a + u3a), (u2b - u3b) * (u2b + u3b)};
      p4[jj] = {(u3a - u1a) * (u3a + u1a), (u3b - u1b) * (u3b + u1b)};
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 4; ++q) wfft<R, LM, 1>(buf + q * GL, wf);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      Cx<R> *dst = io + q * cstr + row0 * Z::TS;
      for (int i = lane; i < Z::RW * Z::TZ; i += 32) {
        const int rr = i / Z::TZ, kk = i - rr * Z::TZ;
        dst[rr * Z::TS + kk] = wunpack_r2c<R, LM>(buf + q * GL + rr * Z::LS, kk, tw.z);
      }
    }
    __syncwarp();
#pragma unroll
    for (int jj = 0; jj < KP; ++jj) {
      const int i = lane + 32 * jj;
      buf[(i >> LM) * Z::LS + zpos<LM>(i & (Z::M - 1))] = p4[jj];
    }
    __syncwarp();
    wfft<R, LM, 1>(buf, wf);
    {
      Cx<R> *dst = io + 4 * cstr + row0 * Z::TS;
      for (int i = lane; i < Z::RW * Z::TZ; i += 32) {
        const int rr = i / Z::TZ, kk = i - rr * Z::TZ;
        dst[rr * Z::TS + kk] = wunpack_r2c<R, LM>(buf + rr * Z::LS, kk, tw.z);
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// Nonlinear-term centre with prefetch (FP64 fields): as k_zw_products, but
// each warp owns
// four line groups and a stage area: while it transforms one row group,
// cp.async brings the next group's three input rows into the stage.  Four
// products go through the line groups; the fifth waits in registers and
// reuses group 0 once the first four are stored.
template <typename R, int LM>
struct ZProd {
  using Z = ZL<LM>;
  static constexpr int GL = Z::RW * Z::LS;     // one line group
  static constexpr int SG = 3 * Z::RW * Z::TS;  // staged input of a row group
  static constexpr int WARP = 4 * GL + SG;      // elements per warp
  static constexpr int KP = Z::RW * Z::M / 32;  // product elements per lane
};

template <typename R, int LM, int NW>
__global__ void __launch_bounds__(NW * 32) k_zw_products_pf(Geo g, Twiddles<R> tw, Cx<R> *__restrict__ io) {
  using Z = ZL<LM>;
  using P = ZProd<R, LM>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_begin();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Cx<R> *buf = reinterpret_cast<Cx<R> *>(smem_raw) + (size_t)warp * P::WARP;
  Cx<R> *stage = buf + 4 * P::GL;  // [3][RW][TS]
  Cx<R> wi[Z::N1], wf[Z::N1], wk[Z::KW];
  wfft_twiddles<R, LM, -1>(tw.m, wi);
  wfft_twiddles<R, LM, 1>(tw.m, wf);
  wpre_twiddles<R, LM>(tw.z, wk);
  const size_t rows = (size_t)g.NX * g.NY;
  const size_t cstr = rows * Z::TS;
  const int ngroups = (int)(rows / Z::RW);
  const int gstride = gridDim.x * NW;
  const R sc = R(g.inv_n);
  int grp = blockIdx.x * NW + warp;
  auto issue = [&](int gq) {
    const size_t r0 = (size_t)gq * Z::RW;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const Cx<R> *src = io + c * cstr + r0 * Z::TS;
      for (int i = lane; i < Z::RW * Z::TS; i += 32) cp_async_cx(stage + c * Z::RW * Z::TS + i, src + i);
    }
    cp_async_commit();
  };
  if (grp < ngroups) issue(grp);
  for (; grp < ngroups; grp += gstride) {
    const size_t row0 = (size_t)grp * Z::RW;
    cp_async_wait_all();
    __syncwarp();
#pragma unroll
    for (int c = 0; c < 3; ++c)
      for (int rr = 0; rr < Z::RW; ++rr)
        wpack_c2r<R, LM>(stage + (c * Z::RW + rr) * Z::TS, buf + c * P::GL + rr * Z::LS, wk);
    __syncwarp();
    if (grp + gstride < ngroups) issue(grp + gstride);
#pragma unroll
    for (int c = 0; c < 3; ++c) wfft<R, LM, -1>(buf + c * P::GL, wi);
    Cx<R> p4[P::KP];
#pragma unroll
    for (int jj = 0; jj < P::KP; ++jj) {
      const int i = lane + 32 * jj;
      const int rr = i >> LM, n = rr * Z::LS + zpos<LM>(i & (Z::M - 1));
      const Cx<R> U1 = buf[n], U2 = buf[P::GL + n], U3 = buf[2 * P::GL + n];
      const R u1a = U1.x * sc, u1b = U1.y * sc, u2a = U2.x * sc, u2b = U2.y * sc, u3a = U3.x * sc, u3b = U3.y * sc;
      buf[n] = {u2a * u3a, u2b * u3b};
      buf[P::GL + n] = {u3a * u1a, u3b * u1b};
      buf[2 * P::GL + n] = {u1a * u2a, u1b * u2b};
      buf[3 * P::GL + n] = {(u2a - u3a) * (u2a + u3a), (u2b - u3b) * (u2b + u3b)};
      p4[jj] = {(u3a - u1a) * (u3a + u1a), (u3b - u1b) * (u3b + u1b)};
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 4; ++q) wfft<R, LM, 1>(buf + q * P::GL, wf);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      Cx<R> *dst = io + q * cstr + row0 * Z::TS;
      for (int i = lane; i < Z::RW * Z::TZ; i += 32) {
        const int rr = i / Z::TZ, k = i - rr * Z::TZ;
        dst[rr * Z::TS + k] = wunpack_r2c<R, LM>(buf + q * P::GL + rr * Z::LS, k, tw.z);
      }
    }
    __syncwarp();
#pragma unroll
    for (int jj = 0; jj < P::KP; ++jj) {
      const int i = lane + 32 * jj;
      buf[(i >> LM) * Z::LS + zpos<LM>(i & (Z::M - 1))] = p4[jj];
    }
    __syncwarp();
    wfft<R, LM, 1>(buf, wf);
    {
      Cx<R> *dst = io + 4 * cstr + row0 * Z::TS;
      for (int i = lane; i < Z::RW * Z::TZ; i += 32) {
        const int rr = i / Z::TZ, k = i - rr * Z::TZ;
        dst[rr * Z::TS + k] = wunpack_r2c<R, LM>(buf + rr * Z::LS, k, tw.z);
      }
    }
    __syncwarp();
  }
}

// Inverse z to real space (as k_z_c2r): out[c][row][pitch] = A_k2a-scaled
// reals.  Tasks (component, row group).  Blocks at or past `nblk` run the
// particle position update instead (MD_solver_position_Euler / _AB2), which
// needs no field and must finish before the hydrodynamic gather, as u* must.
template <typename R, int LM, int NW>
__global__ void __launch_bounds__(NW * 32) k_zw_c2r(Geo g, Twiddles<R> tw, const Cx<R> *__restrict__ in,
                                                    R *__restrict__ out, size_t out_cstride, int out_pitch,
                                                    int ncomp, int nblk, PPar pp, DPart *__restrict__ parts,
                                                    int euler, int *__restrict__ status) {
  using Z = ZL<LM>;
  using V2 = typename Vec2<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_begin();
  if ((int)blockIdx.x >= nblk) {
    const int n = ((int)blockIdx.x - nblk) * blockDim.x + threadIdx.x;
    if (parts && n < pp.Np) position_update_one(pp, parts, n, euler, status);
    return;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // one line group per warp: the packing reads the rows straight from global
  // memory, and the small footprint keeps more warps resident
  Cx<R> *buf = reinterpret_cast<Cx<R> *>(smem_raw) + (size_t)warp * Z::RW * Z::LS;
  Cx<R> wi[Z::N1], wk[Z::KW];
  wfft_twiddles<R, LM, -1>(tw.m, wi);
  wpre_twiddles<R, LM>(tw.z, wk);
  const size_t rows = (size_t)g.NX * g.NY;
  const int ngroups = (int)(rows / Z::RW);
  const R sc = R(g.inv_n);
  for (int task = blockIdx.x * NW + warp; task < ncomp * ngroups; task += nblk * NW) {
    const int c = task / ngroups;
    const size_t row0 = (size_t)(task - c * ngroups) * Z::RW;
    const Cx<R> *src = in + c * rows * Z::TS + row0 * Z::TS;
    for (int rr = 0; rr < Z::RW; ++rr) wpack_c2r<R, LM>(src + rr * Z::TS, buf + rr * Z::LS, wk);
    __syncwarp();
    wfft<R, LM, -1>(buf, wi);
    R *dst = out + c * out_cstride + row0 * (size_t)out_pitch;
    for (int i = lane; i < Z::RW * Z::M; i += 32) {
      const int rr = i >> LM, n = i & (Z::M - 1);
      const Cx<R> v = buf[rr * Z::LS + zpos<LM>(n)];
      V2 o;
      o.x = v.x * sc;
      o.y = v.y * sc;
      *reinterpret_cast<V2 *>(dst + rr * (size_t)out_pitch + 2 * n) = o;
    }
    __syncwarp();
  }
}

// One element pair of the rigidity force: phi > 1 clamp, f = up' - phi' u*
// into the three padded lines, and phi/up cleared where phi was written.
template <typename R, int LM>
__device__ __forceinline__ void zw_force_item(Cx<R> *buf, R *__restrict__ phiup, size_t npts, size_t row0, int i,
                                              typename Vec2<R>::T ph, typename Vec2<R>::T (&up)[3],
                                              const typename Vec2<R>::T (&us)[3]) {
  using Z = ZL<LM>;
  using V2 = typename Vec2<R>::T;
  const int rr = i >> LM, n = i & (Z::M - 1);
  const size_t o = row0 * Z::NZ + 2 * (size_t)i;
  R p0 = ph.x, p1 = ph.y;
  if (p0 > R(1)) {
    const R inv = R(1) / p0;
#pragma unroll
    for (int d = 0; d < 3; ++d) up[d].x *= inv;
    p0 = R(1);
  }
  if (p1 > R(1)) {
    const R inv = R(1) / p1;
#pragma unroll
    for (int d = 0; d < 3; ++d) up[d].y *= inv;
    p1 = R(1);
  }
#pragma unroll
  for (int d = 0; d < 3; ++d)
    buf[(d * Z::RW + rr) * Z::LS + zpos<LM>(n)] = {up[d].x - p0 * us[d].x, up[d].y - p1 * us[d].y};
  if (ph.x != R(0) || ph.y != R(0)) {
    const V2 zero = {R(0), R(0)};
    *reinterpret_cast<V2 *>(phiup + o) = zero;
#pragma unroll
    for (int d = 0; d < 3; ++d) *reinterpret_cast<V2 *>(phiup + (1 + d) * npts + o) = zero;
  }
}

// Rigidity force (as k_z_force): f = up' - phi' u* with the phi > 1 clamp,
// phi/up cleared where written, forward z, kz < TZ kept -> out [3][rows][TZ].
// phi >= 0 at every point and up is zero wherever phi is, so clearing both
// values of an element pair when either phi is non-zero is exact.
template <typename R, int LM, int NW>
__global__ void __launch_bounds__(NW * 32) k_zw_force(Geo g, Twiddles<R> tw, R *__restrict__ phiup,
                                                      const R *__restrict__ ustar, Cx<R> *__restrict__ out) {
  using Z = ZL<LM>;
  using V2 = typename Vec2<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_begin();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Cx<R> *buf = reinterpret_cast<Cx<R> *>(smem_raw) + (size_t)warp * 3 * Z::RW * Z::LS;
  Cx<R> wf[Z::N1];
  wfft_twiddles<R, LM, 1>(tw.m, wf);
  const size_t rows = (size_t)g.NX * g.NY;
  const size_t npts = rows * Z::NZ;
  const int ngroups = (int)(rows / Z::RW);
  constexpr int NI = Z::RW * Z::M / 32;  // element pairs per lane
  for (int grp = blockIdx.x * NW + warp; grp < ngroups; grp += gridDim.x * NW) {
    const size_t row0 = (size_t)grp * Z::RW;
    // phi first, all of the lane's element pairs at once: where phi is zero
    // up is zero too and f = up - phi u* = 0, so up and u* are read only
    // where a particle's profile reaches (about an eighth of the points at
    // a solid fraction of 0.14); the rest of the pass is unchanged
    V2 ph[NI];
#pragma unroll
    for (int h = 0; h < NI; ++h)
      ph[h] = *reinterpret_cast<const V2 *>(phiup + row0 * Z::NZ + 2 * (size_t)(lane + 32 * h));
#pragma unroll 1
    for (int h = 0; h < NI; ++h) {
      const int i = lane + 32 * h;
      const size_t o = row0 * Z::NZ + 2 * (size_t)i;
      V2 up[3], us[3];
      if (ph[h].x != R(0) || ph[h].y != R(0)) {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          up[d] = *reinterpret_cast<const V2 *>(phiup + (1 + d) * npts + o);
          us[d] = *reinterpret_cast<const V2 *>(ustar + d * npts + o);
        }
      } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) up[d] = us[d] = V2{R(0), R(0)};
      }
      zw_force_item<R, LM>(buf, phiup, npts, row0, i, ph[h], up, us);
    }
    __syncwarp();
#pragma unroll
    for (int d = 0; d < 3; ++d) wfft<R, LM, 1>(buf + d * Z::RW * Z::LS, wf);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      Cx<R> *dst = out + d * rows * Z::TS + row0 * Z::TS;
      for (int i = lane; i < Z::RW * Z::TZ; i += 32) {
        const int rr = i / Z::TZ, k = i - rr * Z::TZ;
        dst[rr * Z::TS + k] = wunpack_r2c<R, LM>(buf + (d * Z::RW + rr) * Z::LS, k, tw.z);
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// y pass with compile-time NY = 2^LY (as k_y_pass).  A work item is RW
// consecutive kz columns of one (component, x) plane; each warp of a
// persistent grid walks its items.  NSLOT = 2 (FP64): two shared-memory
// slots, and while the warp transforms item k from one, cp.async brings item
// k+1 into the other.  NSLOT = 1 (FP32): one slot, half the shared memory
// per warp and so more resident warps; measured faster for FP32 fields and
// slower for FP64.  The
// gather lands each element straight at its padded-line position.  FULLY:
// the retained box spans every ky (the untruncated half spectrum).
//   inverse: in [c][NX][KYc][TS] -> out [c][NX][NY][TS]
//   forward: in [c][NX][NY][TS] -> out [c][NX][KYc][TS] (|ky| < TY kept)
template <typename R, bool INVERSE, int LY, bool FULLY>
__device__ __forceinline__ void yw_issue(const Geo &g, const Cx<R> *__restrict__ in, Cx<R> *slot, int item,
                                         int nbatch) {
  using Y = ZL<LY>;
  using YL = YLines<R, LY>;
  constexpr int RW = Y::RW, NY = Y::M;
  constexpr int TYc = FULLY ? NY / 2 + 1 : (NY + 2) / 3, KYc = FULLY ? NY : 2 * TYc - 1;
  constexpr int RIN = INVERSE ? KYc : NY;
  const int lane = threadIdx.x & 31;
  const int batch = item % nbatch, plane = item / nbatch;
  const int col0 = batch * RW, ncols = min(RW, g.TZ - col0);
  const Cx<R> *src = in + (size_t)plane * RIN * g.TS + col0;
  const Cx<R> zero = {R(0), R(0)};
  for (int i = lane; i < RIN * RW; i += 32) {
    const int r = i >> Y::LR, col = i & (RW - 1);
    const int j = INVERSE ? (r < TYc ? r : NY + r - KYc) : r;
    Cx<R> *d = slot + YL::template base<LY>(col) + zpos<LY>(j);
    if (col < ncols)
      cp_async_cx(d, src + (size_t)r * g.TS + col);
    else
      *d = zero;
  }
  if (INVERSE)
    for (int i = lane; i < (NY - KYc) * RW; i += 32) {
      const int j = TYc + (i >> Y::LR), col = i & (RW - 1);
      slot[YL::template base<LY>(col) + zpos<LY>(j)] = zero;
    }
}

// blocks of the y pass resident per SM that the register budget must allow
#ifndef KAPSEL_YW_MINB
#define KAPSEL_YW_MINB 1
#endif
template <typename R, bool INVERSE, int LY, bool FULLY, int NW, int NSLOT>
__global__ void __launch_bounds__(NW * 32, KAPSEL_YW_MINB) k_yw_pass(Geo g, Twiddles<R> tw, const Cx<R> *__restrict__ in,
                                                     Cx<R> *__restrict__ out, int ncomp) {
  using Y = ZL<LY>;
  using YL = YLines<R, LY>;
  constexpr int RW = Y::RW, NY = Y::M, SLOT = RW * YL::LS;
  static_assert(NSLOT == 1 || NSLOT == 2, "slots");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_begin();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Cx<R> *slots = reinterpret_cast<Cx<R> *>(smem_raw) + (size_t)warp * NSLOT * SLOT;
  const int nbatch = (g.TZ + RW - 1) / RW;
  const int nitems = ncomp * g.NX * nbatch;
  const int rows_out = INVERSE ? NY : g.KYc;
  Cx<R> w[Y::N1];
  wfft_twiddles<R, LY, INVERSE ? -1 : 1>(tw.y, w);
  const int stride = gridDim.x * NW;
  int item = blockIdx.x * NW + warp;
  if (NSLOT == 2 && item < nitems) yw_issue<R, INVERSE, LY, FULLY>(g, in, slots, item, nbatch);
  cp_async_commit();
  for (int k = 0; item < nitems; ++k, item += stride) {
    Cx<R> *cur = slots + (NSLOT == 2 ? (k & 1) * SLOT : 0);
    if (NSLOT == 2) {
      if (item + stride < nitems)
        yw_issue<R, INVERSE, LY, FULLY>(g, in, slots + ((k + 1) & 1) * SLOT, item + stride, nbatch);
      cp_async_commit();
      cp_async_wait_group<1>();
    } else {
      yw_issue<R, INVERSE, LY, FULLY>(g, in, slots, item, nbatch);
      cp_async_commit();
      cp_async_wait_all();
    }
    __syncwarp();
    wfft<R, LY, INVERSE ? -1 : 1, YL>(cur, w);
    const int batch = item % nbatch, plane = item / nbatch;
    const int col0 = batch * RW, ncols = min(RW, g.TZ - col0);
    Cx<R> *dst = out + (size_t)plane * rows_out * g.TS + col0;
    for (int i = lane; i < rows_out * RW; i += 32) {
      const int r = i >> Y::LR, col = i & (RW - 1);
      const int j = INVERSE ? r : full_from_compact(r, g.TY, g.KYc, NY);
      if (col < ncols) dst[(size_t)r * g.TS + col] = cur[YL::template base<LY>(col) + zpos<LY>(j)];
    }
    __syncwarp();
  }
  cp_async_wait_all();
}

}  // namespace kapsel
