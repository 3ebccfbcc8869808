// Pruned 3D real FFT passes with the SPM k-space and real-space operators
// fused into them.
//
// Storage (per field component, complex values in the reference's Ooura sign):
//   zeta   [2][KXc][KYc][TS]   reduced vorticity, 2/3-rule modes only
//   I1     [c][NX][KYc][TS]    after the x transform (x in real space)
//   I2     [c][NX][NY][TS]     after the y transform (x, y in real space)
// (kz < TZ is used; rows are padded to TS so that every row starts on 32 bytes)
//   real   [c][NX][NY][NZ]     real-space fields
// KXc = 2*TX-1 holds kx = 0..TX-1, -(TX-1)..-1 (compact index ix, kx = ix
// for ix < TX, else ix - KXc); likewise KYc.  Only kz < TZ is stored.  The
// 2/3 rule of Truncate_two_third_rule_ooura (fft_wrapper.h:723-766) keeps
// exactly these modes, so every inverse transform starts from zero outside
// them and every forward transform whose result is truncated need not
// compute the rest.
#pragma once

#include "fft_device.cuh"
#include "particle_kernels.cuh"
#include "rfft_device.cuh"

namespace kapsel {

struct Geo {
  int NX, NY, NZ, M;      // M = NZ/2
  int lx, ly, lm;         // log2 of NX, NY, M
  int TX, TY, TZ;         // TRN = (N+2)/3 (input.cxx:297)
  int TS;                 // storage stride of the kz dimension: TZ rounded up to 4 (32-byte rows in FP32)
  int KXc, KYc;           // 2*TRN-1
  double wave[3];         // 2 pi / L
  double nu, dt;
  int fix_cell[3];
  int fp64_exp;           // 1: exp(x)-1 as the reference, 0: expm1
  double inv_n;           // 1/(NX*NY*NZ): the A_k2a scale (fft_wrapper.h:552)
};

template <typename R>
struct Twiddles {
  const Cx<R> *x, *y, *m, *z;  // exp(+2 pi i j/n) for n = NX, NY, NZ/2, NZ
};

__device__ __forceinline__ int full_from_compact(int c, int T, int Kc, int N) { return c < T ? c : N + c - Kc; }
__device__ __forceinline__ int signed_k(int i, int N) { return i > N / 2 ? i - N : i; }

// Zeta_k2u_k (fft_wrapper.cxx:408-511) for one mode: the third vorticity
// component from k.omega = 0 under the 3-case map, u = -i k x omega / k^2.
template <typename R>
__device__ __forceinline__ void zeta_to_u(int KXi, int KYi, R kx, R ky, R kz, R ik2, Cx<R> z0, Cx<R> z1,
                                          Cx<R> u[3]) {
  Cx<R> w0, w1, w2;
  if (KXi != 0) {
    const R inv = R(1) / kx;
    w0 = {-inv * (ky * z0.x + kz * z1.x), -inv * (ky * z0.y + kz * z1.y)};
    w1 = z0;
    w2 = z1;
  } else if (KYi != 0) {
    const R d = -(kz / ky);
    w0 = z1;
    w1 = {d * z0.x, d * z0.y};
    w2 = z0;
  } else {
    w0 = z0;
    w1 = z1;
    w2 = {R(0), R(0)};
  }
  const R ax = kx * ik2, ay = ky * ik2, az = kz * ik2;
  // u = -i (k/k^2) x omega
  Cx<R> c0 = {ay * w2.x - az * w1.x, ay * w2.y - az * w1.y};
  Cx<R> c1 = {az * w0.x - ax * w2.x, az * w0.y - ax * w2.y};
  Cx<R> c2 = {ax * w1.x - ay * w0.x, ax * w1.y - ay * w0.y};
  u[0] = cmul_mi(c0);
  u[1] = cmul_mi(c1);
  u[2] = cmul_mi(c2);
}

// Component map of Omega_k2zeta_k (fft_wrapper.cxx:137-173) / U_k2zeta_k
// (:258-339): kx != 0 -> (w1, w2); ky != 0 -> (w2, w0); else (w0, w1).
template <typename R>
__device__ __forceinline__ void select_zeta(int KXi, int KYi, const Cx<R> w[3], Cx<R> &z0, Cx<R> &z1) {
  if (KXi != 0) {
    z0 = w[1];
    z1 = w[2];
  } else if (KYi != 0) {
    z0 = w[2];
    z1 = w[0];
  } else {
    z0 = w[0];
    z1 = w[1];
  }
}

// ---------------------------------------------------------------------------
// x pass, inverse: zeta -> u_k (Zeta_k2u_k) -> inverse x transform.
// grid (KYc, ceil(TZ/KC)), out I1[3][NX][KYc][TZ].
template <typename R, int KC, int LX = 0, int XS = 0>
__global__ void __launch_bounds__(256) k_x_zeta_to_u(Geo g, Twiddles<R> tw, const Cx<R> *__restrict__ zeta,
                                                     const double *__restrict__ uk_dc, Cx<R> *__restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_begin();
  const int NXv = LX > 0 ? (1 << LX) : g.NX, LXv = LX > 0 ? LX : g.lx;
  constexpr int W = 3 * KC;
  Cx<R> *twx = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *Zt = twx + NXv;          // [2][KXc][KC] staged zeta tile
  Cx<R> *U = Zt + 2 * g.KXc * KC;  // [NX rows][3*KC]
  Cx<R> *scr = U + NXv * W;       // FFT scratch, NX*3*KC
  const int iy = blockIdx.x;
  const int kz0 = blockIdx.y * KC;
  const int ncol = min(KC, g.TZ - kz0);
  const size_t zplane = (size_t)g.KXc * g.KYc * g.TS;
  for (int it = threadIdx.x; it < 2 * g.KXc * KC; it += blockDim.x) {
    const int col = it % KC, rest = it / KC, ix = rest % g.KXc, c = rest / g.KXc;
    if (col < ncol)
      cp_async_cx(Zt + it, zeta + c * zplane + ((size_t)ix * g.KYc + iy) * g.TS + kz0 + col);
  }
  load_twiddles(twx, tw.x, NXv);
  cp_async_wait_all();
  __syncthreads();
  const int KYi = signed_k(full_from_compact(iy, g.TY, g.KYc, g.NY), g.NY);
  const R ky = R(g.wave[1] * KYi);
  for (int it = threadIdx.x; it < NXv * KC; it += blockDim.x) {
    const int col = it % KC, i = it / KC;
    Cx<R> u[3] = {{R(0), R(0)}, {R(0), R(0)}, {R(0), R(0)}};
    const int KXi = signed_k(i, NXv);
    if (col < ncol && abs(KXi) < g.TX) {
      const int ix = KXi >= 0 ? KXi : KXi + g.KXc;
      const int kz = kz0 + col;
      const Cx<R> z0 = Zt[ix * KC + col], z1 = Zt[(g.KXc + ix) * KC + col];
      const R kx = R(g.wave[0] * KXi), kzr = R(g.wave[2] * kz);
      const R k2 = kx * kx + ky * ky + kzr * kzr;
      const R ik2 = k2 > R(0) ? R(1) / k2 : R(0);
      zeta_to_u(KXi, KYi, kx, ky, kzr, ik2, z0, z1, u);
      if (KXi == 0 && KYi == 0 && kz == 0) {
        u[0] = {R(uk_dc[0]), R(0)};
        u[1] = {R(uk_dc[1]), R(0)};
        u[2] = {R(uk_dc[2]), R(0)};
      }
    }
    U[i * W + col] = u[0];
    U[i * W + KC + col] = u[1];
    U[i * W + 2 * KC + col] = u[2];
  }
  __syncthreads();
  fft2_smem<R, -1, W, LX, XS>(U, scr, LXv, 1, W, twx);
  for (int it = threadIdx.x; it < 3 * NXv * KC; it += blockDim.x) {
    const int col = it % KC, rest = it / KC, x = rest & (NXv - 1), c = rest >> LXv;
    if (col < ncol)
      out[(((size_t)c * NXv + x) * g.KYc + iy) * g.TS + kz0 + col] = U[x * W + c * KC + col];
  }
}

// ---------------------------------------------------------------------------
// y pass.  inverse: in [c][NX][KYc][TZ] -> out [c][NX][NY][TZ]
//          forward: in [c][NX][NY][TZ] -> out [c][NX][KYc][TZ] (|ky| < TY kept)
// grid (NX, ncomp, ceil(TZ/KC)).
template <typename R, bool INVERSE, int KC>
__global__ void __launch_bounds__(256, 3) k_y_pass(Geo g, Twiddles<R> tw, const Cx<R> *__restrict__ in,
                                                Cx<R> *__restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_begin();
  Cx<R> *twy = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *Y = twy + g.NY;      // [NY rows][KC]
  Cx<R> *scr = Y + g.NY * KC;  // FFT scratch
  const int x = blockIdx.x, c = blockIdx.y;
  const int kz0 = blockIdx.z * KC;
  const int ncol = min(KC, g.TZ - kz0);
  const int rows_in = INVERSE ? g.KYc : g.NY;
  const int rows_out = INVERSE ? g.NY : g.KYc;
  const Cx<R> *src = in + ((size_t)c * g.NX + x) * rows_in * g.TS + kz0;
  Cx<R> *dst = out + ((size_t)c * g.NX + x) * rows_out * g.TS + kz0;
  // each thread keeps one column and walks rows (256/KC rows apart)
  constexpr int RSTEP = 256 / KC;
  const int col = threadIdx.x % KC, j0 = threadIdx.x / KC;
  const bool colok = col < ncol;
  for (int j = j0; j < g.NY; j += RSTEP) {
    Cx<R> *d = Y + j * KC + col;
    int srow = j;
    if (INVERSE) {
      const int KYi = j > g.NY / 2 ? j - g.NY : j;
      srow = abs(KYi) < g.TY ? (KYi >= 0 ? KYi : KYi + g.KYc) : -1;
    }
    if (colok && srow >= 0)
      cp_async_cx(d, src + (size_t)srow * g.TS + col);
    else
      *d = {R(0), R(0)};
  }
  load_twiddles(twy, tw.y, g.NY);
  cp_async_wait_all();
  __syncthreads();
  fft2_smem<R, INVERSE ? -1 : 1, KC>(Y, scr, g.ly, 1, KC, twy);
  if (colok)
    for (int r = j0; r < rows_out; r += RSTEP) {
      const int j = INVERSE ? r : full_from_compact(r, g.TY, g.KYc, g.NY);
      dst[(size_t)r * g.TS + col] = Y[j * KC + col];
    }
}

// ---------------------------------------------------------------------------
// z pass helpers.  A row holds A[k], k < TZ, of a real line of NZ points.
// c2r: Z[k] = (A[k] + conj A[M-k]) + i (A[k] - conj A[M-k]) w^{-k}, k < M,
//      z = IFFT_M(Z), a[2n] = Re z[n], a[2n+1] = Im z[n].
// r2c: z[n] = a[2n] + i a[2n+1], Z = FFT_M(z),
//      A[k] = (Z[k] + conj Z[M-k])/2 - i/2 (Z[k] - conj Z[M-k]) w^{k}.
// Lines are held element-major in shared memory (element e of line s at
// [e*nseq + s]) so that consecutive threads touch consecutive words.
template <typename R>
__device__ __forceinline__ Cx<R> c2r_pre(const Cx<R> *row, int k, int M, int TZ, const Cx<R> *twz) {
  const Cx<R> zero = {R(0), R(0)};
  const Cx<R> a = k < TZ ? row[k] : zero;
  const Cx<R> b = (M - k) < TZ ? cconj(row[M - k]) : zero;
  const Cx<R> w = twid(twz, k, -1);
  return cadd(cadd(a, b), cmul_pi(cmul(csub(a, b), w)));
}

// seq: natural-order FFT result, element e at seq[e*es]; Z[M] is Z[0]
template <typename R>
__device__ __forceinline__ Cx<R> r2c_post(const Cx<R> *seq, int es, int k, int M, const Cx<R> *twz) {
  const Cx<R> zk = seq[(k & (M - 1)) * es];
  const Cx<R> zm = cconj(seq[((M - k) & (M - 1)) * es]);
  const Cx<R> e = cadd(zk, zm), d = csub(zk, zm);
  const Cx<R> w = twid(twz, k, 1);
  const Cx<R> t = cmul_mi(cmul(d, w));
  return cscale(cadd(e, t), R(0.5));
}

// Rows per block of the z kernels.
constexpr int ZROWS = 8;

// z pass fused at the centre of the nonlinear term (operate_omega.cxx:14-58):
// inverse z transform of the three velocity components of each row, the
// five real-space products u2u3, u3u1, u1u2, (u2-u3)(u2+u3), (u3-u1)(u3+u1),
// and their forward z transforms (kz < TZ kept).  In place on I2: reads
// components 0..2, writes 0..4.  grid (NX*NY/ZROWS).
template <typename R>
__global__ void __launch_bounds__(256) k_z_products(Geo g, Twiddles<R> tw, Cx<R> *__restrict__ io) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_begin();
  const int M = g.M;
  constexpr int NV = ZROWS * 3, NQ = ZROWS * 5;
  constexpr int EV = NV + 1, EQ = NQ + 1;  // odd element strides: conflict-free columns
  Cx<R> *twm = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *twz = twm + M;
  Cx<R> *V = twz + g.NZ;     // [M][EV] velocity lines, line = rr*3 + c
  Cx<R> *Q = V + M * EV;     // [M][EQ] product lines, line = rr*5 + c
  Cx<R> *scr = Q + M * EQ;   // FFT scratch [M*NQ]; also the staged input and output rows
  Cx<R> *A = scr;            // [NV][TZ + 1]
  const int TA = g.TZ + 1;
  const size_t rows = (size_t)g.NX * g.NY;
  const size_t row0 = (size_t)blockIdx.x * ZROWS;
  const size_t cstr = rows * g.TS;
  for (int it = threadIdx.x; it < NV * g.TZ; it += blockDim.x) {
    const int k = it % g.TZ, q = it / g.TZ, c = q % 3, rr = q / 3;
    cp_async_cx(A + q * TA + k, io + c * cstr + (row0 + rr) * g.TS + k);
  }
  load_twiddles(twm, tw.m, M);
  load_twiddles(twz, tw.z, g.NZ);
  cp_async_wait_all();
  __syncthreads();
  for (int it = threadIdx.x; it < NV * M; it += blockDim.x) {
    const int q = it % NV, k = it / NV;  // q = rr*3 + c
    V[k * EV + q] = c2r_pre(A + q * TA, k, M, g.TZ, twz);
  }
  __syncthreads();
  fft2_smem<R, -1, NV>(V, scr, g.lm, 1, EV, twm);
  const R sc = R(g.inv_n);
  for (int it = threadIdx.x; it < ZROWS * M; it += blockDim.x) {
    const int rr = it % ZROWS, n = it / ZROWS;
    const Cx<R> *v = V + n * EV + rr * 3;
    const Cx<R> U1 = v[0], U2 = v[1], U3 = v[2];
    const R u1a = U1.x * sc, u1b = U1.y * sc, u2a = U2.x * sc, u2b = U2.y * sc, u3a = U3.x * sc,
            u3b = U3.y * sc;
    Cx<R> *q = Q + n * EQ + rr * 5;
    q[0] = {u2a * u3a, u2b * u3b};
    q[1] = {u3a * u1a, u3b * u1b};
    q[2] = {u1a * u2a, u1b * u2b};
    q[3] = {(u2a - u3a) * (u2a + u3a), (u2b - u3b) * (u2b + u3b)};
    q[4] = {(u3a - u1a) * (u3a + u1a), (u3b - u1b) * (u3b + u1b)};
  }
  __syncthreads();
  fft2_smem<R, 1, NQ>(Q, scr, g.lm, 1, EQ, twm);
  // post-process line by line (consecutive threads: consecutive lines), then
  // copy the [line][TZ] tile out with consecutive threads on consecutive k
  Cx<R> *O = scr;  // [NQ][TA]
  for (int it = threadIdx.x; it < NQ * g.TZ; it += blockDim.x) {
    const int q = it % NQ, k = it / NQ;
    O[q * TA + k] = r2c_post(Q + q, EQ, k, M, twz);
  }
  __syncthreads();
  for (int it = threadIdx.x; it < NQ * g.TZ; it += blockDim.x) {
    const int k = it % g.TZ, q = it / g.TZ, rr = q / 5, c = q % 5;
    io[c * cstr + (row0 + rr) * g.TS + k] = O[q * TA + k];
  }
}

// z pass, inverse to real space: in I2 [c][NX][NY][TZ], out real [c][rows][pitch]
// scaled by 1/(NX NY NZ).  grid (NX*NY/ZROWS, ncomp).
// Blocks past the row blocks (blockIdx.y == 0 only) run the particle position
// update of the step (MD_solver_position_Euler / _AB2), which needs no field
// and must finish before the hydrodynamic gather, as u* must: one launch
// serves both.
template <typename R>
__global__ void __launch_bounds__(256) k_z_c2r(Geo g, Twiddles<R> tw, const Cx<R> *__restrict__ in,
                                               R *__restrict__ out, size_t out_cstride, int out_pitch, PPar pp,
                                               DPart *__restrict__ parts, int euler, int *__restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_begin();
  const int nrow_blocks = (g.NX * g.NY) / ZROWS;
  if ((int)blockIdx.x >= nrow_blocks) {
    const int n = ((int)blockIdx.x - nrow_blocks) * blockDim.x + threadIdx.x;
    if (blockIdx.y == 0 && parts && n < pp.Np) position_update_one(pp, parts, n, euler, status);
    return;
  }
  const int M = g.M;
  constexpr int ES = ZROWS + 1;
  Cx<R> *twm = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *twz = twm + M;
  Cx<R> *S = twz + g.NZ;        // [M][ES]
  Cx<R> *scr = S + M * ES;      // FFT scratch [M*ZROWS]; first the staged rows [ZROWS][TZ+1]
  Cx<R> *A = scr;
  const int TA = g.TZ + 1;
  const int c = blockIdx.y;
  const size_t rows = (size_t)g.NX * g.NY;
  const size_t row0 = (size_t)blockIdx.x * ZROWS;
  const Cx<R> *src = in + c * rows * g.TS + row0 * g.TS;
  for (int it = threadIdx.x; it < ZROWS * g.TZ; it += blockDim.x) {
    const int k = it % g.TZ, rr = it / g.TZ;
    cp_async_cx(A + rr * TA + k, src + rr * g.TS + k);
  }
  load_twiddles(twm, tw.m, M);
  load_twiddles(twz, tw.z, g.NZ);
  cp_async_wait_all();
  __syncthreads();
  for (int it = threadIdx.x; it < ZROWS * M; it += blockDim.x) {
    const int rr = it % ZROWS, k = it / ZROWS;
    S[k * ES + rr] = c2r_pre(A + rr * TA, k, M, g.TZ, twz);
  }
  __syncthreads();
  fft2_smem<R, -1, ZROWS>(S, scr, g.lm, 1, ES, twm);
  const R sc = R(g.inv_n);
  R *dst = out + c * out_cstride;
  for (int it = threadIdx.x; it < ZROWS * M; it += blockDim.x) {
    const int n = it & (M - 1), rr = it >> g.lm;
    const Cx<R> v = S[n * ES + rr];
    R *o = dst + (row0 + rr) * (size_t)out_pitch + 2 * n;
    o[0] = v.x * sc;
    o[1] = v.y * sc;
  }
}

// z pass of the rigidity force (Make_f_particle_dt_nonsole, f_particle.h:41-64,
// with the phi > 1 clamp of make_phi.cxx:278-297 applied on the fly):
// f = up' - phi' u*, forward z transform, kz < TZ kept -> out [3][NX][NY][TZ].
// The scattered phi/up fields are cleared where they were written, so they are
// all-zero again for the next scatter.  grid (NX*NY/ZROWS).
template <typename R>
__global__ void __launch_bounds__(256) k_z_force(Geo g, Twiddles<R> tw, R *__restrict__ phiup,
                                                 const R *__restrict__ ustar, Cx<R> *__restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_begin();
  const int M = g.M;
  constexpr int NS = ZROWS * 3, ES = NS + 1;
  Cx<R> *twm = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *twz = twm + M;
  Cx<R> *S = twz + g.NZ;     // [M][ES], line = rr*3 + d
  Cx<R> *scr = S + M * ES;   // FFT scratch
  load_twiddles(twm, tw.m, M);
  load_twiddles(twz, tw.z, g.NZ);
  const size_t npts = (size_t)g.NX * g.NY * g.NZ;
  const size_t row0 = (size_t)blockIdx.x * ZROWS;
  for (int it = threadIdx.x; it < ZROWS * M; it += blockDim.x) {
    const int n = it & (M - 1), rr = it >> g.lm;
    const size_t o = (row0 + rr) * g.NZ + 2 * n;
    R ph[2], up[3][2], us[3][2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      ph[e] = phiup[o + e];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        up[d][e] = phiup[(1 + d) * npts + o + e];
        us[d][e] = ustar[d * npts + o + e];
      }
    }
    R f[3][2];
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      R p = ph[e];
      if (p > R(1)) {
        const R inv = R(1) / p;
#pragma unroll
        for (int d = 0; d < 3; ++d) up[d][e] *= inv;
        p = R(1);
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) f[d][e] = up[d][e] - p * us[d][e];
      if (ph[e] != R(0)) {
        phiup[o + e] = R(0);
#pragma unroll
        for (int d = 0; d < 3; ++d) phiup[(1 + d) * npts + o + e] = R(0);
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) S[n * ES + rr * 3 + d] = {f[d][0], f[d][1]};
  }
  __syncthreads();
  fft2_smem<R, 1, NS>(S, scr, g.lm, 1, ES, twm);
  const size_t rows = (size_t)g.NX * g.NY;
  const int TA = g.TZ + 1;
  Cx<R> *O = scr;  // [NS][TA]
  for (int it = threadIdx.x; it < NS * g.TZ; it += blockDim.x) {
    const int q = it % NS, k = it / NS;
    O[q * TA + k] = r2c_post(S + q, ES, k, M, twz);
  }
  __syncthreads();
  for (int it = threadIdx.x; it < NS * g.TZ; it += blockDim.x) {
    const int k = it % g.TZ, q = it / g.TZ, d = q % 3, rr = q / 3;
    out[d * rows * g.TS + (row0 + rr) * g.TS + k] = O[q * TA + k];
  }
}

// z pass, forward of a real field with padded pitch (routine-level A2a_k):
// in real [c][NX][NY][pitch] -> out [c][NX][NY][NZ/2+1] (all kz).
template <typename R>
__global__ void __launch_bounds__(256) k_z_r2c_full(Geo g, Twiddles<R> tw, const R *__restrict__ in,
                                                    int in_pitch, Cx<R> *__restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int M = g.M;
  Cx<R> *twm = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *twz = twm + M;
  constexpr int ES = ZROWS + 1;
  Cx<R> *S = twz + g.NZ;        // [M][ES]
  Cx<R> *scr = S + M * ES;
  load_twiddles(twm, tw.m, M);
  load_twiddles(twz, tw.z, g.NZ);
  const size_t row0 = (size_t)blockIdx.x * ZROWS;
  for (int it = threadIdx.x; it < ZROWS * M; it += blockDim.x) {
    const int n = it & (M - 1), rr = it >> g.lm;
    const R *r = in + (row0 + rr) * (size_t)in_pitch + 2 * n;
    S[n * ES + rr] = {r[0], r[1]};
  }
  __syncthreads();
  fft2_smem<R, 1, ZROWS>(S, scr, g.lm, 1, ES, twm);
  for (int it = threadIdx.x; it < ZROWS * (M + 1); it += blockDim.x) {
    const int k = it % (M + 1), rr = it / (M + 1);
    out[(row0 + rr) * (M + 1) + k] = r2c_post(S + rr, ES, k, M, twz);
  }
}

// One retained mode of the nonlinear term and the fluid update
// (operate_omega.cxx:60-97, Omega_k2zeta_k, NS_solver_slavedEuler
// fluid_solver.cxx:328-354; EULER: Add_zeta_viscous_term + Field_solver_Euler,
// fluid_solver.cxx:122-135): from the five forward-transformed product
// spectra at wavevector (k1, k2, k3), update the reduced vorticity (z0, z1).
template <typename R, int EULER>
__device__ __forceinline__ void advect_mode_update(const Geo &g, int KXi, int KYi, R k1, R k2, R k3, Cx<R> a23,
                                                   Cx<R> a31, Cx<R> a12, Cx<R> b2233, Cx<R> b3311, Cx<R> &z0,
                                                   Cx<R> &z1) {
  const Cx<R> b1122 = {-b3311.x - b2233.x, -b3311.y - b2233.y};
  const R k1k2 = k1 * k2, k2k3 = k2 * k3, k3k1 = k3 * k1;
  const R d32 = (k3 - k2) * (k3 + k2), d13 = (k1 - k3) * (k1 + k3), d21 = (k2 - k1) * (k2 + k1);
  Cx<R> w[3];
  w[0] = {-(k2k3 * b2233.x + d32 * a23.x + k3k1 * a12.x - k1k2 * a31.x),
          -(k2k3 * b2233.y + d32 * a23.y + k3k1 * a12.y - k1k2 * a31.y)};
  w[1] = {-(k3k1 * b3311.x + d13 * a31.x + k1k2 * a23.x - k2k3 * a12.x),
          -(k3k1 * b3311.y + d13 * a31.y + k1k2 * a23.y - k2k3 * a12.y)};
  w[2] = {-(k1k2 * b1122.x + d21 * a12.x + k2k3 * a31.x - k3k1 * a23.x),
          -(k1k2 * b1122.y + d21 * a12.y + k2k3 * a31.y - k3k1 * a23.y)};
  Cx<R> f0, f1;
  select_zeta(KXi, KYi, w, f0, f1);
  const R K2 = k1 * k1 + k2 * k2 + k3 * k3;
  const R IK2 = K2 > R(0) ? R(1) / K2 : R(0);
  if (EULER) {
    const R nk2 = R(g.nu) * K2, dt = R(g.dt);
    const Cx<R> r0 = {f0.x + -(nk2 * z0.x), f0.y + -(nk2 * z0.y)};
    const Cx<R> r1 = {f1.x + -(nk2 * z1.x), f1.y + -(nk2 * z1.y)};
    z0 = {z0.x + dt * r0.x, z0.y + dt * r0.y};
    z1 = {z1.x + dt * r1.x, z1.y + dt * r1.y};
  } else {
    const double arg = -g.nu * g.dt * (double)K2;
    const R dmy = R(g.fp64_exp ? exp(arg) - 1.0 : expm1(arg));
    const R c1 = R(1.0 / g.nu) * IK2;
    z0 = {z0.x + dmy * (z0.x - c1 * f0.x), z0.y + dmy * (z0.y - c1 * f0.y)};
    z1 = {z1.x + dmy * (z1.x - c1 * f1.x), z1.y + dmy * (z1.y - c1 * f1.y)};
  }
}

// ---------------------------------------------------------------------------
// Row tiles of the x passes move KC consecutive kz values per row.  With float
// complex values a pair is one 16-byte transfer when both addresses are
// 16-byte aligned (always, for the layouts here: row strides, plane strides
// and kz0 are multiples of four values), else two 8-byte ones; `left` is the
// number of values of the row that exist from this pair on (values past the
// retained columns are zero-filled in shared memory, never read or written in
// global memory).
template <typename R>
__device__ __forceinline__ bool aligned16(const void *a, const void *b) {
  return ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15u) == 0;
}
template <typename R>
__device__ __forceinline__ void stage_pair(Cx<R> *d, const Cx<R> *s, int left) {
  if (left >= 2 && aligned16<R>(d, s)) {
    cp_async_16(d, s);
    return;
  }
  if (left >= 1) cp_async_cx(d, s); else d[0] = {R(0), R(0)};
  if (left >= 2) cp_async_cx(d + 1, s + 1); else d[1] = {R(0), R(0)};
}
template <typename R>
__device__ __forceinline__ void store_pair(Cx<R> *o, const Cx<R> *p, int left) {
  if (left >= 2 && aligned16<R>(o, p)) {
    *reinterpret_cast<float4 *>(o) = *reinterpret_cast<const float4 *>(p);
    return;
  }
  if (left >= 1) o[0] = p[0];
  if (left >= 2) o[1] = p[1];
}

// ---------------------------------------------------------------------------
// x pass, forward, of the five product spectra fused with the rest of
// NS_solver_slavedEuler (fluid_solver.cxx:328-354) and the next inverse:
//   Omega from the product spectra (operate_omega.cxx:60-97), its reduction
//   (Omega_k2zeta_k), the slaved-Euler update of zeta on the retained modes,
//   FIX_CELL on uk_dc (sp_3d_ns.cxx:67-73), then Zeta_k2u_k of the updated
//   zeta and the inverse x transform of u*.
// In place on buf: reads [5][NX][KYc][TZ], writes [3][NX][KYc][TZ].
// grid (KYc, ceil(TZ/KC)).
// EULER = 1 is the Electrolyte variant: explicit Euler of
// NSsolute_solver_Euler (Add_zeta_viscous_term then Field_solver_Euler,
// fluid_solver.cxx:122-135, operate_omega.cxx:172-184) instead of the slaved
// step, and no u* output (the electrolyte rebuilds u after the Coulomb force).
template <typename R, int KC, int EULER = 0, int LX = 0, int XS = 0>
__global__ void __launch_bounds__(256) k_x_advect_update(Geo g, Twiddles<R> tw, Cx<R> *__restrict__ buf,
                                                         Cx<R> *__restrict__ zeta, double *__restrict__ uk_dc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_begin();
  const int NXv = LX > 0 ? (1 << LX) : g.NX, LXv = LX > 0 ? LX : g.lx;
  constexpr int W5 = 5 * KC, W3 = 3 * KC;
  Cx<R> *twx = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *Zs = twx + NXv;               // [2][KXc][KC] zeta tile (updated in place)
  Cx<R> *Pb = Zs + 2 * g.KXc * KC;       // [NX][5*KC], later [NX][3*KC]
  Cx<R> *scr = Pb + NXv * W5;            // FFT scratch
  __shared__ double ukd[3];
  const int iy = blockIdx.x;
  const int kz0 = blockIdx.y * KC;
  const int ncol = min(KC, g.TZ - kz0);
  const size_t cstr = (size_t)NXv * g.KYc * g.TS;
  const size_t zplane = (size_t)g.KXc * g.KYc * g.TS;
  // stage the five product spectra (bit-reversed rows) and the zeta tile
  if constexpr (sizeof(R) == 4 && KC % 2 == 0) {
    constexpr int KP = KC / 2;
    for (int it = threadIdx.x; it < 5 * NXv * KP; it += blockDim.x) {
      const int col = 2 * (it % KP), rest = it / KP, x = rest & (NXv - 1), c = rest >> LXv;
      stage_pair(Pb + x * W5 + c * KC + col, buf + c * cstr + ((size_t)x * g.KYc + iy) * g.TS + kz0 + col,
                 ncol - col);
    }
    for (int it = threadIdx.x; it < 2 * g.KXc * KP; it += blockDim.x) {
      const int col = 2 * (it % KP), rest = it / KP, ix = rest % g.KXc, c = rest / g.KXc;
      stage_pair(Zs + rest * KC + col, zeta + c * zplane + ((size_t)ix * g.KYc + iy) * g.TS + kz0 + col, ncol - col);
    }
  } else {
    for (int it = threadIdx.x; it < 5 * NXv * KC; it += blockDim.x) {
      const int col = it % KC, rest = it / KC, x = rest & (NXv - 1), c = rest >> LXv;
      Cx<R> *d = Pb + x * W5 + c * KC + col;
      if (col < ncol)
        cp_async_cx(d, buf + c * cstr + ((size_t)x * g.KYc + iy) * g.TS + kz0 + col);
      else
        *d = {R(0), R(0)};
    }
    for (int it = threadIdx.x; it < 2 * g.KXc * KC; it += blockDim.x) {
      const int col = it % KC, rest = it / KC, ix = rest % g.KXc, c = rest / g.KXc;
      if (col < ncol) cp_async_cx(Zs + it, zeta + c * zplane + ((size_t)ix * g.KYc + iy) * g.TS + kz0 + col);
    }
  }
  load_twiddles(twx, tw.x, NXv);
  const bool has_k0 = (iy == 0 && blockIdx.y == 0);
  if (threadIdx.x < 3) {
    double v = 0.0;
    if (has_k0) {
      v = g.fix_cell[threadIdx.x] ? 0.0 : uk_dc[threadIdx.x];
      uk_dc[threadIdx.x] = v;
    }
    ukd[threadIdx.x] = v;
  }
  cp_async_wait_all();
  __syncthreads();
  fft2_smem<R, 1, W5, LX, XS>(Pb, scr, LXv, 1, W5, twx);
  const int KYi = signed_k(full_from_compact(iy, g.TY, g.KYc, g.NY), g.NY);
  const R ky = R(g.wave[1] * KYi);
  for (int it = threadIdx.x; it < g.KXc * KC; it += blockDim.x) {
    const int col = it % KC, ix = it / KC;
    if (col >= ncol) continue;
    const int KXi = ix < g.TX ? ix : ix - g.KXc;
    const int i = KXi >= 0 ? KXi : KXi + NXv;
    const int kz = kz0 + col;
    const R k1 = R(g.wave[0] * KXi), k2 = ky, k3 = R(g.wave[2] * kz);
    const Cx<R> *p = Pb + i * W5 + col;
    Cx<R> z0 = Zs[ix * KC + col], z1 = Zs[(g.KXc + ix) * KC + col];
    advect_mode_update<R, EULER>(g, KXi, KYi, k1, k2, k3, p[0], p[KC], p[2 * KC], p[3 * KC], p[4 * KC], z0, z1);
    const size_t o = ((size_t)ix * g.KYc + iy) * g.TS + kz;
    zeta[o] = z0;
    zeta[zplane + o] = z1;
    Zs[ix * KC + col] = z0;
    Zs[(g.KXc + ix) * KC + col] = z1;
  }
  if (EULER) return;
  __syncthreads();
  // u*_k = Zeta_k2u_k(zeta', uk_dc) on all NX rows (zero outside |kx| < TX)
  for (int it = threadIdx.x; it < NXv * KC; it += blockDim.x) {
    const int col = it % KC, i = it / KC;
    Cx<R> u[3] = {{R(0), R(0)}, {R(0), R(0)}, {R(0), R(0)}};
    const int KXi = signed_k(i, NXv);
    if (col < ncol && abs(KXi) < g.TX) {
      const int ix = KXi >= 0 ? KXi : KXi + g.KXc;
      const int kz = kz0 + col;
      const R kx = R(g.wave[0] * KXi), kzr = R(g.wave[2] * kz);
      const R k2 = kx * kx + ky * ky + kzr * kzr;
      const R ik2 = k2 > R(0) ? R(1) / k2 : R(0);
      zeta_to_u(KXi, KYi, kx, ky, kzr, ik2, Zs[ix * KC + col], Zs[(g.KXc + ix) * KC + col], u);
      if (KXi == 0 && KYi == 0 && kz == 0) {
        u[0] = {R(ukd[0]), R(0)};
        u[1] = {R(ukd[1]), R(0)};
        u[2] = {R(ukd[2]), R(0)};
      }
    }
    Pb[i * W3 + col] = u[0];
    Pb[i * W3 + KC + col] = u[1];
    Pb[i * W3 + 2 * KC + col] = u[2];
  }
  __syncthreads();
  fft2_smem<R, -1, W3, LX, XS>(Pb, scr, LXv, 1, W3, twx);
  if constexpr (sizeof(R) == 4 && KC % 2 == 0) {
    constexpr int KP = KC / 2;
    for (int it = threadIdx.x; it < 3 * NXv * KP; it += blockDim.x) {
      const int col = 2 * (it % KP), rest = it / KP, x = rest & (NXv - 1), c = rest >> LXv;
      store_pair(buf + c * cstr + ((size_t)x * g.KYc + iy) * g.TS + kz0 + col, Pb + x * W3 + c * KC + col,
                 ncol - col);
    }
  } else {
    for (int it = threadIdx.x; it < 3 * NXv * KC; it += blockDim.x) {
      const int col = it % KC, rest = it / KC, x = rest & (NXv - 1), c = rest >> LXv;
      if (col < ncol) buf[c * cstr + ((size_t)x * g.KYc + iy) * g.TS + kz0 + col] = Pb[x * W3 + c * KC + col];
    }
  }
}

// ---------------------------------------------------------------------------
// x pass, forward, of the rigidity force f fused with the end of the step:
// 2/3 truncation (implicit), Solenoidal_uk (operate_omega.cxx:186-219) and
// the k-space form of Add_f_particle + U2zeta_k (f_particle.h:83-99,
// operate_omega.h:186-189): zeta += U_k2zeta_k(f_sol), uk_dc += Re f(k=0).
// The velocity before the force is Zeta_k2u of the truncated zeta, so its
// own U2zeta_k is that zeta again (linearity; parity up to roundoff).
// in buf [3][NX][KYc][TZ].  grid (KYc, ceil(TZ/KC)).
// NEXTU = 1 also does the first launch of the next step on the same tile:
// u_k = Zeta_k2u_k(zeta, uk_dc) of the updated values and the inverse x
// transform, written over buf (as k_x_zeta_to_u writes it, with the same
// arithmetic), so the next step starts at its y pass.
template <typename R, int KC, int LX = 0, int NEXTU = 0, int XS = 0>
__global__ void __launch_bounds__(256) k_x_force_to_zeta(Geo g, Twiddles<R> tw, Cx<R> *__restrict__ buf,
                                                         Cx<R> *__restrict__ zeta, double *__restrict__ uk_dc) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_begin();
  const int NXv = LX > 0 ? (1 << LX) : g.NX, LXv = LX > 0 ? LX : g.lx;
  constexpr int W3 = 3 * KC;
  Cx<R> *twx = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *Zs = twx + NXv;          // [2][KXc][KC]
  Cx<R> *Pb = Zs + 2 * g.KXc * KC;  // [NX][3*KC]
  Cx<R> *scr = Pb + NXv * W3;       // FFT scratch
  __shared__ double ukn[3];         // uk_dc after the update (NEXTU)
  const int iy = blockIdx.x;
  const int kz0 = blockIdx.y * KC;
  const int ncol = min(KC, g.TZ - kz0);
  const size_t cstr = (size_t)NXv * g.KYc * g.TS;
  const size_t zplane = (size_t)g.KXc * g.KYc * g.TS;
  if constexpr (sizeof(R) == 4 && KC % 2 == 0) {
    constexpr int KP = KC / 2;
    for (int it = threadIdx.x; it < 3 * NXv * KP; it += blockDim.x) {
      const int col = 2 * (it % KP), rest = it / KP, x = rest & (NXv - 1), c = rest >> LXv;
      stage_pair(Pb + x * W3 + c * KC + col, buf + c * cstr + ((size_t)x * g.KYc + iy) * g.TS + kz0 + col,
                 ncol - col);
    }
    for (int it = threadIdx.x; it < 2 * g.KXc * KP; it += blockDim.x) {
      const int col = 2 * (it % KP), rest = it / KP, ix = rest % g.KXc, c = rest / g.KXc;
      stage_pair(Zs + rest * KC + col, zeta + c * zplane + ((size_t)ix * g.KYc + iy) * g.TS + kz0 + col, ncol - col);
    }
  } else {
    for (int it = threadIdx.x; it < 3 * NXv * KC; it += blockDim.x) {
      const int col = it % KC, rest = it / KC, x = rest & (NXv - 1), c = rest >> LXv;
      Cx<R> *d = Pb + x * W3 + c * KC + col;
      if (col < ncol)
        cp_async_cx(d, buf + c * cstr + ((size_t)x * g.KYc + iy) * g.TS + kz0 + col);
      else
        *d = {R(0), R(0)};
    }
    for (int it = threadIdx.x; it < 2 * g.KXc * KC; it += blockDim.x) {
      const int col = it % KC, rest = it / KC, ix = rest % g.KXc, c = rest / g.KXc;
      if (col < ncol) cp_async_cx(Zs + it, zeta + c * zplane + ((size_t)ix * g.KYc + iy) * g.TS + kz0 + col);
    }
  }
  load_twiddles(twx, tw.x, NXv);
  cp_async_wait_all();
  __syncthreads();
  fft2_smem<R, 1, W3, LX, XS>(Pb, scr, LXv, 1, W3, twx);
  const int KYi = signed_k(full_from_compact(iy, g.TY, g.KYc, g.NY), g.NY);
  const R ky = R(g.wave[1] * KYi);
  for (int it = threadIdx.x; it < g.KXc * KC; it += blockDim.x) {
    const int col = it % KC, ix = it / KC;
    if (col >= ncol) continue;
    const int KXi = ix < g.TX ? ix : ix - g.KXc;
    const int i = KXi >= 0 ? KXi : KXi + NXv;
    const int kz = kz0 + col;
    const R kx = R(g.wave[0] * KXi), kzr = R(g.wave[2] * kz);
    const Cx<R> *p = Pb + i * W3 + col;
    Cx<R> f0 = p[0], f1 = p[KC], f2 = p[2 * KC];
    if (KXi == 0 && KYi == 0 && kz == 0) {
      uk_dc[0] += (double)f0.x;
      uk_dc[1] += (double)f1.x;
      uk_dc[2] += (double)f2.x;
      if (NEXTU)
        for (int d = 0; d < 3; ++d) ukn[d] = uk_dc[d];
      continue;  // zeta(k=0) stays 0
    }
    const R K2 = kx * kx + ky * ky + kzr * kzr;
    const R IK2 = R(1) / K2;
    const Cx<R> dk = {IK2 * (f0.x * kx + f1.x * ky + f2.x * kzr), IK2 * (f0.y * kx + f1.y * ky + f2.y * kzr)};
    f0 = {f0.x - dk.x * kx, f0.y - dk.y * kx};
    f1 = {f1.x - dk.x * ky, f1.y - dk.y * ky};
    f2 = {f2.x - dk.x * kzr, f2.y - dk.y * kzr};
    // omega = -i k x f
    Cx<R> w[3];
    w[0] = cmul_mi(Cx<R>{ky * f2.x - kzr * f1.x, ky * f2.y - kzr * f1.y});
    w[1] = cmul_mi(Cx<R>{kzr * f0.x - kx * f2.x, kzr * f0.y - kx * f2.y});
    w[2] = cmul_mi(Cx<R>{kx * f1.x - ky * f0.x, kx * f1.y - ky * f0.y});
    Cx<R> z0, z1;
    select_zeta(KXi, KYi, w, z0, z1);
    const size_t o = ((size_t)ix * g.KYc + iy) * g.TS + kz;
    z0 = cadd(Zs[ix * KC + col], z0);
    z1 = cadd(Zs[(g.KXc + ix) * KC + col], z1);
    zeta[o] = z0;
    zeta[zplane + o] = z1;
    if (NEXTU) {
      Zs[ix * KC + col] = z0;
      Zs[(g.KXc + ix) * KC + col] = z1;
    }
  }
  if (!NEXTU) return;
  __syncthreads();
  // the next step's k_x_zeta_to_u on this tile, from the updated Zs / ukn
  for (int it = threadIdx.x; it < NXv * KC; it += blockDim.x) {
    const int col = it % KC, i = it / KC;
    Cx<R> u[3] = {{R(0), R(0)}, {R(0), R(0)}, {R(0), R(0)}};
    const int KXi = signed_k(i, NXv);
    if (col < ncol && abs(KXi) < g.TX) {
      const int ix = KXi >= 0 ? KXi : KXi + g.KXc;
      const int kz = kz0 + col;
      const Cx<R> z0 = Zs[ix * KC + col], z1 = Zs[(g.KXc + ix) * KC + col];
      const R kx = R(g.wave[0] * KXi), kzr = R(g.wave[2] * kz);
      const R k2 = kx * kx + ky * ky + kzr * kzr;
      const R ik2 = k2 > R(0) ? R(1) / k2 : R(0);
      zeta_to_u(KXi, KYi, kx, ky, kzr, ik2, z0, z1, u);
      if (KXi == 0 && KYi == 0 && kz == 0) {
        u[0] = {R(ukn[0]), R(0)};
        u[1] = {R(ukn[1]), R(0)};
        u[2] = {R(ukn[2]), R(0)};
      }
    }
    Pb[i * W3 + col] = u[0];
    Pb[i * W3 + KC + col] = u[1];
    Pb[i * W3 + 2 * KC + col] = u[2];
  }
  __syncthreads();
  fft2_smem<R, -1, W3, LX, XS>(Pb, scr, LXv, 1, W3, twx);
  if constexpr (sizeof(R) == 4 && KC % 2 == 0) {
    constexpr int KP = KC / 2;
    for (int it = threadIdx.x; it < 3 * NXv * KP; it += blockDim.x) {
      const int col = 2 * (it % KP), rest = it / KP, x = rest & (NXv - 1), c = rest >> LXv;
      store_pair(buf + (((size_t)c * NXv + x) * g.KYc + iy) * g.TS + kz0 + col, Pb + x * W3 + c * KC + col,
                 ncol - col);
    }
  } else {
    for (int it = threadIdx.x; it < 3 * NXv * KC; it += blockDim.x) {
      const int col = it % KC, rest = it / KC, x = rest & (NXv - 1), c = rest >> LXv;
      if (col < ncol) buf[(((size_t)c * NXv + x) * g.KYc + iy) * g.TS + kz0 + col] = Pb[x * W3 + c * KC + col];
    }
  }
}

}  // namespace kapsel
