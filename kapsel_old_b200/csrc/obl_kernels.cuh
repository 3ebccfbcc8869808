// Kernels of the Lees-Edwards sheared step on the oblique (deforming) grid,
// Time_evolution_hydro_OBL (sp_3d_ns.cxx:214-390).
//
// State that changes every step lives in device memory so that the step can
// be captured into a CUDA graph: ObState[0] = degree_oblique (input.cxx:271),
// [1] = Shear_rate_eff, [2] = 1 when this step reset the oblique grid,
// [3] = Shear_strain_realized (sp_3d_ns.cxx:600), [8..] reduction partials.
//
// k-space operators (one mode at a time, retained 2/3 box only; the
// reference truncates zeta at the start of every step, operate_omega.cxx:
// 118-120, so the modes outside are never read):
//   zeta -> contravariant u (Zeta_k2u_k_OBL, fft_wrapper.cxx:513-595) and
//   vorticity (Zeta_k2omega_k_OBL, :597-640); the advection term with the
//   shear correction, its curl and the slaved-Euler update
//   (Zeta_k2advection_k_OBL, operate_omega.cxx:115-170;
//   NS_solver_slavedEuler_Shear_OBL, fluid_solver.cxx:398-430); the
//   oblique projection, contra->co and U_k2zeta_k_OBL (operate_omega.cxx:
//   222-263, fft_wrapper.h:327-361, fft_wrapper.cxx:341-406).
// Real-space kernels: the grid reset when degree_oblique passes 1
// (sp_3d_ns.cxx:278-317), oblique <-> Cartesian interpolation (U_oblique2u,
// U2u_oblique, fft_wrapper.h:204-325), the effective shear rate
// (Calc_shear_rate_eff, sp_3d_ns.h:174-196), the rigidity force and the
// Lees-Edwards particle kernels (PBC_OBL periodic_boundary.h:22-42,
// Relative_coord_check_stepover_Y make_phi.h:198-236, Distance0_OBL
// interaction.h:39-65, Calc_f_hydro_correct_precision_OBL md_force.cxx:
// 391-520, Make_phi_u_primitive_OBL make_phi.cxx:299-384,
// MD_solver_*_OBL particle_solver.cxx:292-440).
#pragma once

#include "particle_kernels.cuh"
#include "spectral_kernels.cuh"

namespace kapsel {

enum { OB_DEG = 0, OB_SRATE = 1, OB_REMAP = 2, OB_STRAIN = 3, OB_PART = 8 };
constexpr int OB_RED_BLOCKS = 296;

struct OblPar {
  double shear_rate;  // Shear_rate of the DC external field
  double dt;
  double srate_scale; // Ivolume DX^3 NY/(NY-1) (sp_3d_ns.h:175,192)
  double dx;
  int NX, NY, NZ;
};

// K2 of the oblique grid (sp_3d_ns.cxx:325-338): kx^2 + (ky - deg kx)^2 + kz^2.
__device__ __forceinline__ double obl_k2(const Geo &g, double deg, int KXi, int KYi, int kz) {
  const double a = g.wave[0] * (double)KXi;
  const double b = g.wave[1] * (double)KYi - g.wave[0] * deg * (double)KXi;
  const double c = g.wave[2] * (double)kz;
  return a * a + b * b + c * c;
}

// Contravariant vorticity from the reduced one (the kx != 0 / kz != 0 / else
// map of Zeta_k2omega_k_OBL, fft_wrapper.cxx:597-640).
template <typename R>
__device__ __forceinline__ void obl_omega(int KXi, int kz, R kx, R ky, R kzr, Cx<R> z0, Cx<R> z1, Cx<R> w[3]) {
  if (KXi != 0) {
    const R inv = -(R(1) / kx);
    w[0] = {inv * (ky * z0.x + kzr * z1.x), inv * (ky * z0.y + kzr * z1.y)};
    w[1] = z0;
    w[2] = z1;
  } else if (kz != 0) {
    const R d = -(ky / kzr);
    w[0] = z1;
    w[1] = z0;
    w[2] = {d * z0.x, d * z0.y};
  } else {
    w[0] = z0;
    w[1] = {R(0), R(0)};
    w[2] = z1;
  }
}

// Zeta_k2u_k_OBL for one mode k != 0: omega to covariant, then
// u = -i (k/K2) x omega_co (contravariant velocity).
template <typename R>
__device__ __forceinline__ void obl_zeta_to_u(int KXi, int kz, R kx, R ky, R kzr, R ik2, R deg, Cx<R> z0, Cx<R> z1,
                                              Cx<R> u[3]) {
  Cx<R> w[3];
  obl_omega(KXi, kz, kx, ky, kzr, z0, z1, w);
  const R dd = R(1) + deg * deg;
  const Cx<R> c0 = {w[0].x + deg * w[1].x, w[0].y + deg * w[1].y};
  const Cx<R> c1 = {deg * w[0].x + dd * w[1].x, deg * w[0].y + dd * w[1].y};
  const Cx<R> c2 = w[2];
  const R ax = kx * ik2, ay = ky * ik2, az = kzr * ik2;
  u[0] = {ay * c2.y - az * c1.y, -(ay * c2.x - az * c1.x)};
  u[1] = {az * c0.y - ax * c2.y, -(az * c0.x - ax * c2.x)};
  u[2] = {ax * c1.y - ay * c0.y, -(ax * c1.x - ay * c0.x)};
}

// ---------------------------------------------------------------------------
// x pass, inverse, from the compact zeta:
//   NOUT = 6: contravariant u (Zeta_k2u_k_OBL, k = 0 from uk_dc) and the
//             contravariant vorticity (Zeta_k2omega_k_OBL), for the advection
//             term (Zeta_k2u_cpuky / Zeta_k2omega_OBL, operate_omega.h:144-172);
//   NOUT = 3: u after the FIX_CELL reset of uk_dc (sp_3d_ns.cxx:240-253).
// IK2 and the metric use degree_oblique at the start of the step.
// out I1: [NOUT][NX][KYc][TS].  grid (KYc, ceil(TZ/KC)).
template <typename R, int KC, int NOUT>
__global__ void __launch_bounds__(256) k_x_obl_inv(Geo g, Twiddles<R> tw, const Cx<R> *__restrict__ zeta,
                                                   double *__restrict__ uk_dc, const double *__restrict__ st,
                                                   Cx<R> *__restrict__ out) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int W = NOUT * KC;
  Cx<R> *twx = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *Zt = twx + g.NX;           // [2][KXc][KC]
  Cx<R> *U = Zt + 2 * g.KXc * KC;   // [NX][NOUT*KC]
  Cx<R> *scr = U + g.NX * W;
  __shared__ double ukd[3];
  const int iy = blockIdx.x;
  const int kz0 = blockIdx.y * KC;
  const int ncol = min(KC, g.TZ - kz0);
  const size_t zplane = (size_t)g.KXc * g.KYc * g.TS;
  for (int it = threadIdx.x; it < 2 * g.KXc * KC; it += blockDim.x) {
    const int col = it % KC, rest = it / KC, ix = rest % g.KXc, c = rest / g.KXc;
    if (col < ncol) cp_async_cx(Zt + it, zeta + c * zplane + ((size_t)ix * g.KYc + iy) * g.TS + kz0 + col);
  }
  load_twiddles(twx, tw.x, g.NX);
  const bool has_k0 = (iy == 0 && blockIdx.y == 0);
  if (threadIdx.x < 3) {
    double v = has_k0 ? uk_dc[threadIdx.x] : 0.0;
    if (NOUT == 3 && has_k0 && g.fix_cell[threadIdx.x]) {
      v = 0.0;
      uk_dc[threadIdx.x] = 0.0;
    }
    ukd[threadIdx.x] = v;
  }
  cp_async_wait_all();
  __syncthreads();
  const double deg = st[OB_DEG];
  const int KYi = signed_k(full_from_compact(iy, g.TY, g.KYc, g.NY), g.NY);
  const R ky = R(g.wave[1] * KYi);
  for (int it = threadIdx.x; it < g.NX * KC; it += blockDim.x) {
    const int col = it % KC, i = it / KC;
    Cx<R> o[NOUT];
#pragma unroll
    for (int c = 0; c < NOUT; ++c) o[c] = {R(0), R(0)};
    const int KXi = signed_k(i, g.NX);
    if (col < ncol && abs(KXi) < g.TX) {
      const int ix = KXi >= 0 ? KXi : KXi + g.KXc;
      const int kz = kz0 + col;
      const R kx = R(g.wave[0] * KXi), kzr = R(g.wave[2] * kz);
      const Cx<R> z0 = Zt[ix * KC + col], z1 = Zt[(g.KXc + ix) * KC + col];
      const double k2 = obl_k2(g, deg, KXi, KYi, kz);
      const R ik2 = k2 > 0.0 ? R(1.0 / k2) : R(0);
      Cx<R> u[3];
      obl_zeta_to_u(KXi, kz, kx, ky, kzr, ik2, R(deg), z0, z1, u);
      if (KXi == 0 && KYi == 0 && kz == 0) {
#pragma unroll
        for (int d = 0; d < 3; ++d) u[d] = {R(ukd[d]), R(0)};
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) o[d] = u[d];
      if (NOUT == 6) {
        Cx<R> w[3];
        obl_omega(KXi, kz, kx, ky, kzr, z0, z1, w);
#pragma unroll
        for (int d = 0; d < 3; ++d) o[(3 + d) % NOUT] = w[d];
      }
    }
#pragma unroll
    for (int c = 0; c < NOUT; ++c) U[i * W + c * KC + col] = o[c];
  }
  __syncthreads();
  fft2_smem<R, -1, W>(U, scr, g.lx, 1, W, twx);
  for (int it = threadIdx.x; it < NOUT * g.NX * KC; it += blockDim.x) {
    const int col = it % KC, rest = it / KC, x = rest & (g.NX - 1), c = rest >> g.lx;
    if (col < ncol) out[(((size_t)c * g.NX + x) * g.KYc + iy) * g.TS + kz0 + col] = U[x * W + c * KC + col];
  }
}

// ---------------------------------------------------------------------------
// x pass, forward, of three spectra in (I1 layout) with the update of zeta:
//   ADV = 1: in = the advection term u x omega.  A -= 2 S_eff (1, deg, 0) u^y_k
//            (operate_omega.cxx:155-164; u^y_k of the zeta at the start of the
//            step, recomputed here), curl (U_k2rotation_k, fft_wrapper.cxx:
//            679-722), Omega_k2zeta_k_OBL (fft_wrapper.cxx:175-197) and the
//            slaved-Euler step with the oblique K2 (fluid_solver.cxx:398-430);
//   ADV = 0: in = the contravariant u of the end of the step: Solenoidal_uk_OBL
//            (operate_omega.cxx:222-263), contra2co (fft_wrapper.h:327-361),
//            U_k2zeta_k_OBL with uk_dc = co2contra(u_co(0)) (fft_wrapper.cxx:
//            341-406), all with the updated degree_oblique.
// grid (KYc, ceil(TZ/KC)).
template <typename R, int KC, int ADV>
__global__ void __launch_bounds__(256) k_x_obl_fwd(Geo g, Twiddles<R> tw, const Cx<R> *__restrict__ in,
                                                   Cx<R> *__restrict__ zeta, double *__restrict__ uk_dc,
                                                   const double *__restrict__ st) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int W = 3 * KC;
  Cx<R> *twx = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *Pb = twx + g.NX;  // [NX][3*KC]
  Cx<R> *scr = Pb + g.NX * W;
  const int iy = blockIdx.x;
  const int kz0 = blockIdx.y * KC;
  const int ncol = min(KC, g.TZ - kz0);
  const size_t cstr = (size_t)g.NX * g.KYc * g.TS;
  const size_t zplane = (size_t)g.KXc * g.KYc * g.TS;
  for (int it = threadIdx.x; it < 3 * g.NX * KC; it += blockDim.x) {
    const int col = it % KC, rest = it / KC, x = rest & (g.NX - 1), c = rest >> g.lx;
    Cx<R> *d = Pb + x * W + c * KC + col;
    if (col < ncol)
      cp_async_cx(d, in + c * cstr + ((size_t)x * g.KYc + iy) * g.TS + kz0 + col);
    else
      *d = {R(0), R(0)};
  }
  load_twiddles(twx, tw.x, g.NX);
  cp_async_wait_all();
  __syncthreads();
  fft2_smem<R, 1, W>(Pb, scr, g.lx, 1, W, twx);
  const double deg = st[OB_DEG];
  const R degr = R(deg);
  const int KYi = signed_k(full_from_compact(iy, g.TY, g.KYc, g.NY), g.NY);
  const R ky = R(g.wave[1] * KYi);
  for (int it = threadIdx.x; it < g.KXc * KC; it += blockDim.x) {
    const int col = it % KC, ix = it / KC;
    if (col >= ncol) continue;
    const int KXi = ix < g.TX ? ix : ix - g.KXc;
    const int i = KXi >= 0 ? KXi : KXi + g.NX;
    const int kz = kz0 + col;
    const size_t o = ((size_t)ix * g.KYc + iy) * g.TS + kz;
    const Cx<R> *p = Pb + i * W + col;
    const R kx = R(g.wave[0] * KXi), kzr = R(g.wave[2] * kz);
    const double k2 = obl_k2(g, deg, KXi, KYi, kz);
    const R ik2 = k2 > 0.0 ? R(1.0 / k2) : R(0);
    const bool k0 = (KXi == 0 && KYi == 0 && kz == 0);
    if (ADV) {
      Cx<R> z0 = zeta[o], z1 = zeta[zplane + o];
      Cx<R> uo[3];
      obl_zeta_to_u(KXi, kz, kx, ky, kzr, ik2, degr, z0, z1, uo);
      const R uy_re = k0 ? R(uk_dc[1]) : uo[1].x, uy_im = k0 ? R(0) : uo[1].y;
      const R s2 = R(2.0 * st[OB_SRATE]), s2d = R(2.0 * st[OB_SRATE] * deg);
      const Cx<R> a0 = {p[0].x - s2 * uy_re, p[0].y - s2 * uy_im};
      const Cx<R> a1 = {p[KC].x - s2d * uy_re, p[KC].y - s2d * uy_im};
      const Cx<R> a2 = p[2 * KC];
      Cx<R> w[3];
      w[0] = {ky * a2.y - kzr * a1.y, -(ky * a2.x - kzr * a1.x)};
      w[1] = {kzr * a0.y - kx * a2.y, -(kzr * a0.x - kx * a2.x)};
      w[2] = {kx * a1.y - ky * a0.y, -(kx * a1.x - ky * a0.x)};
      Cx<R> f0, f1;
      if (KXi != 0) {
        f0 = w[1];
        f1 = w[2];
      } else if (kz != 0) {
        f0 = w[1];
        f1 = w[0];
      } else {
        f0 = w[0];
        f1 = w[2];
      }
      const double arg = -g.nu * g.dt * k2;
      const R dmy = R(g.fp64_exp ? exp(arg) - 1.0 : expm1(arg));
      const R c1 = R(1.0 / g.nu) * ik2;
      z0 = {z0.x + dmy * (z0.x - c1 * f0.x), z0.y + dmy * (z0.y - c1 * f0.y)};
      z1 = {z1.x + dmy * (z1.x - c1 * f1.x), z1.y + dmy * (z1.y - c1 * f1.y)};
      zeta[o] = z0;
      zeta[zplane + o] = z1;
    } else {
      Cx<R> u0 = p[0], u1 = p[KC], u2 = p[2 * KC];
      const R kxc = (R(1) + degr * degr) * kx - degr * ky;
      const R kyc = -degr * kx + ky;
      const Cx<R> dm = {ik2 * (u0.x * kx + u1.x * ky + u2.x * kzr), ik2 * (u0.y * kx + u1.y * ky + u2.y * kzr)};
      u0 = {u0.x - dm.x * kxc, u0.y - dm.y * kxc};
      u1 = {u1.x - dm.x * kyc, u1.y - dm.y * kyc};
      u2 = {u2.x - dm.x * kzr, u2.y - dm.y * kzr};
      const R dd = R(1) + degr * degr;
      const Cx<R> c0 = {u0.x + degr * u1.x, u0.y + degr * u1.y};
      const Cx<R> c1 = {degr * u0.x + dd * u1.x, degr * u0.y + dd * u1.y};
      const Cx<R> c2 = u2;
      Cx<R> w[3];
      w[0] = {ky * c2.y - kzr * c1.y, -(ky * c2.x - kzr * c1.x)};
      w[1] = {kzr * c0.y - kx * c2.y, -(kzr * c0.x - kx * c2.x)};
      w[2] = {kx * c1.y - ky * c0.y, -(kx * c1.x - ky * c0.x)};
      if (KXi != 0) {
        zeta[o] = w[1];
        zeta[zplane + o] = w[2];
      } else if (kz != 0) {
        zeta[o] = w[1];
        zeta[zplane + o] = w[0];
      } else {
        zeta[o] = w[0];
        zeta[zplane + o] = w[2];
      }
      if (k0) {
        // co2contra_single of the real parts (fft_wrapper.h:412-423)
        const double a = (double)c0.x, b = (double)c1.x;
        uk_dc[0] = (1. + deg * deg) * a - deg * b;
        uk_dc[1] = -deg * a + b;
        uk_dc[2] = (double)c2.x;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Real-space kernels over [c][NX][NY][NZ] fields (pitch NZ).

// u x omega (operate_omega.cxx:131-150): uw = [u0 u1 u2 w0 w1 w2] -> out[3].
template <typename R>
__global__ void k_obl_cross(size_t n, const R *__restrict__ uw, R *__restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const R u1 = uw[i], u2 = uw[n + i], u3 = uw[2 * n + i];
    const R w1 = uw[3 * n + i], w2 = uw[4 * n + i], w3 = uw[5 * n + i];
    out[i] = u2 * w3 - u3 * w2;
    out[n + i] = u3 * w1 - u1 * w3;
    out[2 * n + i] = u1 * w2 - u2 * w1;
  }
}

// degree_oblique += Shear_rate dt, Shear_rate_eff = Shear_rate, and the grid
// reset when it reaches 1 (sp_3d_ns.cxx:261,278-303).  One thread.  The
// product and the sum are rounded separately, as the reference computes them.
__global__ void k_obl_degree(OblPar o, double *__restrict__ st) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double deg = __dadd_rn(st[OB_DEG], __dmul_rn(o.shear_rate, o.dt));
  const int remap = deg >= 1.0;
  if (remap) deg = __dsub_rn(deg, 1.0);
  st[OB_DEG] = deg;
  st[OB_SRATE] = o.shear_rate;
  st[OB_REMAP] = (double)remap;
}

// Grid reset (sp_3d_ns.cxx:279-302): when the step passed degree_oblique = 1,
// out[0](i', j) = u0(i, j) + u1(i, j), out[1..2](i', j) = u(i, j) with
// i' = i + j - NY/2 (mod NX); otherwise a copy.
template <typename R>
__global__ void k_obl_remap(OblPar o, const double *__restrict__ st, const R *__restrict__ in, R *__restrict__ out) {
  const size_t n = (size_t)o.NX * o.NY * o.NZ;
  const bool remap = st[OB_REMAP] != 0.0;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(e % o.NZ);
    const int j = (int)((e / o.NZ) % o.NY);
    const int id = (int)(e / ((size_t)o.NZ * o.NY));
    if (!remap) {
      for (int c = 0; c < 3; ++c) out[c * n + e] = in[c * n + e];
      continue;
    }
    const int i = ((id - (j - o.NY / 2)) % o.NX + o.NX) % o.NX;
    const size_t s = ((size_t)i * o.NY + j) * o.NZ + k;
    out[e] = in[s] + in[n + s];
    out[n + e] = in[n + s];
    out[2 * n + e] = in[2 * n + s];
  }
}

// Interpolation weights of row j (U_oblique2u, fft_wrapper.h:292-300):
// returns the x shift i_ob - i, alpha and the sign of j - NY/2.
__device__ __forceinline__ int obl_row_o2c(int j, int NY, double deg, double &alpha, double &sign) {
  sign = (double)(j - NY / 2);
  if (!(sign == 0)) sign = sign / fabs(sign);
  const double jd = (double)j - NY / 2.;
  const int io = (int)((double)(int)(sign * deg * jd) * sign + sign);
  alpha = ((double)io - deg * jd) * sign;
  return io;
}

// U_oblique2u (fft_wrapper.h:265-325): oblique-grid contravariant u -> the
// Cartesian u of the sheared frame plus the mean shear flow S (y - NY/2).
// out(i_ob) from in(i), in(i + sign) where i_ob = i + shift (mod NX).
template <typename R>
__global__ void k_obl_to_cart(OblPar o, const double *__restrict__ st, const R *__restrict__ in, R *__restrict__ out) {
  const size_t n = (size_t)o.NX * o.NY * o.NZ;
  const double deg = st[OB_DEG], srate = st[OB_SRATE];
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(e % o.NZ);
    const int j = (int)((e / o.NZ) % o.NY);
    const int iob = (int)(e / ((size_t)o.NZ * o.NY));
    double alpha, sign;
    const int io = obl_row_o2c(j, o.NY, deg, alpha, sign);
    const double beta = 1. - alpha;
    const int i = ((iob - io) % o.NX + o.NX) % o.NX;
    const int ip = ((i + (int)sign) % o.NX + o.NX) % o.NX;
    const size_t s = ((size_t)i * o.NY + j) * o.NZ + k, sp = ((size_t)ip * o.NY + j) * o.NZ + k;
    const double w1 = beta * (double)in[n + s] + alpha * (double)in[n + sp];
    out[e] = (R)((beta * (double)in[s] + alpha * (double)in[sp]) + deg * w1 + srate * ((double)j - o.NY / 2.));
    out[n + e] = (R)w1;
    out[2 * n + e] = (R)(beta * (double)in[2 * n + s] + alpha * (double)in[2 * n + sp]);
  }
}

// f = up' - phi' u with the phi > 1 clamp of Make_phi_u_primitive_OBL
// (make_phi.cxx:366-383; f_particle.h:41-64), Cartesian grid.  phi/up are
// cleared for the next scatter.
template <typename R>
__global__ void k_obl_force(size_t n, R *__restrict__ phiup, const R *__restrict__ u, R *__restrict__ f) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    R ph = phiup[i];
    R up[3] = {phiup[n + i], phiup[2 * n + i], phiup[3 * n + i]};
    if (ph > R(1)) {
      const R inv = R(1) / ph;
      for (int d = 0; d < 3; ++d) up[d] *= inv;
      ph = R(1);
    }
    for (int d = 0; d < 3; ++d) f[d * n + i] = up[d] - ph * u[d * n + i];
    for (int d = 0; d < 4; ++d) phiup[d * n + i] = R(0);
  }
}

// u += U2u_oblique(f) (fft_wrapper.h:204-263, f_particle.h:83-99): the
// Cartesian force interpolated back to the oblique grid, as contravariant
// components.
template <typename R>
__global__ void k_obl_add_force(OblPar o, const double *__restrict__ st, const R *__restrict__ f, R *__restrict__ u) {
  const size_t n = (size_t)o.NX * o.NY * o.NZ;
  const double deg = st[OB_DEG];
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(e % o.NZ);
    const int j = (int)((e / o.NZ) % o.NY);
    const int i = (int)(e / ((size_t)o.NZ * o.NY));
    double sign = (double)(j - o.NY / 2);
    if (!(sign == 0)) sign = sign / fabs(sign);
    const double jd = (double)(j - o.NY / 2);
    const int io = (int)((double)(int)(sign * deg * jd) * sign);
    const double alpha = (deg * jd - (double)io) * sign, beta = 1. - alpha;
    const int iob = ((i + io) % o.NX + o.NX) % o.NX;
    const int iobp = ((iob + (int)sign) % o.NX + o.NX) % o.NX;
    const size_t s = ((size_t)iob * o.NY + j) * o.NZ + k, sp = ((size_t)iobp * o.NY + j) * o.NZ + k;
    const double g1 = beta * (double)f[n + s] + alpha * (double)f[n + sp];
    const double g0 = (beta * (double)f[s] + alpha * (double)f[sp]) - deg * g1;
    const double g2 = beta * (double)f[2 * n + s] + alpha * (double)f[2 * n + sp];
    u[e] = (R)((double)u[e] + g0);
    u[n + e] = (R)((double)u[n + e] + g1);
    u[2 * n + e] = (R)((double)u[2 * n + e] + g2);
  }
}

// Calc_shear_rate_eff (sp_3d_ns.h:174-196): the mean of d u0/dy over the
// NY-1 interior y differences, in two launches (partial sums per block,
// compensated, then the final sum by one block).
template <typename R>
__global__ void __launch_bounds__(256) k_obl_srate_partial(OblPar o, const R *__restrict__ u0, double *__restrict__ st) {
  __shared__ double sh[2 * 32];
  const size_t nterm = (size_t)o.NX * (o.NY - 1) * o.NZ;
  KSum s{0.0, 0.0};
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nterm; e += (size_t)gridDim.x * blockDim.x) {
    const int k = (int)(e % o.NZ);
    const int j = (int)((e / o.NZ) % (o.NY - 1));
    const int i = (int)(e / ((size_t)o.NZ * (o.NY - 1)));
    const size_t a = ((size_t)i * o.NY + j) * o.NZ + k;
    s.add(((double)u0[a + o.NZ] - (double)u0[a]) / o.dx);
  }
  KSum v[1] = {s};
  block_reduce<1>(v, sh);
  if (threadIdx.x == 0) {
    st[OB_PART + 2 * blockIdx.x] = v[0].s;
    st[OB_PART + 2 * blockIdx.x + 1] = v[0].c;
  }
}
__global__ void k_obl_srate_final(OblPar o, double *__restrict__ st, int nblocks) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  KSum s{0.0, 0.0};
  double c = 0.0;
  for (int b = 0; b < nblocks; ++b) {
    s.add(st[OB_PART + 2 * b]);
    c += st[OB_PART + 2 * b + 1];
  }
  const double srate = (s.s + (s.c + c)) * o.srate_scale;
  st[OB_SRATE] = srate;
  st[OB_STRAIN] += srate * o.dt;
}

// ---------------------------------------------------------------------------
// Particles under Lees-Edwards boundaries.

// Relative_coord_check_stepover_Y (make_phi.h:198-236): mesh index and offset
// of one Sekibun point; returns the y image crossing (-1, 0, 1), across which
// x is shifted by degree_oblique NY cells.
__device__ __forceinline__ int obl_stencil_point(const StencilBase &b, const int *cell, const PPar &p, double deg,
                                                 int rm[3], double r[3]) {
  double signY = (double)(b.xi[1] + cell[1]);
  rm[1] = (b.xi[1] + cell[1] + p.N[1]) % p.N[1];
  signY -= (double)rm[1];
  int sign = (int)signY;
  if (!(sign == 0)) sign = sign / abs(sign);
  const double xo = (double)b.xi[0] - (double)sign * deg * (double)p.N[1] + b.res[0] / p.DX + (double)cell[0] +
                    (double)(4 * p.N[0]);
  double xm = fmod(xo, (double)p.N[0]);
  if (xm < 0.0) xm += (double)p.N[0];  // only past 4 box lengths of shift; keeps the index inside the field
  rm[0] = min((int)xm, p.N[0] - 1);
  const double xres = xm - (double)rm[0];
  rm[2] = (b.xi[2] + cell[2] + p.N[2]) % p.N[2];
  r[0] = (double)cell[0] * p.DX - xres * p.DX;
  r[1] = (double)cell[1] * p.DX - b.res[1];
  r[2] = (double)cell[2] * p.DX - b.res[2];
  return sign;
}

// PBC_OBL (periodic_boundary.h:22-42) of one position; returns the crossing
// sign; x is shifted by deg*Ly across a y boundary.
__device__ __forceinline__ int pbc_obl(double *x, const PPar &p, double deg) {
  double signY = x[1];
  x[1] = fmod(x[1] + p.L[1], p.L[1]);
  signY -= x[1];
  int sign = (int)signY;
  if (!(sign == 0)) sign = sign / abs(sign);
  x[0] -= (double)sign * deg * p.L[1];
  x[0] = fmod(x[0] + p.L[0], p.L[0]);
  x[2] = fmod(x[2] + p.L[2], p.L[2]);
  return sign;
}

// MD_solver_position_Euler_OBL / _AB2_OBL (particle_solver.cxx:292-346).
__global__ void k_obl_position(PPar p, DPart *__restrict__ parts, int euler, const double *__restrict__ st,
                               int *__restrict__ status) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= p.Np || p.frozen) return;
  DPart &a = parts[n];
  const double hdt = 0.5 * p.dt;
  for (int d = 0; d < 3; ++d) {
    const double dx = euler ? p.dt * a.v[d] : hdt * (3.0 * a.v[d] - a.v_old[d]);
    a.x_nopbc[d] += dx;
    a.x[d] += dx;
  }
  const int sign = pbc_obl(a.x, p, st[OB_DEG]);
  const double dvx = -(double)sign * st[OB_SRATE] * p.L[1];
  a.v[0] += dvx;
  a.v_old[0] += dvx;
  for (int d = 0; d < 3; ++d)
    if (!(a.x[d] >= 0.0 && a.x[d] < p.L[d])) atomicExch(status, -6);
  if (p.rotation) orientation_update(p, a, euler);
}

// Distance0_OBL (interaction.h:39-65): x12 = LE-image of x2 - x1.
__device__ __forceinline__ double distance_obl(const double *x1, const double *x2, const PPar &p, double deg,
                                               double x12[3]) {
  double dmy = 0.0;
  double signY = x2[1] - x1[1];
  x12[1] = x2[1] - x1[1];
  x12[1] -= nint_d(x12[1] / p.L[1]) * p.L[1];
  signY -= x12[1];
  int sign = (int)signY;
  if (!(sign == 0)) sign = sign / abs(sign);
  dmy += x12[1] * x12[1];
  x12[0] = x2[0] - (x1[0] + (double)sign * deg * p.L[1]);
  x12[0] -= nint_d(x12[0] / p.L[0]) * p.L[0];
  dmy += x12[0] * x12[0];
  x12[2] = x2[2] - x1[2];
  x12[2] -= nint_d(x12[2] / p.L[2]) * p.L[2];
  dmy += x12[2] * x12[2];
  return sqrt(dmy);
}

// Calc_f_hydro_correct_precision_OBL (md_force.cxx:391-520) on the Cartesian
// velocity, Force_OBL (particle_solver.h:111-128: all-pairs LJ,
// md_force.cxx:136-179, then gravity), MD_solver_velocity_Euler_OBL /
// _AB2_hydro_OBL (particle_solver.cxx:348-440) and the thermostat kick.
// One block per particle; the pair forces are summed by thread 0 in the
// reference's order (partner index ascending).
template <typename R>
__global__ void __launch_bounds__(256) k_obl_hydro_velocity(PPar p, DPart *__restrict__ parts,
                                                            const R *__restrict__ u, const int *__restrict__ cells,
                                                            const double *__restrict__ noise, int euler,
                                                            const double *__restrict__ st, int *__restrict__ status) {
  __shared__ double sh[2 * 6 * 32];
  const int n = blockIdx.x;
  DPart &a = parts[n];
  const double deg = st[OB_DEG], srate = st[OB_SRATE];
  const double xp[3] = {a.x[0], a.x[1], a.x[2]};
  const double vp[3] = {a.v[0], a.v[1], a.v[2]};
  const double wp[3] = {a.omega[0], a.omega[1], a.omega[2]};
  const StencilBase b = stencil_base(xp, p);
  const size_t npts = (size_t)p.N[0] * p.N[1] * p.N[2];
  KSum acc[6];
  for (int i = 0; i < 6; ++i) acc[i] = {0.0, 0.0};
  for (int m = threadIdx.x; m < p.S; m += blockDim.x) {
    int rm[3];
    double r[3];
    const int sign = obl_stencil_point(b, cells + 3 * m, p, deg, rm, r);
    const double dist = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    const double ph = (double)prof_phi<R>(dist, p);
    double vr[3] = {0.0, 0.0, 0.0};
    if (p.rotation) {
      vr[0] = wp[1] * r[2] - wp[2] * r[1];
      vr[1] = wp[2] * r[0] - wp[0] * r[2];
      vr[2] = wp[0] * r[1] - wp[1] * r[0];
    }
    const size_t im = ((size_t)rm[0] * p.N[1] + rm[1]) * p.N[2] + rm[2];
    double fp[3];
    fp[0] = ((vp[0] - (double)sign * srate * p.L[1] + vr[0]) - (double)u[im]) * ph;
    fp[1] = ((vp[1] + vr[1]) - (double)u[npts + im]) * ph;
    fp[2] = ((vp[2] + vr[2]) - (double)u[2 * npts + im]) * ph;
    for (int d = 0; d < 3; ++d) acc[d].add(fp[d]);
    acc[3].add(r[1] * fp[2] - r[2] * fp[1]);
    acc[4].add(r[2] * fp[0] - r[0] * fp[2]);
    acc[5].add(r[0] * fp[1] - r[1] * fp[0]);
  }
  block_reduce<6>(acc, sh);
  if (threadIdx.x != 0) return;
  double fr[3] = {0.0, 0.0, 0.0};
  if (p.lj_on) {
    for (int j = 0; j < p.Np; ++j) {
      if (j == n) continue;
      double x12[3];
      const double rij = j < n ? distance_obl(parts[j].x, xp, p, deg, x12) : distance_obl(xp, parts[j].x, p, deg, x12);
      if (rij < p.lj_cut) {
        // Lennard_Jones_f (interaction.h:156-181)
        const double s = p.lj_dia / rij;
        double dmy = (s * s) * (s * s) * (s * s);
        if (p.lj_powers >= 1) dmy = dmy * dmy;
        if (p.lj_powers >= 2) dmy = dmy * (s * s) * (s * s) * (s * s);
        const double f = p.lj_coeff / (rij * rij) * (2.0 * dmy * dmy - dmy);
        for (int d = 0; d < 3; ++d) {
          const double d1 = f * -x12[d];
          fr[d] = j < n ? fr[d] - d1 : fr[d] + d1;
        }
      }
    }
  }
  fr[p.gdir] -= p.grav;
  double fh[3], th[3];
  for (int d = 0; d < 3; ++d) {
    fh[d] = p.fh_coef * (acc[d].s + acc[d].c);
    th[d] = p.rotation ? p.fh_coef * (acc[3 + d].s + acc[3 + d].c) : 0.0;
  }
  if (p.frozen) {
    for (int d = 0; d < 3; ++d) {
      a.fr_prev[d] = fr[d];
      a.f_hydro_prev[d] = fh[d];
      a.t_hydro_prev[d] = th[d];
    }
    return;
  }
  const double hdt = 0.5 * p.dt;
  for (int d = 0; d < 3; ++d) {
    a.v_old[d] = a.v[d];
    a.omega_old[d] = a.omega[d];
    if (euler) {
      const double dmy = p.dt * p.IMASS, dmy_rot = p.dt * p.IMOI;
      a.v[d] += dmy * (fh[d] + fr[d]);
      a.omega[d] += dmy_rot * th[d];
    } else {
      const double dmy = hdt * p.IMASS, dmy_rot = hdt * p.IMOI;
      a.v[d] += dmy * (2.0 * fh[d] + fr[d] + a.fr_prev[d]);
      a.omega[d] += dmy_rot * 2.0 * th[d];
    }
    a.fr_prev[d] = fr[d];
    a.f_hydro_prev[d] = fh[d];
    a.t_hydro_prev[d] = th[d];
  }
  if (p.thermostat) {
    const double *g = noise + 6 * (size_t)n;
    for (int d = 0; d < 3; ++d) {
      a.v[d] += g[d] * p.noise_v * p.IMASS;
      if (p.rotation) a.omega[d] += g[3 + d] * p.noise_o * p.IMOI;
    }
  }
  for (int d = 0; d < 3; ++d)
    if (!isfinite(a.v[d]) || !isfinite(a.omega[d])) atomicExch(status, -5);
}

// Make_phi_u_primitive_OBL scatter (make_phi.cxx:322-364): phi += phi_i,
// up += (v - sign S_eff Ly e_x + omega x r) phi_i.  PCL blocks per particle.
template <typename R>
__global__ void __launch_bounds__(256) k_obl_scatter(PPar p, const DPart *__restrict__ parts,
                                                     const int *__restrict__ cells, const double *__restrict__ st,
                                                     R *__restrict__ phiup) {
  const int n = blockIdx.x / PCL;
  const int stride = PCL * blockDim.x;
  const int first = (blockIdx.x % PCL) * blockDim.x + threadIdx.x;
  const DPart &a = parts[n];
  const double deg = st[OB_DEG], srate = st[OB_SRATE];
  const double xp[3] = {a.x[0], a.x[1], a.x[2]};
  const double vp[3] = {a.v[0], a.v[1], a.v[2]};
  const double wp[3] = {a.omega[0], a.omega[1], a.omega[2]};
  const StencilBase b = stencil_base(xp, p);
  const size_t npts = (size_t)p.N[0] * p.N[1] * p.N[2];
  for (int m = first; m < p.S; m += stride) {
    int rm[3];
    double r[3];
    const int sign = obl_stencil_point(b, cells + 3 * m, p, deg, rm, r);
    const double dist = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
    const double ph = (double)prof_phi<R>(dist, p);
    double vr[3] = {0.0, 0.0, 0.0};
    if (p.rotation) {
      vr[0] = wp[1] * r[2] - wp[2] * r[1];
      vr[1] = wp[2] * r[0] - wp[0] * r[2];
      vr[2] = wp[0] * r[1] - wp[1] * r[0];
    }
    const size_t im = ((size_t)rm[0] * p.N[1] + rm[1]) * p.N[2] + rm[2];
    atomicAdd(phiup + im, (R)ph);
    atomicAdd(phiup + npts + im, (R)(((vp[0] - (double)sign * srate * p.L[1]) + vr[0]) * ph));
    atomicAdd(phiup + 2 * npts + im, (R)((vp[1] + vr[1]) * ph));
    atomicAdd(phiup + 3 * npts + im, (R)((vp[2] + vr[2]) * ph));
  }
}

}  // namespace kapsel
