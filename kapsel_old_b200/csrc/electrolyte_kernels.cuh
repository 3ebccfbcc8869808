// Kernels of the Electrolyte branch of the SPM step (two ion species):
// NSsolute_solver_Euler with Rhs_NS_Nernst_Planck (fluid_solver.cxx:243-326),
// solute_rhs.cxx, operate_electrolyte.cxx and the electrolyte part of
// Time_evolution_hydro (sp_3d_ns.cxx:89-122).
//
// Generic x passes with a k-space operator, generic forward z pass, real-space
// point kernels, the particle scatter of phi / surface charge / surface
// normal, grid reductions and the Hermitian completion of the Ooura inverse.
#pragma once

#include "particle_kernels.cuh"
#include "spectral_kernels.cuh"

namespace kapsel {

struct KOp {
  double a;         // operator scale (1/eps, kBT*L, dt ...)
  double e_amp[3];  // value subtracted from the real part of the k=0 mode (GRADPSI)
};

enum { XI_IDENT = 0, XI_GRADPSI = 1, XI_GRADDIFF = 2 };
enum { XF_STORE = 0, XF_CONCUPD = 1, XF_GRADPSI_FULL = 2, XF_PSI_FULL = 3 };

// x pass, inverse, with a k-space operator on the (compact) input spectra:
//   XI_IDENT     out_c = in_c                        (NOUT == NIN)
//   XI_GRADPSI   out_d = -i k_d in_0 IK2 a, k=0: -e_amp   (A_k2da_k of the
//                Poisson potential, Charge_field_k2Coulomb_potential_k_PBC,
//                Add_constant_field_k; operate_electrolyte.cxx:76-88,
//                fluid_solver.cxx:228-241)
//   XI_GRADDIFF  out_d = -i k_d a in_0                (Diffusion_flux_single,
//                solute_rhs.cxx:214-234)
// in: [NIN][KXc][KYc][TZ] (planes in_cstride apart), out I1: [NOUT][NX][KYc][TZ].
template <typename R, int KC, int OP, int NIN, int NOUT>
__global__ void __launch_bounds__(256) k_x_inv_op(Geo g, Twiddles<R> tw, const Cx<R> *__restrict__ in,
                                                  size_t in_cstride, Cx<R> *__restrict__ out, KOp op) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int W = NOUT * KC;
  Cx<R> *twx = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *Zt = twx + g.NX;            // [NIN][KXc][KC]
  Cx<R> *U = Zt + NIN * g.KXc * KC;  // [NX][NOUT*KC]
  Cx<R> *scr = U + g.NX * W;
  const int iy = blockIdx.x;
  const int kz0 = blockIdx.y * KC;
  const int ncol = min(KC, g.TZ - kz0);
  for (int it = threadIdx.x; it < NIN * g.KXc * KC; it += blockDim.x) {
    const int col = it % KC, rest = it / KC, ix = rest % g.KXc, c = rest / g.KXc;
    if (col < ncol) cp_async_cx(Zt + it, in + c * in_cstride + ((size_t)ix * g.KYc + iy) * g.TS + kz0 + col);
  }
  load_twiddles(twx, tw.x, g.NX);
  cp_async_wait_all();
  __syncthreads();
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
      if (OP == XI_IDENT) {
#pragma unroll
        for (int c = 0; c < NOUT; ++c) o[c] = Zt[(c * g.KXc + ix) * KC + col];
      } else {
        const R kx = R(g.wave[0] * KXi), kzr = R(g.wave[2] * kz);
        const Cx<R> a = Zt[ix * KC + col];
        R s = R(op.a);
        if (OP == XI_GRADPSI) {
          const R k2 = kx * kx + ky * ky + kzr * kzr;
          s = k2 > R(0) ? s / k2 : R(0);
        }
        const Cx<R> v = {a.x * s, a.y * s};
        const R kk[3] = {kx, ky, kzr};
#pragma unroll
        for (int d = 0; d < 3 && d < NOUT; ++d) o[d] = {kk[d] * v.y, -kk[d] * v.x};  // -i k v
        if (OP == XI_GRADPSI && KXi == 0 && KYi == 0 && kz == 0) {
#pragma unroll
          for (int d = 0; d < 3 && d < NOUT; ++d) o[d] = {R(-op.e_amp[d]), R(0)};
        }
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

// x pass, forward, of NIN spectra (I1 layout) with an operator on the kept modes:
//   XF_STORE         out[o] = X_0                       (compact spectrum)
//   XF_CONCUPD       out[o] += a * (-i k.X)             (U_k2divergence_k + the
//                    concentration part of Field_solver_Euler, fluid_solver.cxx:122-135)
//   XF_GRADPSI_FULL  out[d][o] = -i k_d X_0 IK2 a       (full spectrum, no truncation:
//                    Make_Coulomb_force_x_on_fluid, operate_electrolyte.cxx:97-101)
//   XF_PSI_FULL      out[o] = X_0 IK2 a                 (full spectrum: the Coulomb
//                    potential of Output_avs_charge, avs_output.cxx:464-466)
// out planes are out_cstride apart.
template <typename R, int KC, int OP, int NIN>
__global__ void __launch_bounds__(256) k_x_fwd_op(Geo g, Twiddles<R> tw, const Cx<R> *__restrict__ in,
                                                  Cx<R> *__restrict__ out, size_t out_cstride, KOp op) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int W = NIN * KC;
  Cx<R> *twx = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *Pb = twx + g.NX;  // [NX][NIN*KC]
  Cx<R> *scr = Pb + g.NX * W;
  const int iy = blockIdx.x;
  const int kz0 = blockIdx.y * KC;
  const int ncol = min(KC, g.TZ - kz0);
  const size_t cstr = (size_t)g.NX * g.KYc * g.TS;
  for (int it = threadIdx.x; it < NIN * g.NX * KC; it += blockDim.x) {
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
    if (OP == XF_STORE) {
      out[o] = p[0];
    } else if (OP == XF_CONCUPD) {
      const Cx<R> f0 = p[0], f1 = p[KC], f2 = p[2 * KC];
      const Cx<R> dv = {kx * f0.y + ky * f1.y + kzr * f2.y, -(kx * f0.x + ky * f1.x + kzr * f2.x)};
      const R dt = R(op.a);
      out[o] = {out[o].x + dt * dv.x, out[o].y + dt * dv.y};
    } else if (OP == XF_PSI_FULL) {
      const R k2 = kx * kx + ky * ky + kzr * kzr;
      const R s = k2 > R(0) ? R(op.a) / k2 : R(0);
      out[o] = {p[0].x * s, p[0].y * s};
    } else {
      const R k2 = kx * kx + ky * ky + kzr * kzr;
      const R s = k2 > R(0) ? R(op.a) / k2 : R(0);
      const Cx<R> v = {p[0].x * s, p[0].y * s};
      out[o] = {kx * v.y, -kx * v.x};
      out[out_cstride + o] = {ky * v.y, -ky * v.x};
      out[2 * out_cstride + o] = {kzr * v.y, -kzr * v.x};
    }
  }
}

// Forward z transform of real fields, kz < nkeep kept:
// in [c][rows][pitch] (planes in_cstride apart) -> out [c][rows][ostride], k < nkeep.
template <typename R>
__global__ void __launch_bounds__(256) k_z_r2c(Geo g, Twiddles<R> tw, const R *__restrict__ in, int in_pitch,
                                               size_t in_cstride, Cx<R> *__restrict__ out, int nkeep, int ostride) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int M = g.M;
  constexpr int ES = ZROWS + 1;
  Cx<R> *twm = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *twz = twm + M;
  Cx<R> *S = twz + g.NZ;    // [M][ES]
  Cx<R> *scr = S + M * ES;  // FFT scratch, then the output tile [ZROWS][nkeep+1]
  load_twiddles(twm, tw.m, M);
  load_twiddles(twz, tw.z, g.NZ);
  const int c = blockIdx.y;
  const size_t rows = (size_t)g.NX * g.NY;
  const size_t row0 = (size_t)blockIdx.x * ZROWS;
  const R *src = in + c * in_cstride;
  for (int it = threadIdx.x; it < ZROWS * M; it += blockDim.x) {
    const int n = it & (M - 1), rr = it >> g.lm;
    const R *r = src + (row0 + rr) * (size_t)in_pitch + 2 * n;
    S[n * ES + rr] = {r[0], r[1]};
  }
  __syncthreads();
  fft2_smem<R, 1, ZROWS>(S, scr, g.lm, 1, ES, twm);
  const int TA = nkeep + 1;
  for (int it = threadIdx.x; it < ZROWS * nkeep; it += blockDim.x) {
    const int rr = it % ZROWS, k = it / ZROWS;
    scr[rr * TA + k] = r2c_post(S + rr, ES, k, M, twz);
  }
  __syncthreads();
  Cx<R> *dst = out + c * rows * ostride + row0 * ostride;
  for (int it = threadIdx.x; it < ZROWS * nkeep; it += blockDim.x) {
    const int k = it % nkeep, rr = it / nkeep;
    dst[rr * ostride + k] = scr[rr * TA + k];
  }
}

// Hermitian completion of the kz = 0 and kz = NZ/2 planes of full spectra
// [c][NX][NY][M+1], as the Ooura inverse (rdft3dsort isgn<0,
// fftsg3d.c:645-668) reads them: on each plane one half is kept and the
// other half is the conjugate of its partner (-i,-j); at the four
// self-conjugate points only the real part is kept.  grid-stride over
// (c, plane, i, j).
template <typename R>
__global__ void k_hermitian_planes(Geo g, Cx<R> *__restrict__ spec, int ncomp) {
  const int M1 = g.TS;  // row stride of the [c][NX][NY][M+1] spectra
  const int n1 = g.NX, n2 = g.NY, n1h = n1 / 2, n2h = n2 / 2;
  const size_t cstr = (size_t)n1 * n2 * M1;
  const int total = ncomp * 2 * n1 * n2;
  for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < total; it += gridDim.x * blockDim.x) {
    const int j = it % n2, i = (it / n2) % n1, pl = (it / (n1 * n2)) % 2, c = it / (2 * n1 * n2);
    const int kz = pl ? g.M : 0;
    const bool edge = (j == 0 || j == n2h);
    const bool keep = pl ? (j > n2h || (edge && i >= n1h)) : ((j > 0 && j < n2h) || (edge && i <= n1h));
    const bool selfc = (i == 0 || i == n1h) && edge;
    Cx<R> *base = spec + c * cstr;
    const size_t o = ((size_t)i * n2 + j) * M1 + kz;
    if (!keep) {
      const int pi = (n1 - i) & (n1 - 1), pj = (n2 - j) & (n2 - 1);
      const Cx<R> p = base[((size_t)pi * n2 + pj) * M1 + kz];
      base[o] = selfc ? Cx<R>{p.x, R(0)} : Cx<R>{p.x, -p.y};
    } else if (selfc) {
      base[o].y = R(0);
    }
  }
}

// DPhi_compact_sin (profile.h:168-181) with radius RADIUS and xi = 2 HXI.
__device__ __forceinline__ double dphi_compact_sin(double x, const PPar &p) {
  const double xi = 2.0 * p.HXI, hxi = p.HXI;
  const double dmy = p.RADIUS - x;
  return fabs(dmy) < hxi ? M_PI * .5 * (1.0 / xi) * cos(M_PI * dmy * (1.0 / xi)) : 0.0;
}

// Scatter of the particle fields the electrolyte needs, one block per
// (particle, quarter of the Sekibun points):
//   out[0] += Phi            (Make_phi_particle, make_phi.cxx:388-400: no clamp)
//   out[1] += ze DPhi        (Make_phi_qq_particle, operate_electrolyte.cxx:179-216)
//   out[2..4] += r/|r|  where ||r| - RADIUS| < HXI (Make_surface_normal,
//                           make_phi.cxx:17-58), when with_normal
template <typename R>
__global__ void __launch_bounds__(256) k_particles_scatter_el(PPar p, const DPart *__restrict__ parts,
                                                              const int *__restrict__ cells, R *__restrict__ out,
                                                              double ze, int with_normal) {
  const int n = blockIdx.x / PCL;
  const int stride = PCL * blockDim.x;
  const int first = (blockIdx.x % PCL) * blockDim.x + threadIdx.x;
  const DPart &a = parts[n];
  const double xp[3] = {a.x[0], a.x[1], a.x[2]};
  const StencilBase b = stencil_base(xp, p);
  const size_t npts = (size_t)p.N[0] * p.N[1] * p.N[2];
  for (int m = first; m < p.S; m += stride) {
    int rm[3];
    double r[3], dist;
    stencil_point(b, cells + 3 * m, xp, p, rm, r, dist);
    const size_t im = ((size_t)rm[0] * p.N[1] + rm[1]) * p.N[2] + rm[2];
    atomicAdd(out + im, (R)prof_phi<double>(dist, p));
    const double dq = ze * dphi_compact_sin(dist, p);
    if (dq != 0.0) atomicAdd(out + npts + im, (R)dq);
    if (with_normal) {
      const double rr = sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
      if (fabs(rr - p.RADIUS) < p.HXI) {
        const double ir = 1. / rr;
        for (int d = 0; d < 3; ++d) atomicAdd(out + (2 + d) * npts + im, (R)(r[d] * ir));
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Grid reductions (two launches: per-block partial sums, then one block adds
// them in a fixed order, so the result does not depend on scheduling).
//   RED_ABS:   sum |a[i]|                              -> 1 value
//   RED_PHI_C: sum (1 - phi[i]) c_n[i], n = 0..nc-1    -> nc values
//   RED_1MPHI: sum (1 - phi[i])                        -> 1 value
enum { RED_ABS = 0, RED_PHI_C = 1, RED_1MPHI = 2 };
constexpr int RED_BLOCKS = 592;

template <typename R, int MODE>
__global__ void __launch_bounds__(256) k_reduce_partial(size_t n, const R *__restrict__ a, const R *__restrict__ c,
                                                        size_t c_cstride, int nc, double *__restrict__ partial) {
  __shared__ double sh[2 * 2 * 32];
  KSum acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    if (MODE == RED_ABS) {
      acc[0].add(fabs((double)a[i]));
    } else if (MODE == RED_1MPHI) {
      acc[0].add(1.0 - (double)a[i]);
    } else {
      const double w = 1.0 - (double)a[i];
      for (int q = 0; q < nc; ++q) acc[q].add(w * (double)c[q * c_cstride + i]);
    }
  }
  block_reduce<2>(acc, sh);
  if (threadIdx.x == 0)
    for (int q = 0; q < 2; ++q) partial[(size_t)q * gridDim.x + blockIdx.x] = acc[q].s + acc[q].c;
}

// Final sums; then the electrolyte scalars:
//   what == 0: scal[0] = num / (sum0 * DX3)            (surface-charge rescale)
//   what == 1: scal[1+q] = tot[q] / (sum_q * DX3)      (Rescale_solute factors)
//   what == 2: scal[3] = sum0                          (free volume, init)
__global__ void k_reduce_final(const double *__restrict__ partial, int nblocks, int nc, int what, double num,
                               const double *__restrict__ tot, double dx3, double *__restrict__ scal) {
  __shared__ double sh[2 * 2 * 32];
  KSum acc[2] = {{0.0, 0.0}, {0.0, 0.0}};
  for (int q = 0; q < nc; ++q)
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) acc[q].add(partial[(size_t)q * nblocks + i]);
  block_reduce<2>(acc, sh);
  if (threadIdx.x == 0) {
    const double s0 = acc[0].s + acc[0].c, s1 = acc[1].s + acc[1].c;
    if (what == 0) scal[0] = num / (s0 * dx3);
    if (what == 1) {
      scal[1] = tot[0] / (s0 * dx3);
      if (nc > 1) scal[2] = tot[1] / (s1 * dx3);
    }
    if (what == 2) scal[3] = s0;
  }
}

// ---------------------------------------------------------------------------
// Real-space point kernels.
// charge = s0 surf + sum_n ve_n fac_n c_n (1 - phi)     (Conc_k2charge_field)
template <typename R>
__global__ void k_el_charge(size_t n, const R *__restrict__ phiq, const R *__restrict__ creal,
                            const double *__restrict__ scal, int use_fac, double ve0, double ve1,
                            R *__restrict__ charge) {
  const R qs = R(scal[0]);
  const R f0 = use_fac ? R(scal[1]) : R(1), f1 = use_fac ? R(scal[2]) : R(1);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const R w = R(1) - phiq[i];
    R q = qs * phiq[n + i];
    q += R(ve0) * (f0 * creal[i]) * w;
    q += R(ve1) * (f1 * creal[n + i]) * w;
    charge[i] = q;
  }
}

// Ion flux of one species (Solute_solver_rhs_nonlinear_x_single,
// Solute_impermeability, Add_advection_flux; solute_rhs.cxx:42-212):
// flux = diff + c L (ve grad); remove the normal part where |normal| > 0;
// flux -= c u.  flux holds the diffusion flux on entry.
template <typename R>
__global__ void k_el_flux(size_t n, R *__restrict__ flux, const R *__restrict__ c, const R *__restrict__ grad,
                          const R *__restrict__ normal, const R *__restrict__ u, size_t u_cstride, double L,
                          double ve) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const R ci = c[i];
    R f[3], nv[3];
    R n2 = R(0);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      f[d] = flux[d * n + i] + ci * (R(L) * (grad[d * n + i] * R(ve)));
      nv[d] = normal[d * n + i];
      n2 += nv[d] * nv[d];
    }
    if (n2 > R(0)) {
      R dm = f[0] * nv[0] + f[1] * nv[1] + f[2] * nv[2];
      dm /= n2;
#pragma unroll
      for (int d = 0; d < 3; ++d) f[d] -= nv[d] * dm;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) flux[d * n + i] = f[d] + ci * -u[d * u_cstride + i];
  }
}

// Coulomb body force (Make_Coulomb_force_x_on_fluid, operate_electrolyte.cxx:120-176)
// times dt/rho (the u += f dt/rho of sp_3d_ns.cxx:107-117).
template <typename R>
__global__ void k_el_coulomb(size_t n, const R *__restrict__ charge, const R *__restrict__ grad, double e0,
                             double e1, double e2, double scale, R *__restrict__ f) {
  const double e[3] = {e0, e1, e2};
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const R q = charge[i];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      R ef = -grad[d * n + i];
      ef += R(e[d]);
      f[d * n + i] = (q * ef) * R(scale);
    }
  }
}

// conc_k[n] *= fac[n] over the stored modes (Rescale_solute, solute_rhs.cxx:99-128)
template <typename R>
__global__ void k_scale_conc(size_t nz, Cx<R> *__restrict__ conc, const double *__restrict__ scal) {
  const R f0 = R(scal[1]), f1 = R(scal[2]);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < 2 * nz; i += (size_t)gridDim.x * blockDim.x) {
    const R f = i < nz ? f0 : f1;
    conc[i] = {conc[i].x * f, conc[i].y * f};
  }
}

}  // namespace kapsel
