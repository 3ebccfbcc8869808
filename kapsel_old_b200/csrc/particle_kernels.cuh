// Particle-side kernels of the SPM step.  Particle state is double precision
// in every mode; only the fields they read or scatter into follow R.
#pragma once

#include <cuda_runtime.h>

#include "fft_device.cuh"

namespace kapsel {

// One particle (the subset of Particle, variable.h:27-75, the step uses).
// *_prev hold the values reset_Forces (particle_solver.cxx:11-34) moves into
// f_hydro_previous / torque_hydro_previous / fr_previous.
struct DPart {
  double x[3], x_nopbc[3], v[3], v_old[3], omega[3], omega_old[3];
  double f_hydro_prev[3], t_hydro_prev[3], fr_prev[3];
  double q[4], q_old[4];
};

struct PPar {
  int Np, S;           // particles, Sekibun points per particle
  int N[3];
  double L[3], invL[3];
  double DX, RADIUS, HXI;
  double dt;
  double IMASS, IMOI;
  double fh_coef;      // -DX^3 RHO / dt (md_force.cxx:264-265)
  int rotation;
  int lj_on;           // LJ_truncate >= 0
  int lj_powers;
  double lj_dia, lj_cut, lj_coeff;  // sigma, A_R_cutoff*sigma, 24(p+1) EPSILON
  int lc[3];
  double lc_r;         // Cell_length * DX (md_force.cxx:21,48-53)
  double grav;         // Gravity_on_fluid * (MASS_RATIO - 1) (md_force.cxx:181-191)
  int gdir;
  int thermostat;
  double noise_v, noise_o;  // fluct.cxx:13-19
  int frozen;               // positions and velocities held; forces still measured
  int hyd_pcl;              // gather blocks per particle (at most HYD_PCL_MAX)
  int hyd_threads;          // threads per gather block (at most 1024)
  // per-particle neighbour lists ([Np][NBL_MAX + 1]: count, then indices in
  // increasing order) built each step for large particle counts; null: the
  // pair searches scan all particles
  const int *nbl = nullptr;
};

constexpr int NBL_MAX = 64;  // neighbours a list holds (more: KAPSEL_ERANGE)

__device__ __forceinline__ double nint_d(double a) {
  // Nint (macro.h:38-46): round half away from zero
  return a >= 0.0 ? (double)(int)(a + 0.5) : (double)(int)(a - 0.5);
}

// H and Phi (profile.h:29-49), evaluated in the field precision R: double
// for the FP64 path, float (fast exp) for the mixed path, whose profile
// stencils are single precision.
template <typename R>
__device__ __forceinline__ R prof_H(R x, R dx) {
  if (sizeof(R) == 8) return x > R(0) ? R(exp(-((dx / x) * (dx / x)))) : R(0);
  const float q = __fdividef((float)dx, (float)x);
  return x > R(0) ? R(__expf(-q * q)) : R(0);
}
template <typename R>
__device__ __forceinline__ R prof_phi(double x, const PPar &p) {
  const R xr = R(x);
  const R h = prof_H<R>(R(p.RADIUS + p.HXI) - xr, R(p.DX));
  // (x - radius) + HXI as in profile.h:47 for the double path
  const R h2 = prof_H<R>(sizeof(R) == 8 ? (xr - R(p.RADIUS)) + R(p.HXI) : xr - R(p.RADIUS - p.HXI), R(p.DX));
  return sizeof(R) == 8 ? h / (h + h2) : R(__fdividef((float)h, (float)(h + h2)));
}

// Phi of the mixed path with every argument in float: rp = RADIUS + HXI,
// rm = RADIUS - HXI (profile.h:29-49).
__device__ __forceinline__ float prof_phi_f(float x, float rp, float rm, float dx) {
  const float h = prof_H<float>(rp - x, dx), h2 = prof_H<float>(x - rm, dx);
  return __fdividef(h, h + h2);
}

// Stencil geometry shared by the gather and the scatter: Particle_cell
// (make_phi.h:102-130), Relative_coord (:143-160), Distance (interaction.h:110-133).
struct StencilBase {
  int xi[3];
  double res[3];
};
__device__ __forceinline__ StencilBase stencil_base(const double *x, const PPar &p) {
  StencilBase b;
  const double idx = 1.0 / p.DX;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double dmy = x[d] * idx;
    // positions are kept in [0, L) by the integrator; a position outside
    // (flagged through the status word) is folded back so that every grid
    // index stays inside the field
    if (!(dmy >= 0.0 && dmy < (double)p.N[d])) dmy = 0.0;
    b.xi[d] = (int)dmy;
    b.res[d] = (dmy - (double)b.xi[d]) * p.DX;
  }
  return b;
}
// Distance (interaction.h:110-133) from the particle centre xp to grid
// point rm under the minimum image, every operation rounded separately (as
// the reference's x86 build computes it, and identically wherever it is
// inlined: the deterministic scatter compares values computed at
// different sites).
__device__ __forceinline__ double point_dist(const double *xp, const int rm[3], const PPar &p) {
  double s = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double dd = __dsub_rn(xp[d], __dmul_rn((double)rm[d], p.DX));
    dd = __dsub_rn(dd, __dmul_rn(nint_d(__dmul_rn(dd, p.invL[d])), p.L[d]));
    s = __dadd_rn(s, __dmul_rn(dd, dd));
  }
  return __dsqrt_rn(s);
}
__device__ __forceinline__ void stencil_point(const StencilBase &b, const int *cell, const double *xp, const PPar &p,
                                              int rm[3], double r[3], double &dist) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    rm[d] = (b.xi[d] + cell[d] + p.N[d]) & (p.N[d] - 1);  // N is a power of two
    r[d] = __dsub_rn(__dmul_rn((double)cell[d], p.DX), b.res[d]);
  }
  dist = point_dist(xp, rm, p);
}
// The mixed path's offset of a stencil point from the sphere centre and its
// length, in float with every operation rounded separately.
__device__ __forceinline__ float offset_f(const int cell[3], const float resf[3], float dxf, float r[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) r[d] = __fsub_rn(__fmul_rn((float)cell[d], dxf), resf[d]);
  return __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(r[0], r[0]), __fmul_rn(r[1], r[1])), __fmul_rn(r[2], r[2])));
}

// Neumaier compensated accumulation.
struct KSum {
  double s, c;
  __device__ __forceinline__ void add(double v) {
    const double t = s + v;
    c += fabs(s) >= fabs(v) ? (s - t) + v : (v - t) + s;
    s = t;
  }
};

// ---------------------------------------------------------------------------
// quaternion helpers (quaternion.h:173-245, rigid_body.cxx:10-63)
__device__ __forceinline__ void qprod(const double *a, const double *b, double alpha, double *q) {
  q[0] = alpha * (a[0] * b[0] - (a[1] * b[1] + a[2] * b[2] + a[3] * b[3]));
  q[1] = alpha * (a[0] * b[1] + b[0] * a[1] + a[2] * b[3] - a[3] * b[2]);
  q[2] = alpha * (a[0] * b[2] + b[0] * a[2] + a[3] * b[1] - a[1] * b[3]);
  q[3] = alpha * (a[0] * b[3] + b[0] * a[3] + a[1] * b[2] - a[2] * b[1]);
}
__device__ __forceinline__ void space2body(const double *v, const double *q, double *out) {
  const double qx[4] = {0.0, v[0], v[1], v[2]};
  const double qc[4] = {q[0], -q[1], -q[2], -q[3]};
  double t[4], r[4];
  qprod(qx, q, 1.0, t);
  qprod(qc, t, 1.0, r);
  out[0] = r[1];
  out[1] = r[2];
  out[2] = r[3];
}
__device__ __forceinline__ void qnormalize(double *q) {
  double n = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
  n = 1.0 / n;
  for (int i = 0; i < 4; ++i) q[i] *= n;
}

// MD_solver_orientation_Euler / _AB2 (particle_rotation_solver.h:15-39).
__device__ __forceinline__ void orientation_update(const PPar &p, DPart &a, int euler) {
  const double hdt = 0.5 * p.dt;
  double dq[4];
  if (euler) {
    for (int i = 0; i < 4; ++i) a.q_old[i] = a.q[i];
    const double qw[4] = {0.0, a.omega[0], a.omega[1], a.omega[2]};
    qprod(qw, a.q, 0.5, dq);
    for (int i = 0; i < 4; ++i) a.q[i] += dq[i] * p.dt;
  } else {
    double wb[3], wbo[3];
    space2body(a.omega, a.q, wb);
    space2body(a.omega_old, a.q_old, wbo);
    for (int d = 0; d < 3; ++d) wb[d] = 3.0 * wb[d] - wbo[d];
    for (int i = 0; i < 4; ++i) a.q_old[i] = a.q[i];
    const double qw[4] = {0.0, wb[0], wb[1], wb[2]};
    qprod(a.q, qw, 0.5, dq);
    for (int i = 0; i < 4; ++i) a.q[i] += dq[i] * hdt;
  }
  qnormalize(a.q);
}

// MD_solver_position_Euler / _AB2 (particle_solver.cxx:36-88), PBC
// (periodic_boundary.h:9-15), MD_solver_orientation_Euler / _AB2
// (particle_rotation_solver.h:15-39).  One thread per particle.
__device__ __forceinline__ void position_update_one(const PPar &p, DPart *__restrict__ parts, int n, int euler,
                                                    int *__restrict__ status) {
  if (p.frozen) return;
  DPart &a = parts[n];
  const double hdt = 0.5 * p.dt;
  for (int d = 0; d < 3; ++d) {
    const double dx = euler ? p.dt * a.v[d] : hdt * (3.0 * a.v[d] - a.v_old[d]);
    a.x_nopbc[d] += dx;
    a.x[d] += dx;
    a.x[d] = fmod(a.x[d] + p.L[d], p.L[d]);
    if (!(a.x[d] >= 0.0 && a.x[d] < p.L[d])) atomicExch(status, -6);
  }
  if (p.rotation) orientation_update(p, a, euler);
}


__global__ void k_particles_position(PPar p, DPart *__restrict__ parts, int euler, int *__restrict__ status) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n < p.Np) position_update_one(p, parts, n, euler, status);
}

// Block reduction of NV compensated sums; result valid in thread 0.  Warps
// reduce with shuffles, then thread i < NV adds value i over the warps.
template <int NV>
__device__ void block_reduce(KSum (&v)[NV], double *sh /* [2*NV][32] */) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double s = v[i].s, c = v[i].c;
    for (int o = 16; o > 0; o >>= 1) {
      const double so = __shfl_down_sync(0xffffffffu, s, o);
      const double co = __shfl_down_sync(0xffffffffu, c, o);
      KSum k{s, c + co};
      k.add(so);
      s = k.s;
      c = k.c;
    }
    if (lane == 0) {
      sh[(2 * i) * 32 + wid] = s;
      sh[(2 * i + 1) * 32 + wid] = c;
    }
  }
  __syncthreads();
  if (threadIdx.x < NV) {
    const int i = threadIdx.x;
    KSum k{0.0, 0.0};
    double cs = 0.0;
    for (int w = 0; w < nw; ++w) {
      k.add(sh[(2 * i) * 32 + w]);
      cs += sh[(2 * i + 1) * 32 + w];
    }
    sh[(2 * i) * 32] = k.s;
    sh[(2 * i + 1) * 32] = k.c + cs;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      v[i].s = sh[(2 * i) * 32];
      v[i].c = sh[(2 * i + 1) * 32];
    }
  }
}

// Calc_f_hydro_correct_precision (md_force.cxx:263-389), the LJ and gravity
// forces of Force (particle_solver.h:97-109; md_force.cxx:23-134,181-191),
// MD_solver_velocity_Euler / _AB2_hydro with reset_Forces
// (particle_solver.cxx:106-147, 247-289, 11-34) and, when kBT > 0, the
// thermostat kick of Add_random_force_thermostat (fluct.cxx:10-36) from a
// precomputed table of its normals.
// The scatters run PCL blocks per particle.  The gather runs p.hyd_pcl
// blocks of p.hyd_threads threads per particle.  With one block per particle
// the block's sums are the particle's and thread 0 updates it; with several,
// each block stores its partial sums and the block that finishes last (a
// per-particle arrival counter) adds the partials in a fixed order -- the
// result does not depend on block scheduling -- and updates the particle.
constexpr int PCL = 4;
constexpr int HYD_PCL_MAX = 8;

template <typename R>
__global__ void __launch_bounds__(1024) k_particles_hydro_velocity(PPar p, DPart *__restrict__ parts,
                                                                  const R *__restrict__ u, const int *__restrict__ cells,
                                                                  const double *__restrict__ noise, int euler,
                                                                  int *__restrict__ status,
                                                                  double *__restrict__ partial,
                                                                  int *__restrict__ arrivals,
                                                                  double *__restrict__ nc_corr = nullptr,
                                                                  unsigned *__restrict__ ovl = nullptr) {
  __shared__ double sh[2 * 9 * 32];
  __shared__ int last;
  pdl_begin();
  const int n = blockIdx.x / p.hyd_pcl;
  const int rank = blockIdx.x % p.hyd_pcl;
  const int stride = p.hyd_pcl * blockDim.x;
  const int first = rank * blockDim.x + threadIdx.x;
  DPart &a = parts[n];
  const double xp[3] = {a.x[0], a.x[1], a.x[2]};
  const double vp[3] = {a.v[0], a.v[1], a.v[2]};
  const double wp[3] = {a.omega[0], a.omega[1], a.omega[2]};
  const StencilBase b = stencil_base(xp, p);
  const size_t npts = (size_t)p.N[0] * p.N[1] * p.N[2];
  // each thread adds only a few terms: plain sums here, compensated sums in
  // the block and cross-block reductions
  double a9[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) a9[i] = 0.0;
  float f6[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if constexpr (sizeof(R) == 4) {
    // mixed path: the point's offset from the sphere centre, its distance,
    // phi and the momentum-exchange terms in float (the offset is an integer
    // cell shift minus the centre's sub-cell residue, so it is exact to one
    // float ulp); the per-thread and per-warp sums in float, every wider sum
    // in double (compensated)
    const float dxf = (float)p.DX, rpf = (float)(p.RADIUS + p.HXI), rmf = (float)(p.RADIUS - p.HXI);
    const float resf[3] = {(float)b.res[0], (float)b.res[1], (float)b.res[2]};
    const float vpf[3] = {(float)vp[0], (float)vp[1], (float)vp[2]};
    const float wpf[3] = {(float)wp[0], (float)wp[1], (float)wp[2]};
    // GB of the thread's points at a time: their geometry and phi first,
    // then all their velocity loads, then the sums (in the same point
    // order), so that the scattered loads of a batch are in flight together
    constexpr int GB = 4;
    for (int m0 = first; m0 < p.S; m0 += GB * stride) {
      float ph[GB], r[GB][3];
      size_t im[GB];
#pragma unroll
      for (int k = 0; k < GB; ++k) {
        const int m = m0 + k * stride;
        ph[k] = 0.f;
        im[k] = 0;
        if (m < p.S) {
          const int *cell = cells + 3 * m;
          int rm[3];
#pragma unroll
          for (int d = 0; d < 3; ++d) rm[d] = (b.xi[d] + cell[d] + p.N[d]) & (p.N[d] - 1);
          // phi is exactly zero beyond a + xi/2 (about half of the Sekibun
          // points): those terms add zeros, so their loads are skipped
          ph[k] = prof_phi_f(offset_f(cell, resf, dxf, r[k]), rpf, rmf, dxf);
          im[k] = ((size_t)rm[0] * p.N[1] + rm[1]) * p.N[2] + rm[2];
        }
      }
      float ug[GB][3];
#pragma unroll
      for (int k = 0; k < GB; ++k)
        if (ph[k] != 0.f)
#pragma unroll
          for (int d = 0; d < 3; ++d) ug[k][d] = (float)__ldg(u + d * npts + im[k]);
#pragma unroll
      for (int k = 0; k < GB; ++k) {
        if (ph[k] == 0.f) continue;
        float vr[3] = {0.f, 0.f, 0.f};
        if (p.rotation) {
          vr[0] = wpf[1] * r[k][2] - wpf[2] * r[k][1];
          vr[1] = wpf[2] * r[k][0] - wpf[0] * r[k][2];
          vr[2] = wpf[0] * r[k][1] - wpf[1] * r[k][0];
        }
        float fp[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          fp[d] = ((vpf[d] + vr[d]) - ug[k][d]) * ph[k];
          f6[d] += fp[d];
        }
        f6[3] += r[k][1] * fp[2] - r[k][2] * fp[1];
        f6[4] += r[k][2] * fp[0] - r[k][0] * fp[2];
        f6[5] += r[k][0] * fp[1] - r[k][1] * fp[0];
      }
    }
  } else
  for (int m = first; m < p.S; m += stride) {
    int rm[3];
    double r[3], dist;
    stencil_point(b, cells + 3 * m, xp, p, rm, r, dist);
    const double ph = (double)prof_phi<R>(dist, p);
    if (ph == 0.0) continue;  // a zero term: skip its loads
    const size_t im = ((size_t)rm[0] * p.N[1] + rm[1]) * p.N[2] + rm[2];
    const double ug[3] = {(double)__ldg(u + im), (double)__ldg(u + npts + im), (double)__ldg(u + 2 * npts + im)};
    double vr[3] = {0.0, 0.0, 0.0};
    if (p.rotation) {
      vr[0] = wp[1] * r[2] - wp[2] * r[1];
      vr[1] = wp[2] * r[0] - wp[0] * r[2];
      vr[2] = wp[0] * r[1] - wp[1] * r[0];
    }
    double fp[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      fp[d] = ((vp[d] + vr[d]) - ug[d]) * ph;
      a9[d] += fp[d];
    }
    a9[3] += r[1] * fp[2] - r[2] * fp[1];
    a9[4] += r[2] * fp[0] - r[0] * fp[2];
    a9[5] += r[0] * fp[1] - r[1] * fp[0];
  }
  if (p.lj_on) {
    int mc[3];
    for (int d = 0; d < 3; ++d) mc[d] = (int)(xp[d] / p.lc_r);
    // candidates: the neighbour list (every pair within the LJ cutoff is on
    // it) or all particles
    const int *lst = p.nbl ? p.nbl + (size_t)n * (NBL_MAX + 1) : nullptr;
    const int ncand = lst ? lst[0] : p.Np;
    for (int t = first; t < ncand; t += stride) {
      const int j = lst ? lst[1 + t] : t;
      if (j == n) continue;
      const DPart &o = parts[j];
      int mult = 1;
      double x12[3], r2 = 0.0;
      for (int d = 0; d < 3; ++d) {
        // times the cell-list scan (md_force.cxx:72-121) meets this pair
        const int cj = (int)(o.x[d] / p.lc_r);
        int cnt = 0;
        for (int off = -1; off <= 1; ++off) {
          int c = mc[d] + off;
          if (c < 0) c = p.lc[d] - 1;
          if (c > p.lc[d] - 1) c = 0;
          cnt += (c == cj);
        }
        mult *= cnt;
        x12[d] = o.x[d] - xp[d];
        x12[d] -= nint_d(x12[d] * p.invL[d]) * p.L[d];
        r2 += x12[d] * x12[d];
      }
      const double rij = sqrt(r2);
      if (mult > 0 && rij < p.lj_cut) {
        // Lennard_Jones_f (interaction.h:156-181)
        const double s = p.lj_dia / rij;
        double dmy = (s * s) * (s * s) * (s * s);
        if (p.lj_powers >= 1) dmy = dmy * dmy;
        if (p.lj_powers >= 2) dmy = dmy * (s * s) * (s * s) * (s * s);
        const double f = p.lj_coeff / (rij * rij) * (2.0 * dmy * dmy - dmy);
        for (int d = 0; d < 3; ++d) a9[6 + d] += (double)mult * (f * -x12[d]);
      }
    }
  }
  if (ovl && p.hyd_pcl == 1 && !p.nbl) {
    // the overlap candidates of this particle for the scatter that follows
    // (centre distance below 2 (RADIUS + HXI)), as a bit per particle: one
    // word per 32 candidates, written by the warp that tested them
    const double lim = 2.0 * (p.RADIUS + p.HXI), lim2 = lim * lim;
    for (int base = 0; base < p.Np; base += blockDim.x) {
      const int j = base + threadIdx.x;
      bool near = false;
      if (j < p.Np && j != n) {
        double s2 = 0.0;
        for (int d = 0; d < 3; ++d) {
          double dd = parts[j].x[d] - xp[d];
          dd -= nint_d(dd * p.invL[d]) * p.L[d];
          s2 += dd * dd;
        }
        near = s2 < lim2;
      }
      const unsigned bal = __ballot_sync(0xffffffffu, near);
      if ((threadIdx.x & 31) == 0 && base + (threadIdx.x & ~31) < p.Np) ovl[(size_t)n * 32 + (j >> 5)] = bal;
    }
  }
  KSum acc[9];
  if constexpr (sizeof(R) == 4) {
    // each thread's few hydro terms are summed in float; from the warp
    // level up every sum is double (warp sums plain, the sum over the warps
    // compensated)
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int i = 0; i < 6; ++i) a9[i] = (double)f6[i];
#pragma unroll
    for (int i = 0; i < 9; ++i)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) a9[i] += __shfl_xor_sync(0xffffffffu, a9[i], o);
    if (lane == 0)
#pragma unroll
      for (int i = 0; i < 9; ++i) sh[(2 * i) * 32 + wid] = a9[i];
    __syncthreads();
    if (threadIdx.x < 9) {
      const int i = threadIdx.x;
      KSum k{0.0, 0.0};
      for (int w = 0; w < nw; ++w) k.add(sh[(2 * i) * 32 + w]);
      sh[(2 * i) * 32] = k.s;
      sh[(2 * i + 1) * 32] = k.c;
    }
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
      for (int i = 0; i < 9; ++i) acc[i] = {sh[(2 * i) * 32], sh[(2 * i + 1) * 32]};
  } else {
#pragma unroll
    for (int i = 0; i < 9; ++i) acc[i] = {a9[i], 0.0};
    block_reduce<9>(acc, sh);
  }
  KSum tot[9];
  if (p.hyd_pcl == 1) {
    // one block per particle: its sums are the particle's
    if (threadIdx.x != 0) return;
    for (int i = 0; i < 9; ++i) tot[i] = acc[i];
  } else {
    if (threadIdx.x == 0) {
      double *pp = partial + ((size_t)n * p.hyd_pcl + rank) * 18;
      for (int i = 0; i < 9; ++i) {
        pp[2 * i] = acc[i].s;
        pp[2 * i + 1] = acc[i].c;
      }
      __threadfence();
      last = (atomicAdd(arrivals + n, 1) == p.hyd_pcl - 1);
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    arrivals[n] = 0;
    for (int i = 0; i < 9; ++i) tot[i] = {0.0, 0.0};
    for (int q = 0; q < p.hyd_pcl; ++q) {
      const volatile double *pq = partial + ((size_t)n * p.hyd_pcl + q) * 18;
      for (int i = 0; i < 9; ++i) {
        tot[i].add(pq[2 * i]);
        tot[i].c += pq[2 * i + 1];
      }
    }
  }
  double fh[3], th[3], fr[3];
  for (int d = 0; d < 3; ++d) {
    fh[d] = p.fh_coef * (tot[d].s + tot[d].c);
    th[d] = p.rotation ? p.fh_coef * (tot[3 + d].s + tot[3 + d].c) : 0.0;
    fr[d] = tot[6 + d].s + tot[6 + d].c;
  }
  fr[p.gdir] -= p.grav;
  if (nc_corr) {
    // learned near-contact correction of this step's hydrodynamic force/torque
    for (int d = 0; d < 3; ++d) {
      fh[d] += nc_corr[6 * (size_t)n + d];
      if (p.rotation) th[d] += nc_corr[6 * (size_t)n + 3 + d];
      nc_corr[6 * (size_t)n + d] = 0.0;
      nc_corr[6 * (size_t)n + 3 + d] = 0.0;
    }
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

// ---------------------------------------------------------------------------
// Deterministic phi / phi*u_p scatter.
//
// Make_phi_u_primitive (make_phi.cxx:221-277) adds each particle's profile
// phi_i and phi_i (v_i + omega_i x r) into the fields particle by particle,
// so where the supports of several particles overlap a point receives its
// terms in increasing particle index.  Here every point is written by ONE
// thread, the one of the lowest-index particle whose profile is non-zero
// there (its "owner"): it adds its own term and then those of the
// higher-index overlapping particles in index order, and stores the sum.
// No atomics, no dependence on scheduling: graph and eager runs, and every
// run, give the same bits, and the FP64 sums are the reference's own order.
// Every other particle skips the point.  The candidates are the particles
// whose centre is within 2 (RADIUS + HXI) of this one (minimum image): a
// point can only be inside two supports if they overlap.  They come from
// the step's neighbour lists for large particle counts, else from a scan of
// all particles by every block.
constexpr int NB_MAX = 64;  // overlapping neighbours per particle (more: KAPSEL_ERANGE)

struct NbShared {
  double x[3], v[3], w[3], res[3];
  float resf[3];
  int xi[3];
  int idx;
};

// The overlap candidates of particle n in increasing index order, into nb
// (at most NB_MAX); returns their count.  All threads of the block call it.
__device__ void fill_candidate(const PPar &p, const DPart *__restrict__ parts, int j, NbShared &e) {
  const DPart &o = parts[j];
  const StencilBase sb = stencil_base(o.x, p);
  for (int d = 0; d < 3; ++d) {
    e.x[d] = o.x[d];
    e.v[d] = o.v[d];
    e.w[d] = o.omega[d];
    e.res[d] = sb.res[d];
    e.resf[d] = (float)sb.res[d];
    e.xi[d] = sb.xi[d];
  }
  e.idx = j;
}

// The same list from the bit words the gather kernel left (ovl, at most
// 1024 particles): warp 0 orders the set bits with a prefix sum.
__device__ int overlap_from_bits(const PPar &p, const DPart *__restrict__ parts, int n, const unsigned *ovl,
                                 NbShared *nb, int *__restrict__ status) {
  __shared__ int total_b;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const unsigned word = lane * 32 < p.Np ? ovl[(size_t)n * 32 + lane] : 0u;
    const int c = __popc(word);
    int incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    int pos = incl - c;
    for (unsigned w = word; w; w &= w - 1, ++pos)
      if (pos < NB_MAX) fill_candidate(p, parts, lane * 32 + __ffs(w) - 1, nb[pos]);
    if (lane == 31) total_b = incl;
  }
  __syncthreads();
  if (total_b > NB_MAX) {
    if (threadIdx.x == 0) atomicExch(status, -6);
    return NB_MAX;
  }
  return total_b;
}

__device__ int overlap_candidates(const PPar &p, const DPart *__restrict__ parts, int n, NbShared *nb,
                                  int *__restrict__ status) {
  __shared__ int wcount[32];
  __shared__ int total;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const double lim = 2.0 * (p.RADIUS + p.HXI), lim2 = lim * lim;
  const double *xn = parts[n].x;
  // the neighbour list when there is one (in index order), else all particles
  const int *lst = p.nbl ? p.nbl + (size_t)n * (NBL_MAX + 1) : nullptr;
  const int ncand = lst ? lst[0] : p.Np;
  if (threadIdx.x == 0) total = 0;
  __syncthreads();
  for (int base = 0; base < ncand; base += blockDim.x) {
    const int t = base + threadIdx.x;
    const int j = t < ncand ? (lst ? lst[1 + t] : t) : -1;
    bool near = false;
    if (j >= 0 && j != n) {
      double s = 0.0;
      for (int d = 0; d < 3; ++d) {
        double dd = parts[j].x[d] - xn[d];
        dd -= nint_d(dd * p.invL[d]) * p.L[d];
        s += dd * dd;
      }
      near = s < lim2;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, near);
    if (lane == 0) wcount[warp] = __popc(bal);
    __syncthreads();
    int pos = total + __popc(bal & ((1u << lane) - 1u));
    for (int w = 0; w < warp; ++w) pos += wcount[w];
    if (near && pos < NB_MAX) fill_candidate(p, parts, j, nb[pos]);
    __syncthreads();
    if (threadIdx.x == 0)
      for (int w = 0; w < nw; ++w) total += wcount[w];
    __syncthreads();
  }
  if (total > NB_MAX) {
    if (threadIdx.x == 0) atomicExch(status, -6);
    return NB_MAX;
  }
  return total;
}

// Sekibun offset of grid point rm from the stencil base of a sphere (the
// cell index in [-N/2, N/2) that the sphere's own stencil reaches rm with).
__device__ __forceinline__ void offset_from_base(const int rm[3], const int xi[3], const PPar &p, int cell[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int c = (rm[d] - xi[d]) & (p.N[d] - 1);
    cell[d] = c >= p.N[d] / 2 ? c - p.N[d] : c;
  }
}

template <typename R>
__global__ void __launch_bounds__(256) k_particles_scatter(PPar p, const DPart *__restrict__ parts,
                                                           const int *__restrict__ cells, R *__restrict__ phiup,
                                                           int *__restrict__ status,
                                                           const unsigned *__restrict__ ovl = nullptr) {
  __shared__ NbShared nb[NB_MAX];
  pdl_begin();
  const int n = blockIdx.x / PCL;
  const int stride = PCL * blockDim.x;
  const int first = (blockIdx.x % PCL) * blockDim.x + threadIdx.x;
  const int nnb = ovl ? overlap_from_bits(p, parts, n, ovl, nb, status) : overlap_candidates(p, parts, n, nb, status);
  int nlow = 0;  // candidates with a lower index come first
  while (nlow < nnb && nb[nlow].idx < n) ++nlow;
  const DPart &a = parts[n];
  const double xp[3] = {a.x[0], a.x[1], a.x[2]};
  const double vp[3] = {a.v[0], a.v[1], a.v[2]};
  const double wp[3] = {a.omega[0], a.omega[1], a.omega[2]};
  const StencilBase b = stencil_base(xp, p);
  const size_t npts = (size_t)p.N[0] * p.N[1] * p.N[2];
  const double rsup = p.RADIUS + p.HXI;
  if constexpr (sizeof(R) == 4) {
    // mixed path: offset, distance, phi and phi*(v + omega x r) in float
    const float dxf = (float)p.DX, rpf = (float)(p.RADIUS + p.HXI), rmf = (float)(p.RADIUS - p.HXI);
    const float resf[3] = {(float)b.res[0], (float)b.res[1], (float)b.res[2]};
    for (int m = first; m < p.S; m += stride) {
      const int *cell = cells + 3 * m;
      int rm[3];
      float r[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) rm[d] = (b.xi[d] + cell[d] + p.N[d]) & (p.N[d] - 1);
      const float ph = prof_phi_f(offset_f(cell, resf, dxf, r), rpf, rmf, dxf);
      if (ph == 0.f) continue;
      bool own = true;
      for (int k = 0; k < nlow && own; ++k) {
        int cj[3];
        float rj[3];
        offset_from_base(rm, nb[k].xi, p, cj);
        const float dj = offset_f(cj, nb[k].resf, dxf, rj);
        if (dj < rpf && prof_phi_f(dj, rpf, rmf, dxf) != 0.f) own = false;
      }
      if (!own) continue;
      float acc = ph, up[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        float vr = 0.f;
        if (p.rotation) {
          const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
          vr = (float)wp[d1] * r[d2] - (float)wp[d2] * r[d1];
        }
        up[d] = ((float)vp[d] + vr) * ph;
      }
      for (int k = nlow; k < nnb; ++k) {
        int cj[3];
        float rj[3];
        offset_from_base(rm, nb[k].xi, p, cj);
        const float dj = offset_f(cj, nb[k].resf, dxf, rj);
        if (!(dj < rpf)) continue;
        const float phj = prof_phi_f(dj, rpf, rmf, dxf);
        if (phj == 0.f) continue;
        acc += phj;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          float vr = 0.f;
          if (p.rotation) {
            const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
            vr = (float)nb[k].w[d1] * rj[d2] - (float)nb[k].w[d2] * rj[d1];
          }
          up[d] += ((float)nb[k].v[d] + vr) * phj;
        }
      }
      const size_t im = ((size_t)rm[0] * p.N[1] + rm[1]) * p.N[2] + rm[2];
      reinterpret_cast<float *>(phiup)[im] = acc;
#pragma unroll
      for (int d = 0; d < 3; ++d) reinterpret_cast<float *>(phiup)[(1 + d) * npts + im] = up[d];
    }
  } else
  for (int m = first; m < p.S; m += stride) {
    int rm[3];
    double r[3], dist;
    stencil_point(b, cells + 3 * m, xp, p, rm, r, dist);
    const double ph = (double)prof_phi<R>(dist, p);
    if (ph == 0.0) continue;
    bool own = true;
    for (int k = 0; k < nlow && own; ++k) {
      const double dj = point_dist(nb[k].x, rm, p);
      if (dj < rsup && (double)prof_phi<R>(dj, p) != 0.0) own = false;
    }
    if (!own) continue;
    double acc = ph, up[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      double vr = 0.0;
      if (p.rotation) {
        const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
        vr = wp[d1] * r[d2] - wp[d2] * r[d1];
      }
      up[d] = (vp[d] + vr) * ph;
    }
    for (int k = nlow; k < nnb; ++k) {
      const double dj = point_dist(nb[k].x, rm, p);
      if (!(dj < rsup)) continue;
      const double phj = (double)prof_phi<R>(dj, p);
      if (phj == 0.0) continue;
      int cj[3];
      double rj[3];
      offset_from_base(rm, nb[k].xi, p, cj);
#pragma unroll
      for (int d = 0; d < 3; ++d) rj[d] = __dsub_rn(__dmul_rn((double)cj[d], p.DX), nb[k].res[d]);
      acc += phj;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double vr = 0.0;
        if (p.rotation) {
          const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
          vr = nb[k].w[d1] * rj[d2] - nb[k].w[d2] * rj[d1];
        }
        up[d] += (nb[k].v[d] + vr) * phj;
      }
    }
    const size_t im = ((size_t)rm[0] * p.N[1] + rm[1]) * p.N[2] + rm[2];
    phiup[im] = (R)acc;
#pragma unroll
    for (int d = 0; d < 3; ++d) phiup[(1 + d) * npts + im] = (R)up[d];
  }
}

// The phi > 1 clamp of Make_phi_u_primitive (make_phi.cxx:278-297) as a
// separate pass, for the routine-level entry point.
template <typename R>
__global__ void k_clamp_phi(size_t npts, R *__restrict__ phiup) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < npts; i += (size_t)gridDim.x * blockDim.x) {
    const R ph = phiup[i];
    if (ph > R(1)) {
      const R inv = R(1) / ph;
      for (int d = 1; d <= 3; ++d) phiup[d * npts + i] *= inv;
      phiup[i] = R(1);
    }
  }
}

}  // namespace kapsel
