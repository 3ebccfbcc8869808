// kapsel_gpu.cu -- host side of the B200 SPM step: context, buffers, launch
// sequence, CUDA graph replay and the C ABI declared in include/kapsel_gpu.h.
//
// One SPM step (Time_evolution_hydro, sp_3d_ns.cxx:61-212, Navier_Stokes
// branch) is 12 launches (13 kernels; 8 runs in extra blocks of 7), each
// after the first launched with programmatic stream serialization:
//   1 k_x_zeta_to_u        truncated zeta -> u_k -> inverse x
//   2 k_y_pass<inv>        inverse y (3 comps)
//   3 k_z_products         inverse z, 5 products, forward z
//   4 k_y_pass<fwd>        forward y (5 comps)
//   5 k_x_advect_update    forward x, Omega, slaved Euler, FIX_CELL, u*_k, inverse x
//   6 k_y_pass<inv>        inverse y (3 comps)
//   7 k_z_c2r              inverse z -> u* (real)
//   8 (k_z_c2r blocks)     AB2 / Euler positions and orientations
//   9 k_particles_hydro_velocity  hydro force+torque gather, LJ, gravity, velocity, thermostat
//  10 k_particles_scatter  phi, phi*u_p
//  11 k_z_force            clamp, f = up - phi u*, forward z, clear phi/up
//  12 k_y_pass<fwd>        forward y (3 comps)
//  13 k_x_force_to_zeta    forward x, solenoidal projection, zeta += zeta(f), uk_dc += f(0)
// The 20 3D FFTs of the reference become 14 pruned ones because
// U2zeta_k(u* + f_sol) = trunc(zeta) + U_k2zeta_k(f_sol) (linearity).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <sys/stat.h>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/kapsel_gpu.h"
#include "cell_kernels.cuh"
#include "electrolyte_kernels.cuh"
#include "nearcontact_kernels.cuh"
#include "obl_kernels.cuh"
#include "particle_kernels.cuh"
#include "spectral_kernels.cuh"
#include "yz_kernels.cuh"
#include "zwarp_kernels.cuh"

using namespace kapsel;

namespace {

// ---------------------------------------------------------------------------
// MT19937 (Matsumoto & Nishimura 1998) with the init_genrand seeding, the
// generator behind the reference thermostat (mt19937ar.c, seeded with 0 by
// MT_seed at sp_3d_ns.cxx:477).  Written from the published algorithm.
class MT19937 {
 public:
  explicit MT19937(uint32_t s) { seed(s); }
  void seed(uint32_t s) {
    mt_[0] = s;
    for (int i = 1; i < 624; ++i) mt_[i] = 1812433253u * (mt_[i - 1] ^ (mt_[i - 1] >> 30)) + (uint32_t)i;
    idx_ = 624;
  }
  uint32_t next() {
    if (idx_ >= 624) twist();
    uint32_t y = mt_[idx_++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
  }
  // genrand_real3: (y + 0.5) / 2^32, in (0,1)
  double real3() { return ((double)next() + 0.5) * (1.0 / 4294967296.0); }
  // Gauss2 (fluct.h:48-60): polar Box-Muller pair
  void gauss2(double *out) {
    double x1, x2, rsq;
    do {
      x1 = 2. * real3() - 1.;
      x2 = 2. * real3() - 1.;
      rsq = x1 * x1 + x2 * x2;
    } while (rsq >= 1.0 || rsq == 0.0);
    const double f = std::sqrt(-2. * std::log(rsq) / rsq);
    out[0] = f * x1;
    out[1] = f * x2;
  }

 private:
  void twist() {
    for (int i = 0; i < 624; ++i) {
      const uint32_t y = (mt_[i] & 0x80000000u) | (mt_[(i + 1) % 624] & 0x7fffffffu);
      mt_[i] = mt_[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    idx_ = 0;
  }
  uint32_t mt_[624];
  int idx_;
};

int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}

#define KCHECK(call)                                         \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) {                                 \
      fprintf(stderr, "kapsel_gpu: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
      return KAPSEL_ECUDA;                                   \
    }                                                        \
  } while (0)

// Lets `kern` take all the dynamic shared memory a block may opt in to
// (`need` bytes must fit).  The limit is one value per kernel function,
// shared by every context of the process: set to one box shape's size it
// would refuse the same kernel's launches for a larger shape created
// earlier.  Occupancy follows the shared memory a launch asks for, not
// this limit.
template <typename K>
cudaError_t allow_smem(K kern, size_t need) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaFuncAttributes fa;
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, kern);
  if (e != cudaSuccess) return e;
  const size_t lim = (size_t)optin > fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
  if (need > lim) return cudaErrorInvalidValue;
  return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lim);
}

// Sekibun stencil offsets (Particle_domain, profile.cxx:25-74): points with
// |(i,j,k) DX| < RADIUS + HXI + 1.7321 DX, scanned i, j, k from -nh to nh.
std::vector<int> sekibun(double A, double A_XI, double DX) {
  const double radius = A * DX, hxi = 0.5 * A_XI * DX;
  const int nh = (int)A + (int)A_XI + 2;
  const double max_r = radius + hxi + 1.7321 * DX;
  std::vector<int> out;
  for (int i = -nh; i <= nh; ++i)
    for (int j = -nh; j <= nh; ++j)
      for (int k = -nh; k <= nh; ++k) {
        const double x = i * DX, y = j * DX, z = k * DX;
        if (std::sqrt(x * x + y * y + z * z) < max_r) {
          out.push_back(i);
          out.push_back(j);
          out.push_back(k);
        }
      }
  return out;
}

template <typename R, bool INVERSE>
__global__ void k_col_pass(Geo g, const Cx<R> *twn, int logn, int n, const Cx<R> *in, Cx<R> *out,
                           long long line_stride, long long elem_stride, int nlines, int lines_per_plane,
                           long long plane_stride);
template <typename R>
__global__ void k_z_c2r_full(Geo g, Twiddles<R> tw, const Cx<R> *__restrict__ in, R *__restrict__ out, double scale);

// Kernel launch on `st`, optionally with programmatic stream serialization
// (the kernel may start while its predecessor drains; it waits in pdl_begin).
template <typename... KArgs, typename... Args>
void launch_k(bool pdl, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
              Args... args) {
  if (!pdl) {
    kern<<<grid, block, smem, st>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, args...);
}

// ---------------------------------------------------------------------------
struct BoxBase {
  virtual ~BoxBase() {}
  kapsel_params prm;
  Geo g;
  PPar pp;
  int Np = 0, S = 0;
  cudaStream_t stream = nullptr;
  DPart *parts = nullptr;
  int *cells = nullptr;
  double *uk_dc = nullptr;
  int *status = nullptr;
  double *partial_p = nullptr;  // [Np][PCL][18] partial force sums
  int *arrivals = nullptr;    // [Np] blocks done per particle (0 between launches)
  double *noise_dev[2] = {nullptr, nullptr};
  double *noise_host[2] = {nullptr, nullptr};
  cudaEvent_t noise_ev[2] = {nullptr, nullptr};
  std::unique_ptr<MT19937> mt;
  int ts = 0;
  double time = 0.0;
  bool initialised = false;
  bool particles_set = false;
  // bufA holds u_k of the current zeta / uk_dc, left there by the fused last
  // launch of a Navier-Stokes step; the next step then skips its first launch
  bool u_spec_ready = false;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  // learned near-contact correction (off unless a network is attached)
  const kapsel_nc *nc = nullptr;
  float *nc_feat = nullptr, *nc_frames = nullptr;
  int2 *nc_pairs = nullptr;
  int *nc_count = nullptr;
  double *nc_corr = nullptr;
  int nc_cap = 0;

  // the pair search and the network, between the position update and the
  // hydrodynamic gather (both launched without programmatic serialization)
  void launch_nearcontact();

  // per-step cell and neighbour lists (cell_kernels.cuh); pp.nbl points at
  // the lists while they are on
  bool cl_on = false;
  // overlap candidates of each particle as bit words ([Np][32]), written by
  // the gather for the scatter of the same step (at most 1024 particles,
  // without neighbour lists); null otherwise
  unsigned *ovl = nullptr;
  CellPar clp{};
  int *cl_count = nullptr, *cl_start = nullptr, *cl_cursor = nullptr, *cl_list = nullptr, *cl_cellof = nullptr;
  int *nbl = nullptr;
  double cl_rlist = 0.0;
  // (re)build the cell grid for a neighbour range of at least rlist; the
  // captured step graphs hold the old launch parameters and are dropped
  int setup_cells(double rlist) {
    if (Np == 0) return 0;
    if (cl_on && rlist <= cl_rlist) return 0;
    for (int s = 0; s < 2; ++s)
      if (graph[s]) {
        cudaGraphExecDestroy(graph[s]);
        graph[s] = nullptr;
      }
    cudaFree(cl_count);
    cudaFree(cl_start);
    cudaFree(cl_cursor);
    cl_rlist = rlist;
    for (int d = 0; d < 3; ++d) {
      clp.lc[d] = std::max(1, (int)std::floor(pp.L[d] / rlist));
      clp.inv_cl[d] = clp.lc[d] / pp.L[d];
    }
    clp.ncell = clp.lc[0] * clp.lc[1] * clp.lc[2];
    clp.r2list = rlist * rlist;
    KCHECK(cudaMalloc(&cl_count, sizeof(int) * clp.ncell));
    KCHECK(cudaMemset(cl_count, 0, sizeof(int) * clp.ncell));
    KCHECK(cudaMalloc(&cl_start, sizeof(int) * (clp.ncell + 1)));
    KCHECK(cudaMalloc(&cl_cursor, sizeof(int) * clp.ncell));
    if (!cl_list) {
      KCHECK(cudaMalloc(&cl_list, sizeof(int) * Np));
      KCHECK(cudaMalloc(&cl_cellof, sizeof(int) * Np));
      KCHECK(cudaMalloc(&nbl, sizeof(int) * (size_t)Np * (NBL_MAX + 1)));
      KCHECK(cudaMemset(nbl, 0, sizeof(int) * (size_t)Np * (NBL_MAX + 1)));
    }
    pp.nbl = nbl;
    cl_on = true;
    return 0;
  }
  // the lists of the current positions (five launches), before any kernel
  // that reads them
  void launch_cells() {
    if (!cl_on || Np == 0) return;
    k_cell_count<<<(Np + 255) / 256, 256, 0, stream>>>(pp, clp, parts, cl_cellof, cl_count);
    k_cell_scan<<<1, 1024, 0, stream>>>(clp, cl_count, cl_start, cl_cursor);
    k_cell_fill<<<(Np + 255) / 256, 256, 0, stream>>>(pp, cl_cellof, cl_cursor, cl_list);
    k_cell_sort<<<(clp.ncell + 255) / 256, 256, 0, stream>>>(clp, cl_start, cl_list);
    k_neighbor_lists<<<(Np + NBL_WARPS - 1) / NBL_WARPS, NBL_WARPS * 32, 0, stream>>>(pp, clp, parts, cl_start,
                                                                                   cl_list, nbl, status);
  }
  void free_cells() {
    cudaFree(cl_count);
    cudaFree(cl_start);
    cudaFree(cl_cursor);
    cudaFree(cl_list);
    cudaFree(cl_cellof);
    cudaFree(nbl);
    cudaFree(ovl);
  }

  virtual int alloc() = 0;
  // pass variants of the batch autotuner: z passes warp-level (0) or
  // block-level (1); y pass warp-level (0), block-level with the wide (1) or
  // the narrow (2) kz tile.  time_variant runs `reps` steps of this box's
  // workload with a variant on a copy of its state and restores the state.
  virtual float time_variant(int zmode, int ymode, int reps) = 0;
  virtual void set_variant(int zmode, int ymode) = 0;
  virtual bool variant_ok(int zmode, int ymode) const = 0;
  // radix split of the block-level x transforms: 0 the default, 1 the other
  // factorisation of NX (fft2_n1_sel); time_variant times the current one
  int xsplit = 0;
  virtual bool xsplit_ok(int xs) const = 0;
  virtual void set_xsplit(int xs) = 0;
  // the step runs the fused y/z plane kernels (k_yzw_c2r, k_zyw_force)
  virtual bool fused_yz() const { return false; }
  virtual int alloc_el() = 0;
  virtual int alloc_obl() = 0;
  virtual int oblique_state(double *out) = 0;
  virtual int set_oblique_state(double deg, double srate) = 0;
  virtual int init_el() = 0;
  virtual int conc_to_host(double *c) = 0;
  virtual int conc_from_host(const double *c) = 0;
  virtual int total_solute_from_host(const double *t) = 0;  // Total_solute[2]
  virtual void launch_step(const double *noise, int euler, cudaEvent_t *ev = nullptr) = 0;
  virtual void launch_init() = 0;
  // launch the first x pass if bufA does not hold u_k (before a step or a
  // graph replay); true when the step will leave u_k in bufA again
  virtual void ensure_u_spec() = 0;
  virtual bool ends_with_u_spec() const = 0;
  virtual int velocity_to_host(double *u) = 0;
  virtual int zeta_to_host(double *z) = 0;
  virtual int zeta_from_host(const double *z) = 0;
  virtual int fft_fwd_host(double *a) = 0;
  virtual int fft_inv_host(double *a) = 0;
  virtual int solenoidal_host(double *u0, double *u1, double *u2) = 0;
  virtual int phi_up_host(double *phi, double *up0, double *up1, double *up2) = 0;
  virtual int phi_only_host(double *phi) = 0;  // Make_phi_particle: no clamp
  virtual int fhydro_host(const double *u0, const double *u1, const double *u2, double *f, double *t) = 0;
  // NS_solver_slavedEuler on a host zeta (Ooura layout): retained modes updated in place
  virtual int slaved_euler_host(double *z, const double *ukdc) = 0;
  // the Electrolyte routines NSsolute_solver_Euler, Rescale_solute and
  // Make_Coulomb_force_x_on_fluid on host arrays (Ooura layout)
  virtual int ns_solute_host(double *z, const double *ukdc, double *c) = 0;
  virtual int rescale_solute_host(const double *total, double *c, double *factors) = 0;
  virtual int coulomb_force_host(const double *c, double *f0, double *f1, double *f2) = 0;
  virtual int el_snapshot_host(double *phi, double *surf, double *conc, double *pot) = 0;
  virtual void free_all() = 0;

  int fill_noise(int slot) {
    // the normals one call of Add_random_force_thermostat consumes, in order
    // (fluct.cxx:21-35: Gauss2 x3 per particle)
    if (!pp.thermostat) return 0;
    KCHECK(cudaEventSynchronize(noise_ev[slot]));
    double *h = noise_host[slot];
    for (int n = 0; n < Np; ++n) {
      mt->gauss2(h + 6 * n);
      mt->gauss2(h + 6 * n + 2);
      mt->gauss2(h + 6 * n + 4);
    }
    KCHECK(cudaMemcpyAsync(noise_dev[slot], h, sizeof(double) * 6 * Np, cudaMemcpyHostToDevice, stream));
    KCHECK(cudaEventRecord(noise_ev[slot], stream));
    return 0;
  }
  // The normals of step ts are drawn while the GPU runs step ts-1
  // (prefill_noise right after its launch); take_noise uses them when they
  // are there.  The draw order, and so the stream, is unchanged.
  int noise_pre_ts[2] = {-1, -1};
  int take_noise(int slot) {
    if (noise_pre_ts[slot] == ts) {
      noise_pre_ts[slot] = -1;
      return 0;
    }
    return fill_noise(slot);
  }
  int prefill_noise() {
    const int slot = ts & 1;
    if (!pp.thermostat || noise_pre_ts[slot] == ts) return 0;
    const int rc = fill_noise(slot);
    if (!rc) noise_pre_ts[slot] = ts;
    return rc;
  }
  void drop_prefill() { noise_pre_ts[0] = noise_pre_ts[1] = -1; }
  DPart *parts_host = nullptr;  // pinned staging of the particle readout
  int *status_host = nullptr;   // pinned copy of the status word
};

// threads per block of the x passes of the Navier-Stokes step (multiples of
// 32 up to 256); the block-level transforms divide their work over them
#ifndef KAPSEL_XZ_THREADS
#define KAPSEL_XZ_THREADS 256
#endif
#ifndef KAPSEL_XADV_THREADS
#define KAPSEL_XADV_THREADS 256
#endif
#ifndef KAPSEL_XFORCE_THREADS
#define KAPSEL_XFORCE_THREADS 256
#endif
constexpr int kXZThreads = KAPSEL_XZ_THREADS, kXAdvThreads = KAPSEL_XADV_THREADS,
              kXForceThreads = KAPSEL_XFORCE_THREADS;

// warps per block of the fused y/z plane kernels (FP32 fields; 4 measured
// faster than 6 and 8 at 128^3: three 64 KB blocks per SM hold all 384
// planes in one wave)
#ifndef KAPSEL_YZ_NW
#define KAPSEL_YZ_NW 4
#endif

template <typename R>
struct Box : BoxBase {
  Cx<R> *zeta = nullptr;  // [2][KXc][KYc][TS]
  Cx<R> *bufA = nullptr;  // I1-shaped, 5 comps [c][NX][KYc][TS]
  Cx<R> *bufB = nullptr;  // I2-shaped, 5 comps [c][NX][NY][TS]
  R *ustar = nullptr;     // [3][NX][NY][NZ]
  R *phiup = nullptr;     // [4][NX][NY][NZ]
  Cx<R> *twbuf = nullptr;
  Twiddles<R> tw;
  static constexpr int KCX = 4;                         // x-pass kz tile
  static constexpr int KCY = sizeof(R) == 4 ? 32 : 16;  // y-pass kz tile
  size_t smem_xu = 0, smem_xadv = 0, smem_xf = 0, smem_y = 0, smem_zp = 0, smem_zc = 0, smem_zf = 0, smem_zr = 0;

  size_t npts() const { return (size_t)g.NX * g.NY * g.NZ; }

  // x passes with compile-time NX for NX = 32..256 (the runtime-NX kernels otherwise)
  template <int LX, int XS>
  int x_setup_s() {
    KCHECK(allow_smem(k_x_zeta_to_u<R, KCX, LX, XS>, smem_xu));
    KCHECK(allow_smem(k_x_advect_update<R, KCX, 0, LX, XS>, smem_xadv));
    KCHECK(allow_smem(k_x_advect_update<R, KCX, 1, LX, XS>, smem_xadv));
    KCHECK(allow_smem(k_x_force_to_zeta<R, KCX, LX, 0, XS>, smem_xf));
    KCHECK(allow_smem(k_x_force_to_zeta<R, KCX, LX, 1, XS>, smem_xf));
    return 0;
  }
  template <int LX>
  int x_setup() {
    const int rc = x_setup_s<LX, 0>();
    return rc ? rc : x_setup_s<LX, 1>();
  }
  // the x-pass launches, with the radix split of this context (xsplit)
  template <int LX>
  void xz_l(bool pdl, const Cx<R> *z, const double *u, Cx<R> *out) {
    if (xsplit)
      launch_k(pdl, k_x_zeta_to_u<R, KCX, LX, 1>, gx(), dim3(kXZThreads), smem_xu, stream, g, tw, z, u, out);
    else
      launch_k(pdl, k_x_zeta_to_u<R, KCX, LX, 0>, gx(), dim3(kXZThreads), smem_xu, stream, g, tw, z, u, out);
  }
  template <int EU, int LX>
  void xa_l(bool pdl) {
    if (xsplit)
      launch_k(pdl, k_x_advect_update<R, KCX, EU, LX, 1>, gx(), dim3(kXAdvThreads), smem_xadv, stream, g, tw, bufA,
               zeta, uk_dc);
    else
      launch_k(pdl, k_x_advect_update<R, KCX, EU, LX, 0>, gx(), dim3(kXAdvThreads), smem_xadv, stream, g, tw, bufA,
               zeta, uk_dc);
  }
  template <int LX, int NEXTU = 0>
  void xf_l(bool pdl, Cx<R> *in) {
    if (xsplit)
      launch_k(pdl, k_x_force_to_zeta<R, KCX, LX, NEXTU, 1>, gx(), dim3(kXForceThreads), smem_xf, stream, g, tw, in,
               zeta, uk_dc);
    else
      launch_k(pdl, k_x_force_to_zeta<R, KCX, LX, NEXTU, 0>, gx(), dim3(kXForceThreads), smem_xf, stream, g, tw, in,
               zeta, uk_dc);
  }
  void x_zeta(bool pdl, const Cx<R> *z, const double *u, Cx<R> *out) {
    switch (g.NX) {
      case 32: xz_l<5>(pdl, z, u, out); return;
      case 64: xz_l<6>(pdl, z, u, out); return;
      case 128: xz_l<7>(pdl, z, u, out); return;
      case 256: xz_l<8>(pdl, z, u, out); return;
      default: xz_l<0>(pdl, z, u, out);
    }
  }
  template <int EU>
  void x_advect(bool pdl) {
    switch (g.NX) {
      case 32: xa_l<EU, 5>(pdl); return;
      case 64: xa_l<EU, 6>(pdl); return;
      case 128: xa_l<EU, 7>(pdl); return;
      case 256: xa_l<EU, 8>(pdl); return;
      default: xa_l<EU, 0>(pdl);
    }
  }
  void x_force(bool pdl, Cx<R> *in) {
    switch (g.NX) {
      case 32: xf_l<5>(pdl, in); return;
      case 64: xf_l<6>(pdl, in); return;
      case 128: xf_l<7>(pdl, in); return;
      case 256: xf_l<8>(pdl, in); return;
      default: xf_l<0>(pdl, in);
    }
  }
  // the same, followed on each tile by the next step's first x pass (u_k of
  // the updated zeta into bufA)
  void x_force_next(bool pdl) {
    switch (g.NX) {
      case 32: xf_l<5, 1>(pdl, bufA); return;
      case 64: xf_l<6, 1>(pdl, bufA); return;
      case 128: xf_l<7, 1>(pdl, bufA); return;
      case 256: xf_l<8, 1>(pdl, bufA); return;
      default: xf_l<0, 1>(pdl, bufA);
    }
  }

  // warp-level z kernels for NZ = 64, 128, 256 (zw = log2(NZ/2)); 0: block-level
  static constexpr int ZNW = sizeof(R) == 4 ? 8 : 4;  // warps per block
  int zw = 0;
  int zw_grid_p = 0, zw_grid_c = 0, zw_grid_f = 0;
  size_t zw_sm_p = 0, zw_sm_c = 0, zw_sm_f = 0;

  template <int LM>
  int zw_setup() {
    using Z = ZL<LM>;
    const size_t line = sizeof(Cx<R>) * Z::RW * Z::LS * ZNW;
    // FP64: the prefetching products kernel; FP32: four line groups per warp
    zw_sm_p = sizeof(R) == 8 ? sizeof(Cx<R>) * (size_t)ZProd<R, LM>::WARP * ZNW : 4 * line;
    zw_sm_c = line;
    zw_sm_f = 3 * line;
    auto kp = sizeof(R) == 8 ? k_zw_products_pf<R, LM, ZNW> : k_zw_products<R, LM, ZNW>;
    KCHECK(allow_smem(kp, zw_sm_p));
    KCHECK(allow_smem(k_zw_c2r<R, LM, ZNW>, zw_sm_c));
    KCHECK(allow_smem(k_zw_force<R, LM, ZNW>, zw_sm_f));
    int dev = 0, nsm = 0, op = 0, oc = 0, of = 0;
    KCHECK(cudaGetDevice(&dev));
    KCHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    KCHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&op, kp, ZNW * 32, zw_sm_p));
    KCHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&oc, k_zw_c2r<R, LM, ZNW>, ZNW * 32, zw_sm_c));
    KCHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&of, k_zw_force<R, LM, ZNW>, ZNW * 32, zw_sm_f));
    const int groups = g.NX * g.NY / Z::RW;
    zw_grid_p = std::min((groups + ZNW - 1) / ZNW, std::max(op, 1) * nsm);
    zw_grid_c = std::min((3 * groups + ZNW - 1) / ZNW, std::max(oc, 1) * nsm);
    zw_grid_f = std::min((groups + ZNW - 1) / ZNW, std::max(of, 1) * nsm);
    zw = LM;
    yz_ly = 0;
    if (g.KYc < g.NY) {
      if (g.NY == 32) return yz_setup<5, LM>();
      if (g.NY == 64) return yz_setup<6, LM>();
      if (g.NY == 128) return yz_setup<7, LM>();
    }
    return 0;
  }

  // fused y/z plane kernels (pass variant ymode 3): the inverse to u* and the
  // rigidity force as one launch each, for NY = 2^yz_ly (0: not available)
  static constexpr int YZNW = sizeof(R) == 4 ? KAPSEL_YZ_NW : 4;  // warps per block
  int yz_ly = 0;
  size_t yz_sm = 0;
  unsigned *plane_count = nullptr;  // [NX] readers of phi per x plane (k_zyw_force)
  template <int LY, int LM>
  int yz_setup() {
    const size_t sm = YZ<R, LY, LM>::smem(YZNW);
    if (sm > 227 * 1024) return 0;
    KCHECK(allow_smem(k_yzw_c2r<R, LY, LM, false, YZNW>, sm));
    KCHECK(allow_smem(k_zyw_force<R, LY, LM, false, YZNW>, sm));
    yz_sm = sm;
    yz_ly = LY;
    return 0;
  }
  template <int LY, int LM>
  void yz_c2r_l(bool pdl, DPart *pts, int euler) {
    const int posblk = pts ? (Np + YZNW * 32 - 1) / (YZNW * 32) : 0;
    launch_k(pdl, k_yzw_c2r<R, LY, LM, false, YZNW>, dim3(3 * g.NX + posblk), dim3(YZNW * 32), yz_sm, stream, g, tw,
             (const Cx<R> *)bufA, ustar, npts(), g.NZ, 3 * g.NX, pp, pts, euler, status);
  }
  template <int LY, int LM>
  void zy_force_l(bool pdl) {
    launch_k(pdl, k_zyw_force<R, LY, LM, false, YZNW>, dim3(3 * g.NX), dim3(YZNW * 32), yz_sm, stream, g, tw, phiup,
             (const R *)ustar, bufA, plane_count);
  }
  // bufA (x real, ky compact) -> u*, with the position update in extra blocks
  template <int LM>
  void yz_c2r_m(bool pdl, DPart *pts, int euler) {
    if (yz_ly == 5) yz_c2r_l<5, LM>(pdl, pts, euler);
    else if (yz_ly == 6) yz_c2r_l<6, LM>(pdl, pts, euler);
    else yz_c2r_l<7, LM>(pdl, pts, euler);
  }
  void yz_c2r(bool pdl, DPart *pts, int euler) {
    if (zw == 5) yz_c2r_m<5>(pdl, pts, euler);
    else if (zw == 6) yz_c2r_m<6>(pdl, pts, euler);
    else yz_c2r_m<7>(pdl, pts, euler);
  }
  // phi/up, u* -> force spectra in bufA (x real, ky compact)
  template <int LM>
  void zy_force_m(bool pdl) {
    if (yz_ly == 5) zy_force_l<5, LM>(pdl);
    else if (yz_ly == 6) zy_force_l<6, LM>(pdl);
    else zy_force_l<7, LM>(pdl);
  }
  void zy_force(bool pdl) {
    if (zw == 5) zy_force_m<5>(pdl);
    else if (zw == 6) zy_force_m<6>(pdl);
    else zy_force_m<7>(pdl);
  }
  template <int LM>
  void zw_products(bool pdl) {
    launch_k(pdl, sizeof(R) == 8 ? k_zw_products_pf<R, LM, ZNW> : k_zw_products<R, LM, ZNW>, dim3(zw_grid_p),
             dim3(ZNW * 32), zw_sm_p, stream, g, tw, bufB);
  }
  template <int LM>
  void zw_c2r(bool pdl, DPart *pts, int euler) {
    const int posblk = pts ? (Np + ZNW * 32 - 1) / (ZNW * 32) : 0;
    launch_k(pdl, k_zw_c2r<R, LM, ZNW>, dim3(zw_grid_c + posblk), dim3(ZNW * 32), zw_sm_c, stream, g, tw,
             (const Cx<R> *)bufB, ustar, npts(), g.NZ, 3, zw_grid_c, pp, pts, euler, status);
  }
  template <int LM>
  void zw_force(bool pdl) {
    launch_k(pdl, k_zw_force<R, LM, ZNW>, dim3(zw_grid_f), dim3(ZNW * 32), zw_sm_f, stream, g, tw, phiup,
             (const R *)ustar, bufB);
  }
  // dispatch on the compile-time line length
  void zdisp_products(bool pdl) {
    if (zw == 5) zw_products<5>(pdl);
    else if (zw == 6) zw_products<6>(pdl);
    else if (zw == 7) zw_products<7>(pdl);
    else launch_k(pdl, k_z_products<R>, dim3(gz()), dim3(256), smem_zp, stream, g, tw, bufB);
  }
  void zdisp_c2r(bool pdl, DPart *pts, int euler) {
    if (zw == 5) zw_c2r<5>(pdl, pts, euler);
    else if (zw == 6) zw_c2r<6>(pdl, pts, euler);
    else if (zw == 7) zw_c2r<7>(pdl, pts, euler);
    else {
      const int posblk = pts ? (Np + 255) / 256 : 0;
      launch_k(pdl, k_z_c2r<R>, dim3(gz() + posblk, 3), dim3(256), smem_zc, stream, g, tw, (const Cx<R> *)bufB,
               ustar, npts(), g.NZ, pp, pts, euler, status);
    }
  }
  void zdisp_force(bool pdl) {
    if (zw == 5) zw_force<5>(pdl);
    else if (zw == 6) zw_force<6>(pdl);
    else if (zw == 7) zw_force<7>(pdl);
    else launch_k(pdl, k_z_force<R>, dim3(gz()), dim3(256), smem_zf, stream, g, tw, phiup, (const R *)ustar, bufB);
  }

  int alloc() override {
    const size_t nz = (size_t)g.KXc * g.KYc * g.TS;
    const size_t nA = (size_t)g.NX * g.KYc * g.TS;
    const size_t nB = (size_t)g.NX * g.NY * g.TS;
    KCHECK(cudaMalloc(&zeta, sizeof(Cx<R>) * 2 * nz));
    // the Lees-Edwards advection term carries u and the vorticity: 6 spectra
    const int nbuf = prm.eq == KAPSEL_EQ_SHEAR_LE ? 6 : 5;
    KCHECK(cudaMalloc(&bufA, sizeof(Cx<R>) * nbuf * nA));
    KCHECK(cudaMalloc(&bufB, sizeof(Cx<R>) * nbuf * nB));
    KCHECK(cudaMalloc(&ustar, sizeof(R) * 3 * npts()));
    KCHECK(cudaMalloc(&phiup, sizeof(R) * 4 * npts()));
    KCHECK(cudaMalloc(&plane_count, sizeof(unsigned) * g.NX));
    KCHECK(cudaMemset(plane_count, 0, sizeof(unsigned) * g.NX));
    KCHECK(cudaMemset(zeta, 0, sizeof(Cx<R>) * 2 * nz));
    KCHECK(cudaMemset(ustar, 0, sizeof(R) * 3 * npts()));
    KCHECK(cudaMemset(phiup, 0, sizeof(R) * 4 * npts()));
    // twiddles exp(+2 pi i j/n), computed in double
    const int ns[4] = {g.NX, g.NY, g.M, g.NZ};
    std::vector<Cx<R>> h;
    size_t off[4];
    for (int t = 0; t < 4; ++t) {
      off[t] = h.size();
      for (int j = 0; j < ns[t]; ++j) {
        const double a = 2.0 * M_PI * (double)j / (double)ns[t];
        h.push_back({(R)std::cos(a), (R)std::sin(a)});
      }
    }
    KCHECK(cudaMalloc(&twbuf, sizeof(Cx<R>) * h.size()));
    KCHECK(cudaMemcpy(twbuf, h.data(), sizeof(Cx<R>) * h.size(), cudaMemcpyHostToDevice));
    tw.x = twbuf + off[0];
    tw.y = twbuf + off[1];
    tw.m = twbuf + off[2];
    tw.z = twbuf + off[3];
    const size_t C = sizeof(Cx<R>);
    const int P = g.M + 1;
    smem_xu = C * (g.NX + (size_t)2 * g.KXc * KCX + (size_t)2 * g.NX * 3 * KCX);
    smem_xadv = C * (g.NX + (size_t)2 * g.KXc * KCX + (size_t)2 * g.NX * 5 * KCX);
    smem_xf = C * (g.NX + (size_t)2 * g.KXc * KCX + (size_t)2 * g.NX * 3 * KCX);
    smem_y = C * (g.NY + (size_t)2 * g.NY * KCY);
    smem_zp = C * (g.M + g.NZ + (size_t)g.M * (ZROWS * 3 + 1) + (size_t)g.M * (ZROWS * 5 + 1) +
                   std::max((size_t)g.M * ZROWS * 5, (size_t)ZROWS * 5 * (g.TZ + 1)));
    smem_zc = C * (g.M + g.NZ + (size_t)g.M * (ZROWS + 1) + std::max((size_t)g.M * ZROWS, (size_t)ZROWS * (g.TZ + 1)));
    smem_zf = C * (g.M + g.NZ + (size_t)g.M * (ZROWS * 3 + 1) +
                   std::max((size_t)g.M * ZROWS * 3, (size_t)ZROWS * 3 * (g.TZ + 1)));
    smem_zr = C * (g.M + g.NZ + (size_t)g.M * (2 * ZROWS + 1) + (size_t)ZROWS * P);
    const size_t mx = 227 * 1024;
    if (smem_xadv > mx || smem_xu > mx || smem_y > mx || smem_zp > mx) return KAPSEL_ERANGE;
    {
      int rc = 0;
      // the warp-level z kernels give one row group to a warp: below about
      // 16 groups per SM (64^3 and smaller) the block-level kernels, which
      // spread a row group over a whole block, keep more of the GPU busy
      const bool zw_ok = (size_t)g.NX * g.NY >= 16384;
      if (g.NX == 32) rc = x_setup<5>();
      else if (g.NX == 64) rc = x_setup<6>();
      else if (g.NX == 128) rc = x_setup<7>();
      else if (g.NX == 256) rc = x_setup<8>();
      if (rc) return rc;
      if (g.NZ == 64) rc = zw_setup<5>();
      else if (g.NZ == 128) rc = zw_setup<6>();
      else if (g.NZ == 256) rc = zw_setup<7>();
      if (rc) return rc;
      // warp-level z kernels by default only where they fill the GPU (the
      // batch autotuner may choose otherwise per box shape)
      zw_avail = zw;
      if (!zw_ok) zw = 0;
      // FP32: the fused y/z plane kernels wherever the warp-level z kernels
      // run and three plane blocks fit on an SM (128^3 mixed step 0.200 ->
      // 0.189 ms; 256x128x128 0.335 -> 0.316; at 128x128x256, one block per
      // SM, 0.377 -> 0.395, so not there); FP64 planes (90 KB at 128^3)
      // leave one block per SM and run slower than the separate passes
      if (sizeof(R) == 4 && zw && yz_ly && 3 * yz_sm <= 227 * 1024) ymode = 3;
    }
    {
      const int rc = x_setup<0>();
      if (rc) return rc;
    }
    KCHECK(allow_smem(k_y_pass<R, true, KCY>, smem_y));
    KCHECK(allow_smem(k_y_pass<R, false, KCY>, smem_y));
    KCHECK(allow_smem(k_y_pass<R, true, KCY / 2>, smem_y));
    KCHECK(allow_smem(k_y_pass<R, false, KCY / 2>, smem_y));
    KCHECK(allow_smem(k_z_products<R>, smem_zp));
    KCHECK(allow_smem(k_z_c2r<R>, smem_zc));
    KCHECK(allow_smem(k_z_r2c_full<R>, smem_zr));
    KCHECK(allow_smem(k_z_force<R>, smem_zf));
    const int nmax = std::max(g.NX, g.NY);
    const int smem_col = (int)(C * ((size_t)nmax + (size_t)nmax * 16));
    KCHECK(allow_smem(k_col_pass<R, true>, smem_col));
    KCHECK(allow_smem(k_col_pass<R, false>, smem_col));
    KCHECK(allow_smem(k_z_c2r_full<R>, smem_zr));
    return 0;
  }

  dim3 gx() const { return dim3(g.KYc, (g.TZ + KCX - 1) / KCX); }
  dim3 gy(int nc) const { return dim3(g.NX, nc, (g.TZ + KCY - 1) / KCY); }
  // y-pass tile width: KCY, or KCY/2 when the autotuner found it faster for
  // this box shape (kapsel_batch_create)
  bool use_pdl = true;
  // warp-level y pass: persistent grid of YNW-warp blocks, two slots per warp
  static constexpr int YNW = 4;
  static constexpr int YSLOTS = sizeof(R) == 4 ? 1 : 2;
  int yw_occ[2][2] = {{0, 0}, {0, 0}};  // blocks per SM, [inverse][full spectrum]
  int nsm = 0;
  template <bool INV, int LY, bool FULL>
  void yw_launch(const Geo &gg, int nc, const Cx<R> *in, Cx<R> *out, bool pdl) {
    using Y = ZL<LY>;
    auto kern = k_yw_pass<R, INV, LY, FULL, YNW, YSLOTS>;
    const size_t sm = sizeof(Cx<R>) * YSLOTS * Y::RW * YLines<R, LY>::LS * YNW;
    int &occ = yw_occ[INV ? 1 : 0][FULL ? 1 : 0];
    if (!occ) {
      int dev = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      allow_smem(kern, sm);
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, YNW * 32, sm);
      occ = std::max(occ, 1);
    }
    const int items = nc * gg.NX * ((gg.TZ + Y::RW - 1) / Y::RW);
    const int grid = std::min((items + YNW - 1) / YNW, occ * nsm);
    launch_k(pdl, kern, dim3(grid), dim3(YNW * 32), sm, stream, gg, tw, in, out, nc);
  }
  template <bool INV, int LY>
  void yw(const Geo &gg, int nc, const Cx<R> *in, Cx<R> *out, bool pdl) {
    if (gg.KYc == gg.NY)
      yw_launch<INV, LY, true>(gg, nc, in, out, pdl);
    else
      yw_launch<INV, LY, false>(gg, nc, in, out, pdl);
  }
  int ymode = 0;   // y pass variant (time_variant)
  int zw_avail = 0;  // warp-level z kernels set up for this NZ (their line-length log), else 0
  template <bool INV>
  void launch_y(const Geo &gg, int nc, const Cx<R> *in, Cx<R> *out, bool pdl = false) {
    if (ymode == 0 || ymode == 3) switch (gg.NY) {
      case 32: yw<INV, 5>(gg, nc, in, out, pdl); return;
      case 64: yw<INV, 6>(gg, nc, in, out, pdl); return;
      case 128: yw<INV, 7>(gg, nc, in, out, pdl); return;
      case 256: yw<INV, 8>(gg, nc, in, out, pdl); return;
      default: break;
    }
    constexpr int K2 = KCY / 2;
    const size_t sm = std::max(smem_y, sm_y_any);
    if (ymode == 2)
      launch_k(pdl, k_y_pass<R, INV, K2>, dim3(g.NX, nc, (gg.TZ + K2 - 1) / K2), dim3(256), sm, stream, gg, tw, in,
               out);
    else
      launch_k(pdl, k_y_pass<R, INV, KCY>, dim3(g.NX, nc, (gg.TZ + KCY - 1) / KCY), dim3(256), sm, stream, gg, tw,
               in, out);
  }
  size_t sm_y_any = 0;
  bool xsplit_ok(int xs) const override { return xs == 0 || (xs == 1 && g.NX >= 8 && g.NX <= 128); }
  void set_xsplit(int xs) override {
    if (xs == xsplit) return;
    xsplit = xs;
    // bufA's u_k was formed with the other split; the captured graphs hold
    // the other launches
    u_spec_ready = false;
    for (int s = 0; s < 2; ++s)
      if (graph[s]) {
        cudaGraphExecDestroy(graph[s]);
        graph[s] = nullptr;
      }
  }
  bool variant_ok(int zmode, int ymode_) const override {
    if (prm.eq != KAPSEL_EQ_NAVIER_STOKES || zmode < 0 || zmode > 1 || ymode_ < 0 || ymode_ > 3) return false;
    if (zmode == 0 && !zw_avail) return false;
    if ((ymode_ == 0 || ymode_ == 3) && !(g.NY >= 32 && g.NY <= 256)) return false;
    if (ymode_ == 3 && (zmode != 0 || !yz_ly || Np == 0)) return false;
    return true;
  }
  void set_variant(int zmode, int ymode_) override {
    zw = zmode == 0 ? zw_avail : 0;
    ymode = ymode_;
    // the box's captured step graphs hold the previous launches
    for (int s = 0; s < 2; ++s)
      if (graph[s]) {
        cudaGraphExecDestroy(graph[s]);
        graph[s] = nullptr;
      }
  }
  float time_variant(int zmode, int ymode_, int reps) override {
    // a copy of the state the steps change (zeta, uk_dc, particles), restored
    // afterwards; phi/up are all zero again after every step
    const size_t nz = (size_t)g.KXc * g.KYc * g.TS;
    Cx<R> *z0 = nullptr;
    double *u0 = nullptr;
    DPart *p0 = nullptr;
    const int np1 = std::max(Np, 1);
    if (cudaMalloc(&z0, sizeof(Cx<R>) * 2 * nz) != cudaSuccess || cudaMalloc(&u0, sizeof(double) * 3) != cudaSuccess ||
        cudaMalloc(&p0, sizeof(DPart) * np1) != cudaSuccess) {
      cudaFree(z0);
      cudaFree(u0);
      return -1.f;
    }
    cudaMemcpyAsync(z0, zeta, sizeof(Cx<R>) * 2 * nz, cudaMemcpyDeviceToDevice, stream);
    cudaMemcpyAsync(u0, uk_dc, sizeof(double) * 3, cudaMemcpyDeviceToDevice, stream);
    cudaMemcpyAsync(p0, parts, sizeof(DPart) * np1, cudaMemcpyDeviceToDevice, stream);
    const int kz = zw, ky = ymode;
    zw = zmode == 0 ? zw_avail : 0;
    ymode = ymode_;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    u_spec_ready = false;
    ensure_u_spec();
    launch_step(noise_dev[0], 0);  // warm
    cudaEventRecord(a, stream);
    for (int r = 0; r < reps; ++r) launch_step(noise_dev[0], 0);
    cudaEventRecord(b, stream);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    zw = kz;
    ymode = ky;
    cudaMemcpyAsync(zeta, z0, sizeof(Cx<R>) * 2 * nz, cudaMemcpyDeviceToDevice, stream);
    cudaMemcpyAsync(uk_dc, u0, sizeof(double) * 3, cudaMemcpyDeviceToDevice, stream);
    cudaMemcpyAsync(parts, p0, sizeof(DPart) * np1, cudaMemcpyDeviceToDevice, stream);
    cudaStreamSynchronize(stream);
    cudaFree(z0);
    cudaFree(u0);
    cudaFree(p0);
    // the timed steps overwrote bufA: it no longer holds u_k of the current zeta
    u_spec_ready = false;
    return ms / reps;
  }
  int gz() const { return (g.NX * g.NY) / ZROWS; }

  // zeta -> u* (real) through launches 1,2,(7); used by the velocity readout
  void launch_zeta_to_real(R *out, size_t cstride, int pitch) {
    x_zeta(false, zeta, uk_dc, bufA);
    launch_y<true>(g, 3, bufA, bufB);
    k_z_c2r<R><<<dim3(gz(), 3), 256, smem_zc, stream>>>(g, tw, bufB, out, cstride, pitch, PPar{}, nullptr, 0, nullptr);
  }

  // f (from phi/up and u*) -> zeta update, launches 11-13
  void launch_force_to_zeta() {
    zdisp_force(false);
    launch_y<false>(g, 3, bufB, bufA);
    x_force(false, bufA);
  }

  void launch_step(const double *noise, int euler, cudaEvent_t *ev = nullptr) override {
    if (prm.eq == KAPSEL_EQ_ELECTROLYTE) {
      launch_step_el(euler);
      return;
    }
    if (prm.eq == KAPSEL_EQ_SHEAR_LE) {
      launch_step_obl(noise, euler);
      return;
    }
    int e = 0;
    auto mark = [&]() {
      if (ev) cudaEventRecord(ev[e++], stream);
    };
    const bool pdl = use_pdl && !ev;  // events between launches break the programmatic chain
    const Cx<R> *czeta = zeta;
    // the fused path starts at the y pass: the previous step's last launch
    // (or ensure_u_spec) left u_k in bufA; profiling times every launch
    const bool fused = ends_with_u_spec() && !ev;
    mark();
    if (!fused) x_zeta(false, czeta, (const double *)uk_dc, bufA);
    mark();
    launch_y<true>(g, 3, bufA, bufB, pdl);
    mark();
    zdisp_products(pdl);
    mark();
    launch_y<false>(g, 5, bufB, bufA, pdl);
    mark();
    x_advect<0>(pdl);
    mark();
    // ymode 3: the inverse y and z c2r as one launch (k_yzw_c2r), and the
    // force's z and y passes as one (k_zyw_force); their y slots stay empty
    const bool yzf = fused_yz();
    if (!yzf) launch_y<true>(g, 3, bufA, bufB, pdl);
    mark();
    // u* and, in extra blocks, the particle positions (a launch of their own
    // when profiling, so that each launch is timed separately)
    const bool fuse_pos = Np > 0 && !ev;
    if (yzf)
      yz_c2r(pdl, fuse_pos ? parts : (DPart *)nullptr, euler);
    else
      zdisp_c2r(pdl, fuse_pos ? parts : (DPart *)nullptr, euler);
    mark();
    if (Np > 0) {
      if (!fuse_pos) k_particles_position<<<(Np + 127) / 128, 128, 0, stream>>>(pp, parts, euler, status);
      launch_cells();  // neighbour lists of the new positions (large particle counts)
      mark();
      if (nc) launch_nearcontact();  // timed with the position slot when profiling
      launch_k(pdl, k_particles_hydro_velocity<R>, dim3(Np * pp.hyd_pcl), dim3(pp.hyd_threads), 0, stream, pp, parts,
               (const R *)ustar, (const int *)cells, noise, euler, status, partial_p, arrivals,
               nc ? nc_corr : (double *)nullptr, ovl);
      mark();
      launch_k(pdl, k_particles_scatter<R>, dim3(Np * PCL), dim3(256), 0, stream, pp, (const DPart *)parts,
               (const int *)cells, phiup, status, (const unsigned *)ovl);
      mark();
      if (yzf)
        zy_force(pdl);
      else
        zdisp_force(pdl);
      mark();
      if (!yzf) launch_y<false>(g, 3, bufB, bufA, pdl);
      mark();
      if (fused)
        x_force_next(pdl);
      else
        x_force(pdl, bufA);
      mark();
    }
  }

  void ensure_u_spec() override {
    if (!ends_with_u_spec() || u_spec_ready) return;
    x_zeta(false, zeta, uk_dc, bufA);
    u_spec_ready = true;
  }
  bool ends_with_u_spec() const override { return prm.eq == KAPSEL_EQ_NAVIER_STOKES && Np > 0; }
  bool fused_yz() const override { return prm.eq == KAPSEL_EQ_NAVIER_STOKES && ymode == 3 && zw && yz_ly && Np > 0; }

  void launch_init() override {
    // Init_zeta_k gives zeta = 0 and u = 0 (init_fluid.cxx:10-26); the
    // initial rigidity projection (sp_3d_ns.cxx:510-524) is then
    // zeta = U2zeta_k(Solenoidal_u(up - phi*0)), followed by uk_dc = 0.
    cudaMemsetAsync(zeta, 0, sizeof(Cx<R>) * 2 * (size_t)g.KXc * g.KYc * g.TS, stream);
    cudaMemsetAsync(ustar, 0, sizeof(R) * 3 * npts(), stream);
    cudaMemsetAsync(uk_dc, 0, sizeof(double) * 3, stream);
    if (Np > 0) {
      launch_cells();
      k_particles_scatter<R><<<Np * PCL, 256, 0, stream>>>(pp, parts, cells, phiup, status);
      launch_force_to_zeta();
    }
    cudaMemsetAsync(uk_dc, 0, sizeof(double) * 3, stream);
  }

  // ---- Lees-Edwards sheared branch on the oblique grid -----------------------
  R *ob6 = nullptr;        // [6][N]: u and vorticity of the advection term, later the force f
  R *obB = nullptr;        // [3][N]: contravariant u on the oblique grid
  double *obst = nullptr;  // degree_oblique, Shear_rate_eff, ... (obl_kernels.cuh)
  OblPar op{};
  size_t sm_xo6 = 0, sm_xo3 = 0, sm_xof = 0;

  int alloc_obl() override {
    const size_t N = npts(), nst = OB_PART + 2 * (size_t)OB_RED_BLOCKS;
    KCHECK(cudaMalloc(&ob6, sizeof(R) * 6 * N));
    KCHECK(cudaMalloc(&obB, sizeof(R) * 3 * N));
    KCHECK(cudaMalloc(&obst, sizeof(double) * nst));
    KCHECK(cudaMemset(ob6, 0, sizeof(R) * 6 * N));
    KCHECK(cudaMemset(obB, 0, sizeof(R) * 3 * N));
    KCHECK(cudaMemset(obst, 0, sizeof(double) * nst));
    const size_t C = sizeof(Cx<R>);
    sm_xo6 = C * (g.NX + (size_t)2 * g.KXc * KCX + (size_t)2 * g.NX * 6 * KCX);
    sm_xo3 = C * (g.NX + (size_t)2 * g.KXc * KCX + (size_t)2 * g.NX * 3 * KCX);
    sm_xof = C * (g.NX + (size_t)2 * g.NX * 3 * KCX);
    if (sm_xo6 > 227 * 1024 || smem_zc > 227 * 1024) return KAPSEL_ERANGE;
    KCHECK(allow_smem(k_x_obl_inv<R, KCX, 6>, sm_xo6));
    KCHECK(allow_smem(k_x_obl_inv<R, KCX, 3>, sm_xo3));
    KCHECK(allow_smem(k_x_obl_fwd<R, KCX, 1>, sm_xof));
    KCHECK(allow_smem(k_x_obl_fwd<R, KCX, 0>, sm_xof));
    KCHECK(allow_smem(k_z_r2c<R>, smem_zc));
    op.shear_rate = prm.shear_rate;
    op.dt = prm.dt;
    // ivolume = Ivolume * POW3(DX); s_rate_eff *= ivolume*NY/(NY - 1) (sp_3d_ns.h:175,192)
    const double LX = g.NX * prm.dx, LY = g.NY * prm.dx, LZ = g.NZ * prm.dx;
    const double ivolume = (1. / (LX * LY * LZ)) * (prm.dx * prm.dx * prm.dx);
    op.srate_scale = ivolume * g.NY / (g.NY - 1);
    op.dx = prm.dx;
    op.NX = g.NX;
    op.NY = g.NY;
    op.NZ = g.NZ;
    return 0;
  }

  // Time_evolution_hydro_OBL (sp_3d_ns.cxx:214-390).
  void launch_step_obl(const double *noise, int euler) {
    const size_t N = npts();
    const int pb = 592;
    // NS_solver_slavedEuler_Shear_OBL: u and omega of the truncated zeta, u x omega,
    // forward, shear correction, curl and the slaved-Euler step
    k_x_obl_inv<R, KCX, 6><<<gx(), 256, sm_xo6, stream>>>(g, tw, zeta, uk_dc, obst, bufA);
    launch_y<true>(g, 6, bufA, bufB);
    k_z_c2r<R><<<dim3(gz(), 6), 256, smem_zc, stream>>>(g, tw, bufB, ob6, N, g.NZ, PPar{}, nullptr, 0, nullptr);
    k_obl_cross<R><<<pb, 256, 0, stream>>>(N, ob6, obB);
    k_z_r2c<R><<<dim3(gz(), 3), 256, smem_zc, stream>>>(g, tw, obB, g.NZ, N, bufB, g.TZ, g.TS);
    launch_y<false>(g, 3, bufB, bufA);
    k_x_obl_fwd<R, KCX, 1><<<gx(), 256, sm_xof, stream>>>(g, tw, bufA, zeta, uk_dc, obst);
    // FIX_CELL on uk_dc, u = Zeta_k2u_k_OBL(zeta, uk_dc), A_k2a
    k_x_obl_inv<R, KCX, 3><<<gx(), 256, sm_xo3, stream>>>(g, tw, zeta, uk_dc, obst, bufA);
    launch_y<true>(g, 3, bufA, bufB);
    k_z_c2r<R><<<dim3(gz(), 3), 256, smem_zc, stream>>>(g, tw, bufB, ob6, N, g.NZ, PPar{}, nullptr, 0, nullptr);
    // deformation: degree_oblique, grid reset, Cartesian u (ustar), Shear_rate_eff
    k_obl_degree<<<1, 32, 0, stream>>>(op, obst);
    k_obl_remap<R><<<pb, 256, 0, stream>>>(op, (const double *)obst, (const R *)ob6, obB);
    k_obl_to_cart<R><<<pb, 256, 0, stream>>>(op, (const double *)obst, (const R *)obB, ustar);
    k_obl_srate_partial<R><<<OB_RED_BLOCKS, 256, 0, stream>>>(op, (const R *)ustar, obst);
    k_obl_srate_final<<<1, 32, 0, stream>>>(op, obst, OB_RED_BLOCKS);
    if (Np > 0) {
      k_obl_position<<<(Np + 127) / 128, 128, 0, stream>>>(pp, parts, euler, (const double *)obst, status);
      k_obl_hydro_velocity<R><<<Np, 256, 0, stream>>>(pp, parts, (const R *)ustar, (const int *)cells, noise, euler,
                                                       (const double *)obst, status);
      k_obl_scatter<R><<<Np * PCL, 256, 0, stream>>>(pp, (const DPart *)parts, (const int *)cells,
                                                      (const double *)obst, phiup);
    }
    // f = up - phi u (Cartesian), u += U2u_oblique(f), forward, Solenoidal_uk_OBL,
    // contra2co, U_k2zeta_k_OBL
    k_obl_force<R><<<pb, 256, 0, stream>>>(N, phiup, (const R *)ustar, ob6);
    k_obl_add_force<R><<<pb, 256, 0, stream>>>(op, (const double *)obst, (const R *)ob6, obB);
    k_z_r2c<R><<<dim3(gz(), 3), 256, smem_zc, stream>>>(g, tw, obB, g.NZ, N, bufB, g.TZ, g.TS);
    launch_y<false>(g, 3, bufB, bufA);
    k_x_obl_fwd<R, KCX, 0><<<gx(), 256, sm_xof, stream>>>(g, tw, bufA, zeta, uk_dc, obst);
  }

  int oblique_state(double *out) override {
    if (!obst) return KAPSEL_EINVAL;
    KCHECK(cudaMemcpyAsync(out, obst, sizeof(double) * 4, cudaMemcpyDeviceToHost, stream));
    KCHECK(cudaStreamSynchronize(stream));
    return 0;
  }
  int set_oblique_state(double deg, double srate) override {
    if (!obst) return KAPSEL_EINVAL;
    const double h[2] = {deg, srate};
    KCHECK(cudaMemcpyAsync(obst + OB_DEG, h, sizeof(h), cudaMemcpyHostToDevice, stream));
    KCHECK(cudaStreamSynchronize(stream));
    return 0;
  }

  // ---- Electrolyte branch (two ion species) --------------------------------
  Cx<R> *conc_k = nullptr;  // [2][KXc][KYc][TS]
  Cx<R> *rho_k = nullptr;   // [KXc][KYc][TS]
  R *phiq = nullptr;        // [5][N]: phi, surface charge, normal x/y/z
  R *creal = nullptr;       // [2][N]
  R *gradr = nullptr;       // [3][N]
  R *ureal = nullptr;       // [3][N]
  R *fluxr = nullptr;       // [3][N]
  R *charge = nullptr;      // [N]
  Cx<R> *F1 = nullptr, *F2 = nullptr;  // full spectra [3][NX][NY][TS of M+1]
  double *scal = nullptr;   // [0] surface-charge scale, [1..2] rescale factors, [3] free volume
  double *partial = nullptr;
  double *total_solute = nullptr;  // [2]
  Geo gF;                    // geometry whose retained box is the whole half spectrum
  size_t sm_el = 0;          // dynamic shared memory of the electrolyte launches

  int alloc_el() override {
    gF = g;
    gF.TX = g.NX / 2 + 1;
    gF.KXc = g.NX;
    gF.TY = g.NY / 2 + 1;
    gF.KYc = g.NY;
    gF.TZ = g.M + 1;
    gF.TS = (gF.TZ + 3) & ~3;
    const size_t nz = (size_t)g.KXc * g.KYc * g.TS, N = npts();
    const size_t nfull = (size_t)g.NX * g.NY * gF.TS;
    KCHECK(cudaMalloc(&conc_k, sizeof(Cx<R>) * 2 * nz));
    KCHECK(cudaMalloc(&rho_k, sizeof(Cx<R>) * nz));
    KCHECK(cudaMalloc(&phiq, sizeof(R) * 5 * N));
    KCHECK(cudaMalloc(&creal, sizeof(R) * 2 * N));
    KCHECK(cudaMalloc(&gradr, sizeof(R) * 3 * N));
    KCHECK(cudaMalloc(&ureal, sizeof(R) * 3 * N));
    KCHECK(cudaMalloc(&fluxr, sizeof(R) * 3 * N));
    KCHECK(cudaMalloc(&charge, sizeof(R) * N));
    KCHECK(cudaMalloc(&F1, sizeof(Cx<R>) * 3 * nfull));
    KCHECK(cudaMalloc(&F2, sizeof(Cx<R>) * 3 * nfull));
    KCHECK(cudaMalloc(&scal, sizeof(double) * 8));
    KCHECK(cudaMalloc(&partial, sizeof(double) * 2 * RED_BLOCKS));
    KCHECK(cudaMalloc(&total_solute, sizeof(double) * 2));
    KCHECK(cudaMemset(conc_k, 0, sizeof(Cx<R>) * 2 * nz));
    KCHECK(cudaMemset(scal, 0, sizeof(double) * 8));
    // one dynamic shared-memory size for every electrolyte launch: the
    // largest of the x passes (full geometry, 3 components) and z passes
    const size_t C = sizeof(Cx<R>);
    const size_t xi = C * (g.NX + (size_t)3 * gF.KXc * KCX + (size_t)2 * g.NX * 3 * KCX);
    const size_t xf = C * (g.NX + (size_t)2 * g.NX * 3 * KCX);
    const size_t zr = C * (g.M + g.NZ + (size_t)g.M * (ZROWS + 1) + std::max((size_t)g.M * ZROWS, (size_t)ZROWS * (g.M + 2)));
    sm_el = std::max(std::max(xi, xf), std::max(zr, smem_zc));
    sm_el = std::max(sm_el, smem_y);
    sm_y_any = sm_el;
    if (sm_el > 227 * 1024) return KAPSEL_ERANGE;
    const int sm = (int)sm_el;
    KCHECK(allow_smem(k_x_inv_op<R, KCX, XI_IDENT, 2, 2>, sm));
    KCHECK(allow_smem(k_x_inv_op<R, KCX, XI_IDENT, 3, 3>, sm));
    KCHECK(allow_smem(k_x_inv_op<R, KCX, XI_GRADPSI, 1, 3>, sm));
    KCHECK(allow_smem(k_x_inv_op<R, KCX, XI_GRADDIFF, 1, 3>, sm));
    KCHECK(allow_smem(k_x_fwd_op<R, KCX, XF_STORE, 1>, sm));
    KCHECK(allow_smem(k_x_fwd_op<R, KCX, XF_CONCUPD, 3>, sm));
    KCHECK(allow_smem(k_x_fwd_op<R, KCX, XF_GRADPSI_FULL, 1>, sm));
    KCHECK(allow_smem(k_x_fwd_op<R, KCX, XF_PSI_FULL, 1>, sm));
    KCHECK(allow_smem(k_x_inv_op<R, KCX, XI_IDENT, 1, 1>, sm));
    KCHECK(allow_smem(k_z_r2c<R>, sm));
    KCHECK(allow_smem(k_z_c2r<R>, sm));
    KCHECK(allow_smem(k_y_pass<R, true, KCY>, sm));
    KCHECK(allow_smem(k_y_pass<R, false, KCY>, sm));
    KCHECK(allow_smem(k_y_pass<R, true, KCY / 2>, sm));
    KCHECK(allow_smem(k_y_pass<R, false, KCY / 2>, sm));
    KCHECK(allow_smem(k_x_advect_update<R, KCX, 1>, smem_xadv));
    return 0;
  }

  dim3 gxF() const { return dim3(gF.KYc, (gF.TZ + KCX - 1) / KCX); }
  dim3 gyF(int nc) const { return dim3(g.NX, nc, (gF.TZ + KCY - 1) / KCY); }
  double ze() const { return prm.surface_charge * 1.0; }  // Surface_charge_e, Elementary_charge = 1
  bool ext_on() const { return prm.e_ext[0] != 0.0 || prm.e_ext[1] != 0.0 || prm.e_ext[2] != 0.0; }

  // real c_n = A_k2a_out(conc_k[n]) for both species
  void el_conc_real() {
    const size_t nz = (size_t)g.KXc * g.KYc * g.TS;
    k_x_inv_op<R, KCX, XI_IDENT, 2, 2><<<gx(), 256, sm_el, stream>>>(g, tw, conc_k, nz, bufA, KOp{});
    launch_y<true>(g, 2, bufA, bufB);
    k_z_c2r<R><<<dim3(gz(), 2), 256, sm_el, stream>>>(g, tw, bufB, creal, npts(), g.NZ, PPar{}, nullptr, 0, nullptr);
  }
  // surface-charge scale s0 = sum|Z_e| / (sum|surf| DX3) (operate_electrolyte.cxx:217-241)
  void el_surface_scale() {
    k_reduce_partial<R, RED_ABS><<<RED_BLOCKS, 256, 0, stream>>>(npts(), phiq + npts(), nullptr, 0, 1, partial);
    const double dx3 = prm.dx * prm.dx * prm.dx;
    k_reduce_final<<<1, 256, 0, stream>>>(partial, RED_BLOCKS, 1, 0, fabs(ze()) * Np, total_solute, dx3, scal);
  }
  void el_scatter(int with_normal) {
    cudaMemsetAsync(phiq, 0, sizeof(R) * (with_normal ? 5 : 2) * npts(), stream);
    if (Np > 0) k_particles_scatter_el<R><<<Np * PCL, 256, 0, stream>>>(pp, parts, cells, phiq, ze(), with_normal);
  }
  // forward transform of ncomp real fields, 2/3 modes kept, into bufA (I1 layout)
  void el_forward_trunc(const R *real, int ncomp) {
    k_z_r2c<R><<<dim3(gz(), ncomp), 256, sm_el, stream>>>(g, tw, real, g.NZ, npts(), bufB, g.TZ, g.TS);
    launch_y<false>(g, ncomp, bufB, bufA);
  }
  // inverse of three I1-layout components in bufA into real fields
  void el_inverse3(R *out) {
    launch_y<true>(g, 3, bufA, bufB);
    k_z_c2r<R><<<dim3(gz(), 3), 256, sm_el, stream>>>(g, tw, bufB, out, npts(), g.NZ, PPar{}, nullptr, 0, nullptr);
  }

  // NSsolute_solver_Euler (fluid_solver.cxx:306-326): Rhs_NS_Nernst_Planck
  // at the current positions, then the explicit Euler update of zeta and of
  // both ion concentrations (uk_dc is unchanged: its rhs is zero,
  // fluid_solver.cxx:176-178)
  void launch_el_fluid() {
    const size_t N = npts(), nz = (size_t)g.KXc * g.KYc * g.TS;
    const double ve[2] = {prm.valency_p, prm.valency_n}, L[2] = {prm.onsager_p, prm.onsager_n};
    const double ieps = 1.0 / prm.dielectric;
    const int pb = 592;
    // Rhs_NS_Nernst_Planck: charge from the current conc and positions
    el_scatter(1);
    el_surface_scale();
    el_conc_real();
    k_el_charge<R><<<pb, 256, 0, stream>>>(N, phiq, creal, scal, 0, ve[0], ve[1], charge);
    el_forward_trunc(charge, 1);
    k_x_fwd_op<R, KCX, XF_STORE, 1><<<gx(), 256, sm_el, stream>>>(g, tw, bufA, rho_k, 0, KOp{});
    KOp gp{ieps, {prm.e_ext[0] * (double)N, prm.e_ext[1] * (double)N, prm.e_ext[2] * (double)N}};
    k_x_inv_op<R, KCX, XI_GRADPSI, 1, 3><<<gx(), 256, sm_el, stream>>>(g, tw, rho_k, nz, bufA, gp);
    el_inverse3(gradr);
    // Rhs_NS_solute: u, the advection term and the explicit Euler update of zeta
    x_zeta(false, zeta, uk_dc, bufA);
    launch_y<true>(g, 3, bufA, bufB);
    k_z_c2r<R><<<dim3(gz(), 3), 256, sm_el, stream>>>(g, tw, bufB, ureal, N, g.NZ, PPar{}, nullptr, 0, nullptr);
    k_z_products<R><<<gz(), 256, smem_zp, stream>>>(g, tw, bufB);
    launch_y<false>(g, 5, bufB, bufA);
    x_advect<1>(false);
    // ion fluxes and the Euler update of each concentration
    for (int n = 0; n < 2; ++n) {
      KOp dk{prm.kbt * L[n], {0, 0, 0}};
      k_x_inv_op<R, KCX, XI_GRADDIFF, 1, 3><<<gx(), 256, sm_el, stream>>>(g, tw, conc_k + n * nz, nz, bufA, dk);
      el_inverse3(fluxr);
      k_el_flux<R><<<pb, 256, 0, stream>>>(N, fluxr, creal + n * N, gradr, phiq + 2 * N, ureal, N, L[n], ve[n]);
      el_forward_trunc(fluxr, 3);
      k_x_fwd_op<R, KCX, XF_CONCUPD, 3><<<gx(), 256, sm_el, stream>>>(g, tw, bufA, conc_k + n * nz, 0,
                                                                         KOp{prm.dt, {0, 0, 0}});
    }
  }
  // Rescale_solute (solute_rhs.cxx:99-128) at the current positions: the
  // factors total[n] / (sum (1 - phi) c_n DX3) into scal[1..2], conc_k scaled.
  // phiq then holds phi and the surface charge of these positions and creal
  // the concentrations before the scaling.
  void launch_el_rescale() {
    const size_t N = npts(), nz = (size_t)g.KXc * g.KYc * g.TS;
    const double dx3 = prm.dx * prm.dx * prm.dx;
    el_scatter(0);
    el_surface_scale();
    el_conc_real();
    k_reduce_partial<R, RED_PHI_C><<<RED_BLOCKS, 256, 0, stream>>>(N, phiq, creal, N, 2, partial);
    k_reduce_final<<<1, 256, 0, stream>>>(partial, RED_BLOCKS, 2, 1, 0.0, total_solute, dx3, scal);
    k_scale_conc<R><<<592, 256, 0, stream>>>(nz, conc_k, scal);
  }
  // Make_Coulomb_force_x_on_fluid (operate_electrolyte.cxx:90-177) from the
  // charge field: the full (untruncated) potential gradient with the Ooura
  // inverse semantics, then f = charge (-grad psi + E_ext), times `scale`,
  // into fluxr
  void launch_el_coulomb(double scale) {
    const size_t N = npts();
    const double ieps = 1.0 / prm.dielectric;
    const int pb = 592;
    const size_t nfull = (size_t)g.NX * g.NY * gF.TS;
    k_z_r2c<R><<<dim3(gz(), 1), 256, sm_el, stream>>>(gF, tw, charge, g.NZ, N, F2, gF.TZ, gF.TS);
    launch_y<false>(gF, 1, F2, F1);
    k_x_fwd_op<R, KCX, XF_GRADPSI_FULL, 1><<<gxF(), 256, sm_el, stream>>>(gF, tw, F1, F2, nfull,
                                                                             KOp{ieps, {0, 0, 0}});
    k_hermitian_planes<R><<<pb, 256, 0, stream>>>(gF, F2, 3);
    k_x_inv_op<R, KCX, XI_IDENT, 3, 3><<<gxF(), 256, sm_el, stream>>>(gF, tw, F2, nfull, F1, KOp{});
    launch_y<true>(gF, 3, F1, F2);
    k_z_c2r<R><<<dim3(gz(), 3), 256, sm_el, stream>>>(gF, tw, F2, gradr, N, g.NZ, PPar{}, nullptr, 0, nullptr);
    const bool ext = ext_on();
    k_el_coulomb<R><<<pb, 256, 0, stream>>>(N, charge, gradr, ext ? prm.e_ext[0] : 0.0, ext ? prm.e_ext[1] : 0.0,
                                            ext ? prm.e_ext[2] : 0.0, scale, fluxr);
  }

  // the Coulomb potential of the charge field (Conc_k2charge_field, A2a_k,
  // Charge_field_k2Coulomb_potential_k_PBC, A_k2a over the full spectrum;
  // avs_output.cxx:463-466) into out[N]
  void launch_el_potential(R *out) {
    const size_t N = npts();
    const size_t nfull = (size_t)g.NX * g.NY * gF.TS;
    k_z_r2c<R><<<dim3(gz(), 1), 256, sm_el, stream>>>(gF, tw, charge, g.NZ, N, F2, gF.TZ, gF.TS);
    launch_y<false>(gF, 1, F2, F1);
    k_x_fwd_op<R, KCX, XF_PSI_FULL, 1><<<gxF(), 256, sm_el, stream>>>(gF, tw, F1, F2, nfull,
                                                                         KOp{1.0 / prm.dielectric, {0, 0, 0}});
    k_hermitian_planes<R><<<592, 256, 0, stream>>>(gF, F2, 1);
    k_x_inv_op<R, KCX, XI_IDENT, 1, 1><<<gxF(), 256, sm_el, stream>>>(gF, tw, F2, nfull, F1, KOp{});
    launch_y<true>(gF, 1, F1, F2);
    k_z_c2r<R><<<dim3(gz(), 1), 256, sm_el, stream>>>(gF, tw, F2, out, N, g.NZ, PPar{}, nullptr, 0, nullptr);
  }

  // The fields of Output_avs_charge (avs_output.cxx:451-549) at the current
  // state, as NX*NY*NZ_ doubles: phi and the normalised surface charge
  // density of Make_phi_qq_particle (operate_electrolyte.cxx:179-242), the
  // real concentrations of both species (A_k2a of conc_k) and the Coulomb
  // potential.  Scratch fields only: the state is not changed.
  int el_snapshot_host(double *phi, double *surf, double *conc, double *pot) override {
    if (prm.eq != KAPSEL_EQ_ELECTROLYTE || !conc_k) return KAPSEL_EINVAL;
    const size_t N = npts();
    launch_cells();
    el_scatter(0);
    el_surface_scale();
    el_conc_real();
    k_el_charge<R><<<592, 256, 0, stream>>>(N, phiq, creal, scal, 0, prm.valency_p, prm.valency_n, charge);
    launch_el_potential(gradr);
    KCHECK(cudaGetLastError());
    std::vector<R> h(5 * N);  // phi, surface, c0, c1, potential
    double s0 = 0.0;
    KCHECK(cudaMemcpyAsync(h.data(), phiq, sizeof(R) * 2 * N, cudaMemcpyDeviceToHost, stream));
    KCHECK(cudaMemcpyAsync(h.data() + 2 * N, creal, sizeof(R) * 2 * N, cudaMemcpyDeviceToHost, stream));
    KCHECK(cudaMemcpyAsync(h.data() + 4 * N, gradr, sizeof(R) * N, cudaMemcpyDeviceToHost, stream));
    KCHECK(cudaMemcpyAsync(&s0, scal, sizeof(double), cudaMemcpyDeviceToHost, stream));
    KCHECK(cudaStreamSynchronize(stream));
    const int NZ_ = g.NZ + 2;
    const size_t rows = (size_t)g.NX * g.NY, plane = rows * NZ_;
    for (size_t r = 0; r < rows; ++r)
      for (int k = 0; k < g.NZ; ++k) {
        const size_t i = r * g.NZ + k, o = r * NZ_ + k;
        phi[o] = (double)h[i];
        surf[o] = (double)h[N + i] * s0;
        conc[o] = (double)h[2 * N + i];
        conc[plane + o] = (double)h[3 * N + i];
        pot[o] = (double)h[4 * N + i];
      }
    return 0;
  }

  void launch_step_el(int euler) {
    const size_t N = npts();
    const double ve[2] = {prm.valency_p, prm.valency_n};
    launch_el_fluid();
    if (Np > 0) k_particles_position<<<(Np + 127) / 128, 128, 0, stream>>>(pp, parts, euler, status);
    launch_cells();
    // Rescale_solute at the new positions, then the Coulomb force (the
    // charge from the concentrations before the scaling times the factors)
    launch_el_rescale();
    k_el_charge<R><<<592, 256, 0, stream>>>(N, phiq, creal, scal, 1, ve[0], ve[1], charge);
    launch_el_coulomb(prm.dt / prm.rho);
    // u += f dt/rho; Solenoidal_u: in k-space zeta += zeta(sol f), uk_dc += f(0)
    el_forward_trunc(fluxr, 3);
    x_force(false, bufA);
    // u (real) of the updated zeta, then the particle part of the step
    x_zeta(false, zeta, uk_dc, bufA);
    launch_y<true>(g, 3, bufA, bufB);
    k_z_c2r<R><<<dim3(gz(), 3), 256, smem_zc, stream>>>(g, tw, bufB, ustar, N, g.NZ, PPar{}, nullptr, 0, nullptr);
    if (Np > 0) {
      k_particles_hydro_velocity<R><<<Np * pp.hyd_pcl, pp.hyd_threads, 0, stream>>>(pp, parts, ustar, cells, nullptr, euler, status,
                                                                  partial_p, arrivals);
      k_particles_scatter<R><<<Np * PCL, 256, 0, stream>>>(pp, parts, cells, phiup, status);
      launch_force_to_zeta();
    }
  }

  // Init_rho_ion, salt with a uniform initial profile (operate_electrolyte.cxx:
  // 516-575, 692-815): densities from the free volume sum(1 - phi).
  int init_el() override {
    el_scatter(0);
    k_reduce_partial<R, RED_1MPHI><<<RED_BLOCKS, 256, 0, stream>>>(npts(), phiq, nullptr, 0, 1, partial);
    k_reduce_final<<<1, 256, 0, stream>>>(partial, RED_BLOCKS, 1, 2, 0.0, total_solute, 1.0, scal);
    double h[8];
    KCHECK(cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, stream));
    KCHECK(cudaStreamSynchronize(stream));
    const double vol = h[3], dx3 = prm.dx * prm.dx * prm.dx;
    const double Z = prm.surface_charge, v0 = prm.valency_p, v1 = prm.valency_n;
    const double pos = Z < 0. ? fabs(Z * Np / v0) : 0.0, neg = Z > 0. ? fabs(Z * Np / v1) : 0.0;
    const double e = 1.0;  // Elementary_charge
    const double rho_inf = prm.kbt * prm.dielectric / ((e * prm.debye_length) * (e * prm.debye_length));
    const double c0 = pos / (vol * dx3) + rho_inf / (v0 * (v0 - v1));
    const double c1 = neg / (vol * dx3) + -rho_inf / (v1 * (v0 - v1));
    const double tot[2] = {c0 * vol * dx3, c1 * vol * dx3};
    const double Nn = (double)npts();
    const size_t nz = (size_t)g.KXc * g.KYc * g.TS;
    KCHECK(cudaMemsetAsync(conc_k, 0, sizeof(Cx<R>) * 2 * nz, stream));
    const Cx<R> k0[2] = {{(R)(c0 * Nn), (R)0}, {(R)(c1 * Nn), (R)0}};
    KCHECK(cudaMemcpyAsync(conc_k, &k0[0], sizeof(Cx<R>), cudaMemcpyHostToDevice, stream));
    KCHECK(cudaMemcpyAsync(conc_k + nz, &k0[1], sizeof(Cx<R>), cudaMemcpyHostToDevice, stream));
    KCHECK(cudaMemcpyAsync(total_solute, tot, sizeof(tot), cudaMemcpyHostToDevice, stream));
    KCHECK(cudaStreamSynchronize(stream));
    return 0;
  }

  // Concentration fields (2, NX, NY, NZ_) in the Ooura layout -> compact
  // retained modes (the others are truncated before any use).
  int conc_from_host(const double *c) override {
    if (!conc_k) return KAPSEL_ESTATE;
    const size_t nz = (size_t)g.KXc * g.KYc * g.TS;
    std::vector<Cx<R>> h(2 * nz, Cx<R>{R(0), R(0)});
    const int NZ_ = g.NZ + 2;
    const size_t plane = (size_t)g.NX * g.NY * NZ_;
    for (int q = 0; q < 2; ++q)
      for (int ix = 0; ix < g.KXc; ++ix) {
        const int i = ix < g.TX ? ix : g.NX + ix - g.KXc;
        for (int iy = 0; iy < g.KYc; ++iy) {
          const int j = iy < g.TY ? iy : g.NY + iy - g.KYc;
          for (int k = 0; k < g.TZ; ++k) {
            const double *o = c + q * plane + ((size_t)i * g.NY + j) * NZ_ + 2 * k;
            h[q * nz + ((size_t)ix * g.KYc + iy) * g.TS + k] = {(R)o[0], (R)o[1]};
          }
        }
      }
    KCHECK(cudaMemcpyAsync(conc_k, h.data(), sizeof(Cx<R>) * h.size(), cudaMemcpyHostToDevice, stream));
    KCHECK(cudaStreamSynchronize(stream));
    return 0;
  }

  int total_solute_from_host(const double *t) override {
    if (!total_solute) return KAPSEL_ESTATE;
    KCHECK(cudaMemcpyAsync(total_solute, t, sizeof(double) * 2, cudaMemcpyHostToDevice, stream));
    KCHECK(cudaStreamSynchronize(stream));
    return 0;
  }

  int conc_to_host(double *c) override {
    if (!conc_k) return KAPSEL_ESTATE;
    const size_t nz = (size_t)g.KXc * g.KYc * g.TS;
    std::vector<Cx<R>> h(2 * nz);
    KCHECK(cudaMemcpyAsync(h.data(), conc_k, sizeof(Cx<R>) * h.size(), cudaMemcpyDeviceToHost, stream));
    KCHECK(cudaStreamSynchronize(stream));
    const int NZ_ = g.NZ + 2;
    const size_t plane = (size_t)g.NX * g.NY * NZ_;
    memset(c, 0, sizeof(double) * 2 * plane);
    for (int q = 0; q < 2; ++q)
      for (int ix = 0; ix < g.KXc; ++ix) {
        const int i = ix < g.TX ? ix : g.NX + ix - g.KXc;
        for (int iy = 0; iy < g.KYc; ++iy) {
          const int j = iy < g.TY ? iy : g.NY + iy - g.KYc;
          for (int k = 0; k < g.TZ; ++k) {
            const Cx<R> v = h[q * nz + ((size_t)ix * g.KYc + iy) * g.TS + k];
            double *o = c + q * plane + ((size_t)i * g.NY + j) * NZ_ + 2 * k;
            o[0] = (double)v.x;
            o[1] = (double)v.y;
          }
        }
      }
    return 0;
  }

  // ---- host <-> device helpers in the reference layouts
  int velocity_to_host(double *u) override {
    R *tmp = nullptr;
    KCHECK(cudaMallocAsync(&tmp, sizeof(R) * 3 * npts(), stream));
    if (prm.eq == KAPSEL_EQ_SHEAR_LE)
      KCHECK(cudaMemcpyAsync(tmp, ustar, sizeof(R) * 3 * npts(), cudaMemcpyDeviceToDevice, stream));
    else
      launch_zeta_to_real(tmp, npts(), g.NZ);
    std::vector<R> h(3 * npts());
    KCHECK(cudaMemcpyAsync(h.data(), tmp, sizeof(R) * h.size(), cudaMemcpyDeviceToHost, stream));
    KCHECK(cudaFreeAsync(tmp, stream));
    KCHECK(cudaStreamSynchronize(stream));
    const int NZ_ = g.NZ + 2;
    for (int c = 0; c < 3; ++c)
      for (size_t r = 0; r < (size_t)g.NX * g.NY; ++r)
        for (int k = 0; k < g.NZ; ++k)
          u[c * (size_t)g.NX * g.NY * NZ_ + r * NZ_ + k] = (double)h[c * npts() + r * g.NZ + k];
    return 0;
  }

  int zeta_to_host(double *z) override {
    const size_t nz = (size_t)g.KXc * g.KYc * g.TS;
    std::vector<Cx<R>> h(2 * nz);
    KCHECK(cudaMemcpyAsync(h.data(), zeta, sizeof(Cx<R>) * h.size(), cudaMemcpyDeviceToHost, stream));
    KCHECK(cudaStreamSynchronize(stream));
    const int NZ_ = g.NZ + 2;
    const size_t plane = (size_t)g.NX * g.NY * NZ_;
    memset(z, 0, sizeof(double) * 2 * plane);
    for (int c = 0; c < 2; ++c)
      for (int ix = 0; ix < g.KXc; ++ix) {
        const int i = ix < g.TX ? ix : g.NX + ix - g.KXc;
        for (int iy = 0; iy < g.KYc; ++iy) {
          const int j = iy < g.TY ? iy : g.NY + iy - g.KYc;
          for (int k = 0; k < g.TZ; ++k) {
            const Cx<R> v = h[c * nz + ((size_t)ix * g.KYc + iy) * g.TS + k];
            double *o = z + c * plane + ((size_t)i * g.NY + j) * NZ_ + 2 * k;
            o[0] = (double)v.x;
            o[1] = (double)v.y;
          }
        }
      }
    return 0;
  }

  int zeta_from_host(const double *z) override {
    u_spec_ready = false;
    const size_t nz = (size_t)g.KXc * g.KYc * g.TS;
    std::vector<Cx<R>> h(2 * nz);
    const int NZ_ = g.NZ + 2;
    const size_t plane = (size_t)g.NX * g.NY * NZ_;
    for (int c = 0; c < 2; ++c)
      for (int ix = 0; ix < g.KXc; ++ix) {
        const int i = ix < g.TX ? ix : g.NX + ix - g.KXc;
        for (int iy = 0; iy < g.KYc; ++iy) {
          const int j = iy < g.TY ? iy : g.NY + iy - g.KYc;
          for (int k = 0; k < g.TZ; ++k) {
            const double *o = z + c * plane + ((size_t)i * g.NY + j) * NZ_ + 2 * k;
            h[c * nz + ((size_t)ix * g.KYc + iy) * g.TS + k] = {(R)o[0], (R)o[1]};
          }
        }
      }
    KCHECK(cudaMemcpyAsync(zeta, h.data(), sizeof(Cx<R>) * h.size(), cudaMemcpyHostToDevice, stream));
    KCHECK(cudaStreamSynchronize(stream));
    return 0;
  }

  int fft_fwd_host(double *a) override;
  int fft_inv_host(double *a) override;
  int solenoidal_host(double *u0, double *u1, double *u2) override;
  int phi_up_host(double *phi, double *up0, double *up1, double *up2) override;
  int phi_only_host(double *phi) override;
  int fhydro_host(const double *u0, const double *u1, const double *u2, double *f, double *t) override;
  int slaved_euler_host(double *z, const double *ukdc) override {
    // NS_solver_slavedEuler (fluid_solver.cxx:328-354): the advection term
    // of the truncated zeta and the slaved-Euler update of the retained
    // modes (launches 1-5 of the step); the modes outside the 2/3 box, which
    // the reference leaves untouched, keep the caller's values
    if (prm.eq != KAPSEL_EQ_NAVIER_STOKES) return KAPSEL_EINVAL;
    int rc = zeta_from_host(z);
    if (rc) return rc;
    KCHECK(cudaMemcpyAsync(uk_dc, ukdc, sizeof(double) * 3, cudaMemcpyHostToDevice, stream));
    x_zeta(false, zeta, uk_dc, bufA);
    launch_y<true>(g, 3, bufA, bufB);
    zdisp_products(false);
    launch_y<false>(g, 5, bufB, bufA);
    x_advect<0>(false);
    KCHECK(cudaGetLastError());
    // the update also applied FIX_CELL to the device uk_dc and left u_k of the
    // new zeta in bufA; neither is the routine's output: restore uk_dc
    KCHECK(cudaMemcpyAsync(uk_dc, ukdc, sizeof(double) * 3, cudaMemcpyHostToDevice, stream));
    u_spec_ready = false;
    const int NZ_ = g.NZ + 2;
    const size_t plane = (size_t)g.NX * g.NY * NZ_;
    std::vector<double> full(2 * plane);
    if ((rc = zeta_to_host(full.data()))) return rc;
    for (int c = 0; c < 2; ++c)
      for (int ix = 0; ix < g.KXc; ++ix) {
        const int i = ix < g.TX ? ix : g.NX + ix - g.KXc;
        for (int iy = 0; iy < g.KYc; ++iy) {
          const int j = iy < g.TY ? iy : g.NY + iy - g.KYc;
          const size_t o = c * plane + ((size_t)i * g.NY + j) * NZ_;
          memcpy(z + o, full.data() + o, sizeof(double) * 2 * g.TZ);
        }
      }
    return 0;
  }

  // NSsolute_solver_Euler (fluid_solver.cxx:306-326) on host arrays: zeta
  // and both concentrations updated in place.  The reference truncates both
  // to the 2/3 box before it uses them (Rhs_NS_solute, fluid_solver.cxx:
  // 200-210) and updates only that box, so the modes outside it come back
  // zero.  uk_dc is not changed (its right-hand side is zero).
  int ns_solute_host(double *z, const double *ukdc, double *c) override {
    if (prm.eq != KAPSEL_EQ_ELECTROLYTE || !conc_k) return KAPSEL_EINVAL;
    int rc = zeta_from_host(z);
    if (!rc) rc = conc_from_host(c);
    if (rc) return rc;
    KCHECK(cudaMemcpyAsync(uk_dc, ukdc, sizeof(double) * 3, cudaMemcpyHostToDevice, stream));
    launch_cells();
    launch_el_fluid();
    KCHECK(cudaGetLastError());
    // the update applied FIX_CELL to the device uk_dc and overwrote bufA
    KCHECK(cudaMemcpyAsync(uk_dc, ukdc, sizeof(double) * 3, cudaMemcpyHostToDevice, stream));
    u_spec_ready = false;
    if ((rc = zeta_to_host(z))) return rc;
    return conc_to_host(c);
  }

  // Rescale_solute (solute_rhs.cxx:99-128) on host concentrations at the
  // current positions with the caller's target totals; the factors are
  // returned.  The concentrations are the 2/3-truncated ones that
  // NSsolute_solver_Euler leaves (the modes outside the box come back zero).
  // The context's own targets are not changed.
  int rescale_solute_host(const double *total, double *c, double *factors) override {
    if (prm.eq != KAPSEL_EQ_ELECTROLYTE || !conc_k) return KAPSEL_EINVAL;
    int rc = conc_from_host(c);
    if (rc) return rc;
    double *own = total_solute, *tmp = nullptr;
    if (cudaMalloc(&tmp, sizeof(double) * 2) != cudaSuccess) return KAPSEL_ENOMEM;
    if (cudaMemcpyAsync(tmp, total, sizeof(double) * 2, cudaMemcpyHostToDevice, stream) != cudaSuccess) rc = KAPSEL_ECUDA;
    if (!rc) {
      total_solute = tmp;
      launch_cells();
      launch_el_rescale();
      total_solute = own;
      if (cudaGetLastError() != cudaSuccess) rc = KAPSEL_ECUDA;
    }
    double h[3] = {0.0, 0.0, 0.0};
    if (!rc && cudaMemcpyAsync(h, scal, sizeof(h), cudaMemcpyDeviceToHost, stream) != cudaSuccess) rc = KAPSEL_ECUDA;
    if (!rc) rc = conc_to_host(c);  // synchronises the stream
    cudaFree(tmp);
    if (rc) return rc;
    factors[0] = h[1];
    factors[1] = h[2];
    return 0;
  }

  // Make_Coulomb_force_x_on_fluid (operate_electrolyte.cxx:90-177) from host
  // concentrations at the current positions: the force density
  // charge * (-grad psi + E_ext) as three real fields in the reference layout
  // (NX*NY*NZ_ doubles each, the two padding entries of a row zero).
  int coulomb_force_host(const double *c, double *f0, double *f1, double *f2) override {
    if (prm.eq != KAPSEL_EQ_ELECTROLYTE || !conc_k) return KAPSEL_EINVAL;
    int rc = conc_from_host(c);
    if (rc) return rc;
    const size_t N = npts();
    launch_cells();
    el_scatter(0);
    el_surface_scale();
    el_conc_real();
    k_el_charge<R><<<592, 256, 0, stream>>>(N, phiq, creal, scal, 0, prm.valency_p, prm.valency_n, charge);
    launch_el_coulomb(1.0);
    KCHECK(cudaGetLastError());
    std::vector<R> h(3 * N);
    KCHECK(cudaMemcpyAsync(h.data(), fluxr, sizeof(R) * h.size(), cudaMemcpyDeviceToHost, stream));
    KCHECK(cudaStreamSynchronize(stream));
    double *f[3] = {f0, f1, f2};
    const int NZ_ = g.NZ + 2;
    const size_t rows = (size_t)g.NX * g.NY;
    for (int d = 0; d < 3; ++d)
      for (size_t r = 0; r < rows; ++r) {
        double *o = f[d] + r * NZ_;
        const R *in = h.data() + d * N + r * g.NZ;
        for (int k = 0; k < g.NZ; ++k) o[k] = (double)in[k];
        o[g.NZ] = o[g.NZ + 1] = 0.0;
      }
    return 0;
  }

  void free_all() override {
    cudaFree(ob6);
    cudaFree(obB);
    cudaFree(obst);
    cudaFree(conc_k);
    cudaFree(rho_k);
    cudaFree(phiq);
    cudaFree(creal);
    cudaFree(gradr);
    cudaFree(ureal);
    cudaFree(fluxr);
    cudaFree(charge);
    cudaFree(F1);
    cudaFree(F2);
    cudaFree(scal);
    cudaFree(partial);
    cudaFree(total_solute);
    cudaFree(zeta);
    cudaFree(bufA);
    cudaFree(bufB);
    cudaFree(ustar);
    cudaFree(phiup);
    cudaFree(twbuf);
    cudaFree(plane_count);
  }
};

// Host copies of padded NX*NY*NZ_ real fields to packed R device arrays.
template <typename R>
std::vector<R> pack_real(const double *a, const Geo &g) {
  const int NZ_ = g.NZ + 2;
  std::vector<R> h((size_t)g.NX * g.NY * g.NZ);
  for (size_t r = 0; r < (size_t)g.NX * g.NY; ++r)
    for (int k = 0; k < g.NZ; ++k) h[r * g.NZ + k] = (R)a[r * NZ_ + k];
  return h;
}
template <typename R>
void unpack_real(double *a, const R *h, const Geo &g) {
  const int NZ_ = g.NZ + 2;
  for (size_t r = 0; r < (size_t)g.NX * g.NY; ++r)
    for (int k = 0; k < g.NZ; ++k) a[r * NZ_ + k] = (double)h[r * g.NZ + k];
}

// The full-spectrum transforms are built from the same passes with a
// geometry whose "retained" box is the whole half spectrum:
// KXc = NX (ix == i), KYc = NY, TZ = NZ/2+1.  The x pass kernels of the step
// are specialised to the SPM operators, so the routine-level transforms use
// the y pass twice (x and y are both complex transforms over a row of a
// transposed view) -- here done through a generic column pass below.
template <typename R, bool INVERSE>
__global__ void k_col_pass(Geo g, const Cx<R> *twn, int logn, int n, const Cx<R> *in,
                                                  Cx<R> *out,
                                                  long long line_stride, long long elem_stride, int nlines,
                                                  int lines_per_plane, long long plane_stride) {
  // generic batched FFT over lines: line l = p*lines_per_plane + q starts at
  // p*plane_stride + q*line_stride, element e at + e*elem_stride
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cx<R> *tws = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *B = tws + n;  // [n][16]
  load_twiddles(tws, twn, n);
  const int l0 = blockIdx.x * 16;
  auto line_base = [&](int l) {
    const int p = l / lines_per_plane, q = l - p * lines_per_plane;
    return (long long)p * plane_stride + (long long)q * line_stride;
  };
  for (int it = threadIdx.x; it < n * 16; it += blockDim.x) {
    const int col = it % 16, e = it / 16;
    Cx<R> v = {R(0), R(0)};
    if (l0 + col < nlines) v = in[line_base(l0 + col) + (long long)e * elem_stride];
    B[bitrev(e, logn) * 16 + col] = v;
  }
  __syncthreads();
  fft_inplace(B, logn, 16, 1, 16, tws, INVERSE ? -1 : 1);
  for (int it = threadIdx.x; it < n * 16; it += blockDim.x) {
    const int col = it % 16, e = it / 16;
    if (l0 + col < nlines) out[line_base(l0 + col) + (long long)e * elem_stride] = B[e * 16 + col];
  }
}

// z c2r over all kz (routine-level A_k2a): in [NX*NY][M+1] complex
template <typename R>
__global__ void k_z_c2r_full(Geo g, Twiddles<R> tw, const Cx<R> *__restrict__ in,
                                                    R *__restrict__ out, double scale) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int M = g.M, P = M + 1;
  Cx<R> *twm = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *twz = twm + M;
  Cx<R> *S = twz + g.NZ;
  load_twiddles(twm, tw.m, M);
  load_twiddles(twz, tw.z, g.NZ);
  __syncthreads();
  const size_t row0 = (size_t)blockIdx.x * ZROWS;
  for (int it = threadIdx.x; it < ZROWS * M; it += blockDim.x) {
    const int k = it % M, rr = it / M;
    S[rr * P + bitrev(k, g.lm)] = c2r_pre(in + (row0 + rr) * (M + 1), k, M, M + 1, twz);
  }
  __syncthreads();
  fft_inplace(S, g.lm, ZROWS, P, 1, twm, -1);
  for (int it = threadIdx.x; it < ZROWS * M; it += blockDim.x) {
    const int n = it % M, rr = it / M;
    const Cx<R> v = S[rr * P + n];
    out[(row0 + rr) * g.NZ + 2 * n] = (R)(v.x * scale);
    out[(row0 + rr) * g.NZ + 2 * n + 1] = (R)(v.y * scale);
  }
}

template <typename R>
struct FullFFT {
  // forward: real [NX][NY][NZ] -> complex [NX][NY][M+1] (Ooura sign, unscaled)
  static int forward(Box<R> &b, const R *in, Cx<R> *out) {
    const Geo &g = b.g;
    const int M1 = g.M + 1;
    k_z_r2c_full<R><<<b.gz(), 256, b.smem_zr, b.stream>>>(g, b.tw, in, g.NZ, out);
    // y: lines (x, kz): line stride... lines indexed l = x*M1 + kz -> base x*NY*M1 + kz
    col_pass(b, out, g.NY, g.ly, b.tw.y, false, 1);
    col_pass(b, out, g.NX, g.lx, b.tw.x, false, 0);
    (void)M1;
    KCHECK(cudaGetLastError());
    return 0;
  }
  static int inverse(Box<R> &b, Cx<R> *in, R *out) {
    const Geo &g = b.g;
    col_pass(b, in, g.NX, g.lx, b.tw.x, true, 0);
    col_pass(b, in, g.NY, g.ly, b.tw.y, true, 1);
    k_z_c2r_full<R><<<b.gz(), 256, b.smem_zr, b.stream>>>(g, b.tw, in, out, g.inv_n);
    KCHECK(cudaGetLastError());
    return 0;
  }
  // axis 0: transform along x (lines = (y,kz), elem stride NY*M1)
  // axis 1: transform along y (lines = (x,kz), elem stride M1)
  static void col_pass(Box<R> &b, Cx<R> *data, int n, int logn, const Cx<R> *twn, bool inv, int axis) {
    const Geo &g = b.g;
    const int M1 = g.M + 1;
    const size_t sm = sizeof(Cx<R>) * (n + (size_t)n * 16);
    // axis 0: lines are contiguous (l = y*M1 + kz), element stride NY*M1;
    // axis 1: lines (x, kz), kz contiguous within the x-plane, element stride M1
    const int nlines = axis == 0 ? g.NY * M1 : g.NX * M1;
    const int lpp = axis == 0 ? nlines : M1;
    const long long es = axis == 0 ? (long long)g.NY * M1 : M1, ps = axis == 0 ? 0 : (long long)g.NY * M1;
    if (inv)
      k_col_pass<R, true><<<(nlines + 15) / 16, 256, sm, b.stream>>>(g, twn, logn, n, data, data, 1, es, nlines,
                                                                       lpp, ps);
    else
      k_col_pass<R, false><<<(nlines + 15) / 16, 256, sm, b.stream>>>(g, twn, logn, n, data, data, 1, es, nlines,
                                                                        lpp, ps);
  }
};

template <typename R>
int Box<R>::fft_fwd_host(double *a) {
  const size_t npt = npts();
  const int M1 = g.M + 1;
  std::vector<R> h = pack_real<R>(a, g);
  R *din = nullptr;
  Cx<R> *dout = nullptr;
  KCHECK(cudaMalloc(&din, sizeof(R) * npt));
  KCHECK(cudaMalloc(&dout, sizeof(Cx<R>) * (size_t)g.NX * g.NY * M1));
  KCHECK(cudaMemcpyAsync(din, h.data(), sizeof(R) * npt, cudaMemcpyHostToDevice, stream));
  int rc = FullFFT<R>::forward(*this, din, dout);
  std::vector<Cx<R>> o((size_t)g.NX * g.NY * M1);
  KCHECK(cudaMemcpyAsync(o.data(), dout, sizeof(Cx<R>) * o.size(), cudaMemcpyDeviceToHost, stream));
  KCHECK(cudaStreamSynchronize(stream));
  cudaFree(din);
  cudaFree(dout);
  if (rc) return rc;
  const int NZ_ = g.NZ + 2;
  for (size_t r = 0; r < (size_t)g.NX * g.NY; ++r)
    for (int k = 0; k < M1; ++k) {
      a[r * NZ_ + 2 * k] = (double)o[r * M1 + k].x;
      a[r * NZ_ + 2 * k + 1] = (double)o[r * M1 + k].y;
    }
  return 0;
}

template <typename R>
int Box<R>::fft_inv_host(double *a) {
  const size_t npt = npts();
  const int M1 = g.M + 1, NZ_ = g.NZ + 2;
  std::vector<Cx<R>> h((size_t)g.NX * g.NY * M1);
  for (size_t r = 0; r < (size_t)g.NX * g.NY; ++r)
    for (int k = 0; k < M1; ++k) h[r * M1 + k] = {(R)a[r * NZ_ + 2 * k], (R)a[r * NZ_ + 2 * k + 1]};
  Cx<R> *din = nullptr;
  R *dout = nullptr;
  KCHECK(cudaMalloc(&din, sizeof(Cx<R>) * h.size()));
  KCHECK(cudaMalloc(&dout, sizeof(R) * npt));
  KCHECK(cudaMemcpyAsync(din, h.data(), sizeof(Cx<R>) * h.size(), cudaMemcpyHostToDevice, stream));
  int rc = FullFFT<R>::inverse(*this, din, dout);
  std::vector<R> o(npt);
  KCHECK(cudaMemcpyAsync(o.data(), dout, sizeof(R) * npt, cudaMemcpyDeviceToHost, stream));
  KCHECK(cudaStreamSynchronize(stream));
  cudaFree(din);
  cudaFree(dout);
  if (rc) return rc;
  unpack_real<R>(a, o.data(), g);
  return 0;
}

// Solenoidal_u: forward, 2/3 truncation, projection, inverse -- on the
// compact spectra through the step's own passes: the forward z/y passes
// (k_z_r2c via k_z_force with phi = 0 is not usable here), so this path uses
// the full transforms and a k-space kernel.
template <typename R>
__global__ void k_solenoidal_full(Geo g, Cx<R> *u0, Cx<R> *u1, Cx<R> *u2) {
  const int M1 = g.M + 1;
  const size_t n = (size_t)g.NX * g.NY * M1;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int k = idx % M1;
    const int j = (idx / M1) % g.NY;
    const int i = idx / ((size_t)M1 * g.NY);
    const int KXi = signed_k(i, g.NX), KYi = signed_k(j, g.NY);
    if (!(abs(KXi) < g.TX && abs(KYi) < g.TY && k < g.TZ)) {
      u0[idx] = {R(0), R(0)};
      u1[idx] = {R(0), R(0)};
      u2[idx] = {R(0), R(0)};
      continue;
    }
    const R kx = R(g.wave[0] * KXi), ky = R(g.wave[1] * KYi), kz = R(g.wave[2] * k);
    const R K2 = kx * kx + ky * ky + kz * kz;
    const R IK2 = K2 > R(0) ? R(1) / K2 : R(0);
    Cx<R> a = u0[idx], b = u1[idx], c = u2[idx];
    const Cx<R> d = {IK2 * (a.x * kx + b.x * ky + c.x * kz), IK2 * (a.y * kx + b.y * ky + c.y * kz)};
    u0[idx] = {a.x - d.x * kx, a.y - d.y * kx};
    u1[idx] = {b.x - d.x * ky, b.y - d.y * ky};
    u2[idx] = {c.x - d.x * kz, c.y - d.y * kz};
  }
}

template <typename R>
int Box<R>::solenoidal_host(double *u0, double *u1, double *u2) {
  const size_t npt = npts();
  const int M1 = g.M + 1;
  double *hu[3] = {u0, u1, u2};
  R *din = nullptr;
  Cx<R> *dk = nullptr;
  const size_t nk = (size_t)g.NX * g.NY * M1;
  KCHECK(cudaMalloc(&din, sizeof(R) * 3 * npt));
  KCHECK(cudaMalloc(&dk, sizeof(Cx<R>) * 3 * nk));
  for (int c = 0; c < 3; ++c) {
    std::vector<R> h = pack_real<R>(hu[c], g);
    KCHECK(cudaMemcpyAsync(din + c * npt, h.data(), sizeof(R) * npt, cudaMemcpyHostToDevice, stream));
    KCHECK(cudaStreamSynchronize(stream));
    FullFFT<R>::forward(*this, din + c * npt, dk + c * nk);
  }
  k_solenoidal_full<R><<<592, 256, 0, stream>>>(g, dk, dk + nk, dk + 2 * nk);
  for (int c = 0; c < 3; ++c) {
    FullFFT<R>::inverse(*this, dk + c * nk, din + c * npt);
    std::vector<R> o(npt);
    KCHECK(cudaMemcpyAsync(o.data(), din + c * npt, sizeof(R) * npt, cudaMemcpyDeviceToHost, stream));
    KCHECK(cudaStreamSynchronize(stream));
    unpack_real<R>(hu[c], o.data(), g);
  }
  cudaFree(din);
  cudaFree(dk);
  return 0;
}

template <typename R>
int Box<R>::phi_up_host(double *phi, double *up0, double *up1, double *up2) {
  const size_t npt = npts();
  R *d = nullptr;
  KCHECK(cudaMalloc(&d, sizeof(R) * 4 * npt));
  KCHECK(cudaMemsetAsync(d, 0, sizeof(R) * 4 * npt, stream));
  launch_cells();
  if (Np > 0) k_particles_scatter<R><<<Np * PCL, 256, 0, stream>>>(pp, parts, cells, d, status);
  k_clamp_phi<R><<<592, 256, 0, stream>>>(npt, d);
  KCHECK(cudaGetLastError());
  std::vector<R> h(4 * npt);
  KCHECK(cudaMemcpyAsync(h.data(), d, sizeof(R) * h.size(), cudaMemcpyDeviceToHost, stream));
  KCHECK(cudaStreamSynchronize(stream));
  cudaFree(d);
  double *outs[4] = {phi, up0, up1, up2};
  for (int c = 0; c < 4; ++c) unpack_real<R>(outs[c], h.data() + c * npt, g);
  return 0;
}

template <typename R>
int Box<R>::phi_only_host(double *phi) {
  const size_t npt = npts();
  R *d = nullptr;
  KCHECK(cudaMalloc(&d, sizeof(R) * 4 * npt));
  KCHECK(cudaMemsetAsync(d, 0, sizeof(R) * 4 * npt, stream));
  launch_cells();
  if (Np > 0) k_particles_scatter<R><<<Np * PCL, 256, 0, stream>>>(pp, parts, cells, d, status);
  KCHECK(cudaGetLastError());
  std::vector<R> h(npt);
  KCHECK(cudaMemcpyAsync(h.data(), d, sizeof(R) * npt, cudaMemcpyDeviceToHost, stream));
  KCHECK(cudaStreamSynchronize(stream));
  cudaFree(d);
  unpack_real<R>(phi, h.data(), g);
  return 0;
}

template <typename R>
__global__ void k_gather_only(PPar p, const DPart *__restrict__ parts, const R *__restrict__ u,
                              const int *__restrict__ cells, double *__restrict__ out) {
  __shared__ double sh[2 * 6 * 32];
  const int n = blockIdx.x;
  const DPart &a = parts[n];
  const double xp[3] = {a.x[0], a.x[1], a.x[2]};
  const StencilBase b = stencil_base(xp, p);
  const size_t npts = (size_t)p.N[0] * p.N[1] * p.N[2];
  KSum acc[6];
  for (int i = 0; i < 6; ++i) acc[i] = {0.0, 0.0};
  for (int m = threadIdx.x; m < p.S; m += blockDim.x) {
    int rm[3];
    double r[3], dist;
    stencil_point(b, cells + 3 * m, xp, p, rm, r, dist);
    const double ph = (double)prof_phi<R>(dist, p);
    double vr[3] = {0.0, 0.0, 0.0};
    if (p.rotation) {
      vr[0] = a.omega[1] * r[2] - a.omega[2] * r[1];
      vr[1] = a.omega[2] * r[0] - a.omega[0] * r[2];
      vr[2] = a.omega[0] * r[1] - a.omega[1] * r[0];
    }
    const size_t im = ((size_t)rm[0] * p.N[1] + rm[1]) * p.N[2] + rm[2];
    double fp[3];
    for (int d = 0; d < 3; ++d) {
      fp[d] = ((a.v[d] + vr[d]) - (double)u[d * npts + im]) * ph;
      acc[d].add(fp[d]);
    }
    acc[3].add(r[1] * fp[2] - r[2] * fp[1]);
    acc[4].add(r[2] * fp[0] - r[0] * fp[2]);
    acc[5].add(r[0] * fp[1] - r[1] * fp[0]);
  }
  block_reduce<6>(acc, sh);
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d) {
      out[6 * n + d] = p.fh_coef * (acc[d].s + acc[d].c);
      out[6 * n + 3 + d] = p.rotation ? p.fh_coef * (acc[3 + d].s + acc[3 + d].c) : 0.0;
    }
}

template <typename R>
int Box<R>::fhydro_host(const double *u0, const double *u1, const double *u2, double *f, double *t) {
  const size_t npt = npts();
  R *d = nullptr;
  double *o = nullptr;
  KCHECK(cudaMalloc(&d, sizeof(R) * 3 * npt));
  KCHECK(cudaMalloc(&o, sizeof(double) * 6 * (Np > 0 ? Np : 1)));
  const double *hu[3] = {u0, u1, u2};
  for (int c = 0; c < 3; ++c) {
    std::vector<R> h = pack_real<R>(hu[c], g);
    KCHECK(cudaMemcpyAsync(d + c * npt, h.data(), sizeof(R) * npt, cudaMemcpyHostToDevice, stream));
    KCHECK(cudaStreamSynchronize(stream));
  }
  if (Np > 0) k_gather_only<R><<<Np, 256, 0, stream>>>(pp, parts, d, cells, o);
  KCHECK(cudaGetLastError());
  std::vector<double> h(6 * (size_t)Np);
  KCHECK(cudaMemcpyAsync(h.data(), o, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream));
  KCHECK(cudaStreamSynchronize(stream));
  cudaFree(d);
  cudaFree(o);
  for (int n = 0; n < Np; ++n)
    for (int c = 0; c < 3; ++c) {
      f[3 * n + c] = h[6 * n + c];
      t[3 * n + c] = h[6 * n + 3 + c];
    }
  return 0;
}

}  // namespace

// Holds its stream for `ns` nanoseconds of device time (bounded by the
// global timer; no dependence on other work), used only by the profiler.
__global__ void k_time_gate(unsigned long long ns) {
  unsigned long long t0, t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (int i = 0; i < 1000000; ++i) {
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 >= ns) break;
    __nanosleep(1000);
  }
}

// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Learned near-contact correction: network parameters, Adam state and the
// scaling of a trained network.
struct kapsel_nc {
  cudaStream_t stream = nullptr;
  float *params = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr, *loss = nullptr;
  int *status = nullptr;
  long long adam_t = 0;
  nc::NcScale sc{};
  bool scaled = false;
};

static int nc_smem_setup() {
  static std::once_flag once;
  static int rc = 0;
  std::call_once(once, []() {
    if (allow_smem(nc::k_mlp_tile<false>, nc::SMEM_ALLOC) != cudaSuccess ||
        allow_smem(nc::k_mlp_tile<true>, nc::SMEM_ALLOC) != cudaSuccess)
      rc = KAPSEL_ECUDA;
  });
  return rc;
}

void BoxBase::launch_nearcontact() {
  cudaMemsetAsync(nc_count, 0, sizeof(int), stream);
  nc::k_nc_pairs<<<Np, 128, 0, stream>>>(pp, parts, nc->sc, nc_feat, nc_frames, nc_pairs, nc_count, nc_cap, status);
  nc::TileIO io{};
  io.x = nc_feat;
  io.n = -1;
  io.n_dev = nc_count;
  io.n_cap = nc_cap;
  io.status = status;
  io.pairs = nc_pairs;
  io.frames = nc_frames;
  io.corr = nc_corr;
  io.sc = nc->sc;
  // a persistent grid of one CTA per SM walks the tiles of however many
  // pairs the search found (the count is on the device)
  int nsm = 0, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int tiles = (nc_cap + nc::TILE - 1) / nc::TILE;
  nc::k_mlp_tile<false><<<std::min(tiles, std::max(nsm, 1)), 256, nc::SMEM_ALLOC, stream>>>(nc->params, io);
}

struct kapsel_ctx {
  std::unique_ptr<BoxBase> box;
};

extern "C" {

void kapsel_params_default(kapsel_params *p) {
  memset(p, 0, sizeof(*p));
  p->np_xyz[0] = p->np_xyz[1] = p->np_xyz[2] = 6;
  p->eq = KAPSEL_EQ_NAVIER_STOKES;
  p->precision = KAPSEL_FP64;
  p->dx = 1.0;
  p->rho = 1.0;
  p->eta = 1.0;
  p->kbt = 0.0;
  p->alpha_v = 1.0;
  p->alpha_o = 1.0;
  p->dt = 0.01;
  p->a = 5.0;
  p->a_xi = 2.0;
  p->mass_ratio = 1.0;
  p->gravity_dir = 2;
  p->epsilon = 1.0;
  p->lj_powers = 0;
  p->lj_truncate = 1;
  p->rotation = 1;
  p->mt_seed = 0;
}

const char *kapsel_gpu_strerror(int s) {
  switch (s) {
    case KAPSEL_OK: return "ok";
    case KAPSEL_EINVAL: return "invalid argument or unsupported configuration";
    case KAPSEL_ECUDA: return "CUDA runtime error";
    case KAPSEL_ENOMEM: return "device allocation failed";
    case KAPSEL_ESTATE: return "call out of order";
    case KAPSEL_ENONFINITE: return "non-finite particle state";
    case KAPSEL_ERANGE: return "particle out of box or size limit exceeded";
    case KAPSEL_ETIMEOUT: return "a bounded device wait ran out";
    default: return "unknown status";
  }
}

int kapsel_gpu_create(const kapsel_params *p, kapsel_ctx **out) {
  if (!p || !out) return KAPSEL_EINVAL;
  *out = nullptr;
  for (int d = 0; d < 3; ++d)
    // 16..256 per axis: the in-kernel transforms factor a line into two
    // radix-2 networks of at most 16 points
    if (p->np_xyz[d] < 4 || p->np_xyz[d] > 8) return KAPSEL_EINVAL;
  if (p->eq != KAPSEL_EQ_NAVIER_STOKES && p->eq != KAPSEL_EQ_ELECTROLYTE && p->eq != KAPSEL_EQ_SHEAR_LE)
    return KAPSEL_EINVAL;
  if (p->eq == KAPSEL_EQ_SHEAR_LE && !std::isfinite(p->shear_rate)) return KAPSEL_EINVAL;
  if (p->eq == KAPSEL_EQ_ELECTROLYTE && (!(p->dielectric > 0.0) || p->surface_charge == 0.0 || !(p->debye_length > 0.0) ||
                                         !(p->valency_p > 0.0) || !(p->valency_n < 0.0)))
    return KAPSEL_EINVAL;
  if (p->precision != KAPSEL_FP64 && p->precision != KAPSEL_MIXED) return KAPSEL_EINVAL;
  // written so that a NaN fails every test
  if (p->n_particles < 0 || !(p->dx > 0) || !(p->rho > 0) || !(p->eta > 0) || !(p->dt > 0) || !(p->a > 0) ||
      !(p->a_xi > 0))
    return KAPSEL_EINVAL;
  if (!(p->kbt >= 0) || !(p->mass_ratio > 0) || !std::isfinite(p->kbt) || !std::isfinite(p->mass_ratio) ||
      !std::isfinite(p->gravity_g) || !std::isfinite(p->epsilon) || !std::isfinite(p->alpha_v) ||
      !std::isfinite(p->alpha_o) || !std::isfinite(p->e_ext[0]) || !std::isfinite(p->e_ext[1]) ||
      !std::isfinite(p->e_ext[2]))
    return KAPSEL_EINVAL;
  if (p->lj_powers < 0 || p->lj_powers > 2 || p->gravity_dir < 0 || p->gravity_dir > 2) return KAPSEL_EINVAL;
  std::unique_ptr<BoxBase> b;
  if (p->precision == KAPSEL_FP64)
    b.reset(new (std::nothrow) Box<double>());
  else
    b.reset(new (std::nothrow) Box<float>());
  if (!b) return KAPSEL_ENOMEM;
  b->prm = *p;
  Geo &g = b->g;
  g.NX = 1 << p->np_xyz[0];
  g.NY = 1 << p->np_xyz[1];
  g.NZ = 1 << p->np_xyz[2];
  g.M = g.NZ / 2;
  g.lx = ilog2(g.NX);
  g.ly = ilog2(g.NY);
  g.lm = ilog2(g.M);
  g.TX = (g.NX + 2) / 3;
  g.TY = (g.NY + 2) / 3;
  g.TZ = (g.NZ + 2) / 3;
  g.TS = (g.TZ + 3) & ~3;
  g.KXc = 2 * g.TX - 1;
  g.KYc = 2 * g.TY - 1;
  const double L[3] = {g.NX * p->dx, g.NY * p->dx, g.NZ * p->dx};
  for (int d = 0; d < 3; ++d) g.wave[d] = 2.0 * M_PI / L[d];
  g.nu = p->eta / p->rho;
  g.dt = p->dt;
  for (int d = 0; d < 3; ++d) g.fix_cell[d] = p->fix_cell[d] ? 1 : 0;
  // the sheared branches always fix the mean y velocity (input.cxx:1555-1557)
  if (p->eq == KAPSEL_EQ_SHEAR_LE) g.fix_cell[1] = 1;
  g.fp64_exp = p->precision == KAPSEL_FP64 ? 1 : 0;
  g.inv_n = 1.0 / ((double)g.NX * g.NY * g.NZ);

  // particle constants: Set_global_parameters (input.cxx:274-431)
  PPar &pp = b->pp;
  std::vector<int> cells = sekibun(p->a, p->a_xi, p->dx);
  b->Np = p->n_particles;
  b->S = (int)cells.size() / 3;
  pp.Np = b->Np;
  pp.S = b->S;
  pp.N[0] = g.NX;
  pp.N[1] = g.NY;
  pp.N[2] = g.NZ;
  for (int d = 0; d < 3; ++d) {
    pp.L[d] = L[d];
    pp.invL[d] = 1.0 / L[d];
  }
  pp.DX = p->dx;
  pp.RADIUS = p->a * p->dx;
  const double XI = p->a_xi * p->dx;
  pp.HXI = XI * 0.5;
  pp.dt = p->dt;
  const double rho_p = p->mass_ratio * p->rho;
  const double mass = rho_p * 4. / 3. * M_PI * (pp.RADIUS * pp.RADIUS * pp.RADIUS);
  const double moi = 2. / 5. * mass * (pp.RADIUS * pp.RADIUS);
  pp.IMASS = 1. / mass;
  pp.IMOI = 1. / moi;
  const double DX3 = p->dx * p->dx * p->dx;
  pp.fh_coef = (-DX3 * p->rho) / p->dt;
  pp.rotation = p->rotation ? 1 : 0;
  pp.lj_on = p->lj_truncate >= 0 ? 1 : 0;
  pp.lj_powers = p->lj_powers;
  const double sigma = 2.0 * pp.RADIUS;
  double a_r_cutoff = 0.0;
  if (p->lj_truncate > 0) {
    const double pw[3] = {1. / 6., 1. / 12., 1. / 18.};
    a_r_cutoff = std::pow(2., pw[p->lj_powers]);
  } else if (p->lj_truncate == 0) {
    const int nmin = std::min(g.NX, std::min(g.NY, g.NZ));
    a_r_cutoff = std::min(nmin * p->dx * .5 / sigma, 2.5);
  }
  // LJ_dia (input.cxx:388-405): SIGMA, or in the sheared branches
  // MIN((SIGMA + XI)/2^(1/(6(p+1))), SIGMA)
  double lj_dia = sigma;
  if (p->eq == KAPSEL_EQ_SHEAR_LE) {
    const double pw[3] = {1. / 6., 1. / 12., 1. / 18.};
    lj_dia = std::min((sigma + XI) / std::pow(2., pw[p->lj_powers]), sigma);
  }
  pp.lj_dia = lj_dia;
  pp.lj_cut = a_r_cutoff * lj_dia;
  pp.lj_coeff = 24. * (p->lj_powers + 1) * p->epsilon;
  pp.lc[0] = g.NX / 16;
  pp.lc[1] = g.NY / 16;
  pp.lc[2] = g.NZ / 16;
  pp.lc_r = 16 * p->dx;
  const double gravity_on_fluid = p->gravity_g * p->rho * 4. / 3. * M_PI * (pp.RADIUS * pp.RADIUS) * pp.RADIUS;
  pp.grav = p->gravity_g != 0.0 ? gravity_on_fluid * (p->mass_ratio - 1.0) : 0.0;
  pp.gdir = p->gravity_dir;
  // no thermostat in the Electrolyte branch (sp_3d_ns.cxx:183)
  pp.thermostat = (p->kbt > 0.0 && b->Np > 0 && p->eq != KAPSEL_EQ_ELECTROLYTE) ? 1 : 0;
  const double zeta_drag = 6. * M_PI * p->eta * pp.RADIUS;
  const double zeta_drag_rot = 8. * M_PI * p->eta * (pp.RADIUS * pp.RADIUS * pp.RADIUS);
  pp.noise_v = 1.439 * std::sqrt(zeta_drag * p->dt * p->kbt * p->alpha_v);
  pp.noise_o = 1.22 * std::sqrt(zeta_drag_rot * p->dt * p->kbt * p->alpha_o);
  pp.frozen = p->frozen ? 1 : 0;
  // one gather block per particle: 512 threads when there are enough
  // particles to fill the GPU, 1024 (two Sekibun points a thread) otherwise
  pp.hyd_pcl = 1;
  pp.hyd_threads = b->Np >= 128 ? 512 : 1024;
  if (pp.frozen) pp.thermostat = 0;
  if (p->neighbor_lists < -1 || p->neighbor_lists > 1) return KAPSEL_EINVAL;
  b->mt.reset(new MT19937(p->mt_seed));

  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) return KAPSEL_ECUDA;
  int rc = b->alloc();
  if (rc) return rc;
  if (p->eq == KAPSEL_EQ_ELECTROLYTE) {
    rc = b->alloc_el();
    if (rc) return rc;
  }
  if (p->eq == KAPSEL_EQ_SHEAR_LE) {
    rc = b->alloc_obl();
    if (rc) return rc;
  }
  const int np1 = b->Np > 0 ? b->Np : 1;
  if (cudaMalloc(&b->parts, sizeof(DPart) * np1) != cudaSuccess) return KAPSEL_ENOMEM;
  if (cudaMallocHost(&b->parts_host, sizeof(DPart) * np1) != cudaSuccess) return KAPSEL_ENOMEM;
  if (cudaMallocHost(&b->status_host, sizeof(int)) != cudaSuccess) return KAPSEL_ENOMEM;
  if (cudaMemset(b->parts, 0, sizeof(DPart) * np1) != cudaSuccess) return KAPSEL_ECUDA;
  if (cudaMalloc(&b->cells, sizeof(int) * cells.size()) != cudaSuccess) return KAPSEL_ENOMEM;
  if (cudaMemcpy(b->cells, cells.data(), sizeof(int) * cells.size(), cudaMemcpyHostToDevice) != cudaSuccess)
    return KAPSEL_ECUDA;
  if (cudaMalloc(&b->uk_dc, sizeof(double) * 3) != cudaSuccess) return KAPSEL_ENOMEM;
  cudaMemset(b->uk_dc, 0, sizeof(double) * 3);
  if (cudaMalloc(&b->status, sizeof(int)) != cudaSuccess) return KAPSEL_ENOMEM;
  cudaMemset(b->status, 0, sizeof(int));
  // neighbour lists: the Navier_Stokes and Electrolyte particle kernels
  // read them; the range covers the LJ cutoff and two overlapping supports
  if (b->Np > 0 && p->eq != KAPSEL_EQ_SHEAR_LE &&
      (p->neighbor_lists == 1 || (p->neighbor_lists == 0 && b->Np > 1024))) {
    const double rl = std::max(pp.lj_on ? pp.lj_cut : 0.0, 2.0 * (pp.RADIUS + pp.HXI)) * (1.0 + 1e-9);
    rc = b->setup_cells(rl);
    if (rc) return rc;
  }
  if (b->Np > 0 && b->Np <= 1024 && !b->cl_on && pp.hyd_pcl == 1) {
    if (cudaMalloc(&b->ovl, sizeof(unsigned) * 32 * (size_t)b->Np) != cudaSuccess) return KAPSEL_ENOMEM;
    cudaMemset(b->ovl, 0, sizeof(unsigned) * 32 * (size_t)b->Np);
  }
  if (cudaMalloc(&b->partial_p, sizeof(double) * 18 * HYD_PCL_MAX * np1) != cudaSuccess) return KAPSEL_ENOMEM;
  if (cudaMalloc(&b->arrivals, sizeof(int) * np1) != cudaSuccess) return KAPSEL_ENOMEM;
  cudaMemset(b->arrivals, 0, sizeof(int) * np1);
  for (int s = 0; s < 2; ++s) {
    if (cudaMalloc(&b->noise_dev[s], sizeof(double) * 6 * np1) != cudaSuccess) return KAPSEL_ENOMEM;
    if (cudaMallocHost(&b->noise_host[s], sizeof(double) * 6 * np1) != cudaSuccess) return KAPSEL_ENOMEM;
    if (cudaEventCreateWithFlags(&b->noise_ev[s], cudaEventDisableTiming) != cudaSuccess) return KAPSEL_ECUDA;
    cudaMemset(b->noise_dev[s], 0, sizeof(double) * 6 * np1);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return KAPSEL_ECUDA;
  kapsel_ctx *c = new (std::nothrow) kapsel_ctx;
  if (!c) return KAPSEL_ENOMEM;
  c->box = std::move(b);
  *out = c;
  return 0;
}

int kapsel_gpu_destroy(kapsel_ctx *ctx) {
  if (!ctx) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (b) {
    cudaStreamSynchronize(b->stream);
    for (int s = 0; s < 2; ++s) {
      if (b->graph[s]) cudaGraphExecDestroy(b->graph[s]);
      cudaFree(b->noise_dev[s]);
      cudaFreeHost(b->noise_host[s]);
      if (b->noise_ev[s]) cudaEventDestroy(b->noise_ev[s]);
    }
    b->free_all();
    b->free_cells();
    cudaFree(b->parts);
    cudaFreeHost(b->parts_host);
    cudaFreeHost(b->status_host);
    cudaFree(b->cells);
    cudaFree(b->uk_dc);
    cudaFree(b->status);
    cudaFree(b->partial_p);
    cudaFree(b->arrivals);
    cudaFree(b->nc_feat);
    cudaFree(b->nc_frames);
    cudaFree(b->nc_pairs);
    cudaFree(b->nc_count);
    cudaFree(b->nc_corr);
    cudaStreamDestroy(b->stream);
  }
  delete ctx;
  return 0;
}

int kapsel_gpu_set_particles(kapsel_ctx *ctx, const double *x, const double *q) {
  if (!ctx || (!x && ctx->box->Np > 0)) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  std::vector<DPart> h(b->Np > 0 ? b->Np : 1);
  memset(h.data(), 0, sizeof(DPart) * h.size());
  for (int n = 0; n < b->Np; ++n) {
    for (int d = 0; d < 3; ++d) {
      const double v = x[3 * n + d];
      if (!(v >= 0.0 && v < b->pp.L[d])) return KAPSEL_ERANGE;
      h[n].x[d] = v;
      h[n].x_nopbc[d] = v;
    }
    double qq[4] = {1.0, 0.0, 0.0, 0.0};
    if (q) {
      // user_dir orientations are normalised (init_particle.cxx:281-286)
      double nrm = 0.0;
      for (int i = 0; i < 4; ++i) nrm += q[4 * n + i] * q[4 * n + i];
      nrm = std::sqrt(nrm);
      if (!(nrm > 0.0)) return KAPSEL_EINVAL;
      nrm = 1.0 / nrm;
      for (int i = 0; i < 4; ++i) qq[i] = q[4 * n + i] * nrm;
    }
    for (int i = 0; i < 4; ++i) h[n].q[i] = h[n].q_old[i] = qq[i];
  }
  if (cudaMemcpyAsync(b->parts, h.data(), sizeof(DPart) * h.size(), cudaMemcpyHostToDevice, b->stream) !=
          cudaSuccess ||
      cudaMemsetAsync(b->status, 0, sizeof(int), b->stream) != cudaSuccess ||
      cudaStreamSynchronize(b->stream) != cudaSuccess)
    return KAPSEL_ECUDA;
  b->particles_set = true;
  return 0;
}

int kapsel_gpu_init_state(kapsel_ctx *ctx) {
  if (!ctx) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (b->Np > 0 && !b->particles_set) return KAPSEL_ESTATE;
  b->launch_init();
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return KAPSEL_ECUDA;
  if (cudaGetLastError() != cudaSuccess) return KAPSEL_ECUDA;
  if (b->prm.eq == KAPSEL_EQ_ELECTROLYTE) {
    int rc = b->init_el();
    if (rc) return rc;
  }
  if (b->prm.eq == KAPSEL_EQ_SHEAR_LE && b->Np > 0 && !b->prm.frozen) {
    // the sheared branches start every particle with v_x = omega_z = 0 after
    // the initial projection (init_particle.cxx:666-677)
    std::vector<DPart> h(b->Np);
    if (cudaMemcpy(h.data(), b->parts, sizeof(DPart) * b->Np, cudaMemcpyDeviceToHost) != cudaSuccess)
      return KAPSEL_ECUDA;
    for (DPart &a : h) {
      a.v[0] = a.v_old[0] = 0.0;
      a.omega[2] = a.omega_old[2] = 0.0;
    }
    if (cudaMemcpy(b->parts, h.data(), sizeof(DPart) * b->Np, cudaMemcpyHostToDevice) != cudaSuccess)
      return KAPSEL_ECUDA;
  }
  b->ts = 0;
  b->time = 0.0;
  b->drop_prefill();
  b->u_spec_ready = false;
  b->initialised = true;
  return 0;
}

static int check_status(BoxBase *b) {
  int st = 0;
  if (cudaMemcpyAsync(&st, b->status, sizeof(int), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess)
    return KAPSEL_ECUDA;
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return KAPSEL_ECUDA;
  if (cudaGetLastError() != cudaSuccess) return KAPSEL_ECUDA;
  return st;
}

// n steps enqueued on the context's stream (no synchronisation)
static int step_loop(kapsel_ctx *ctx, int n, bool use_graph) {
  if (!ctx || n < 0) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (!b->initialised) return KAPSEL_ESTATE;
  for (int s = 0; s < n; ++s) {
    const int slot = b->ts & 1;
    int rc = b->take_noise(slot);
    if (rc) return rc;
    b->ensure_u_spec();
    const int euler = b->ts == 0 ? 1 : 0;
    if (use_graph && !euler) {
      if (!b->graph[slot]) {
        cudaGraph_t gr;
        if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return KAPSEL_ECUDA;
        b->launch_step(b->noise_dev[slot], 0);
        if (cudaStreamEndCapture(b->stream, &gr) != cudaSuccess) return KAPSEL_ECUDA;
        if (cudaGraphInstantiate(&b->graph[slot], gr, 0) != cudaSuccess) return KAPSEL_ECUDA;
        cudaGraphDestroy(gr);
      }
      if (cudaGraphLaunch(b->graph[slot], b->stream) != cudaSuccess) return KAPSEL_ECUDA;
    } else {
      b->launch_step(b->noise_dev[slot], euler);
    }
    b->u_spec_ready = b->ends_with_u_spec();
    b->ts += 1;
    b->time += b->prm.dt;
    if ((rc = b->prefill_noise())) return rc;
  }
  return 0;
}

static int step_impl(kapsel_ctx *ctx, int n, bool use_graph) {
  const int rc = step_loop(ctx, n, use_graph);
  return rc ? rc : check_status(ctx->box.get());
}

// The particle records (KAPSEL_P_STRIDE doubles each) of the pinned copy.
static void particle_records(const BoxBase *b, double *out) {
  const DPart *h = b->parts_host;
  for (int n = 0; n < b->Np; ++n) {
    double *o = out + (size_t)KAPSEL_P_STRIDE * n;
    const DPart &a = h[n];
    for (int d = 0; d < 3; ++d) {
      o[KAPSEL_P_X + d] = a.x[d];
      o[KAPSEL_P_V + d] = a.v[d];
      o[KAPSEL_P_OMEGA + d] = a.omega[d];
      o[KAPSEL_P_FHYDRO + d] = a.f_hydro_prev[d];
      o[KAPSEL_P_THYDRO + d] = a.t_hydro_prev[d];
      o[KAPSEL_P_FR + d] = a.fr_prev[d];
      o[KAPSEL_P_XNOPBC + d] = a.x_nopbc[d];
      o[KAPSEL_P_VOLD + d] = a.v_old[d];
      o[KAPSEL_P_OMEGAOLD + d] = a.omega_old[d];
    }
    for (int i = 0; i < 4; ++i) {
      o[KAPSEL_P_Q + i] = a.q[i];
      o[KAPSEL_P_QOLD + i] = a.q_old[i];
    }
  }
}

int kapsel_gpu_step(kapsel_ctx *ctx, int n) { return step_impl(ctx, n, false); }
int kapsel_gpu_step_graph(kapsel_ctx *ctx, int n) { return step_impl(ctx, n, true); }

int kapsel_gpu_get_zeta(kapsel_ctx *ctx, double *zeta, double *uk_dc) {
  if (!ctx || !zeta) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  int rc = b->zeta_to_host(zeta);
  if (rc) return rc;
  if (uk_dc) {
    if (cudaMemcpyAsync(uk_dc, b->uk_dc, sizeof(double) * 3, cudaMemcpyDeviceToHost, b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess)
      return KAPSEL_ECUDA;
  }
  return 0;
}

int kapsel_gpu_set_zeta(kapsel_ctx *ctx, const double *zeta, const double *uk_dc) {
  if (!ctx || !zeta || !uk_dc) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  int rc = b->zeta_from_host(zeta);
  if (rc) return rc;
  if (cudaMemcpyAsync(b->uk_dc, uk_dc, sizeof(double) * 3, cudaMemcpyHostToDevice, b->stream) != cudaSuccess ||
      cudaMemsetAsync(b->status, 0, sizeof(int), b->stream) != cudaSuccess ||
      cudaStreamSynchronize(b->stream) != cudaSuccess)
    return KAPSEL_ECUDA;
  b->initialised = true;
  return 0;
}

int kapsel_gpu_get_velocity(kapsel_ctx *ctx, double *u) {
  if (!ctx || !u) return KAPSEL_EINVAL;
  return ctx->box->velocity_to_host(u);
}

int kapsel_gpu_get_particles(kapsel_ctx *ctx, double *out) {
  if (!ctx || (!out && ctx->box->Np > 0)) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (cudaMemcpyAsync(b->parts_host, b->parts, sizeof(DPart) * std::max(b->Np, 1), cudaMemcpyDeviceToHost,
                      b->stream) != cudaSuccess)
    return KAPSEL_ECUDA;
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return KAPSEL_ECUDA;
  particle_records(b, out);
  return 0;
}

int kapsel_gpu_step_graph_particles(kapsel_ctx *ctx, int n, double *out) {
  // the copies of the particles and of the status word follow the steps on
  // the stream, so one synchronisation covers steps, status and readout
  if (!ctx || (!out && ctx->box->Np > 0)) return KAPSEL_EINVAL;
  int rc = step_loop(ctx, n, true);
  if (rc) return rc;
  BoxBase *b = ctx->box.get();
  if (cudaMemcpyAsync(b->parts_host, b->parts, sizeof(DPart) * std::max(b->Np, 1), cudaMemcpyDeviceToHost,
                      b->stream) != cudaSuccess ||
      cudaMemcpyAsync(b->status_host, b->status, sizeof(int), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess)
    return KAPSEL_ECUDA;
  if (cudaStreamSynchronize(b->stream) != cudaSuccess || cudaGetLastError() != cudaSuccess) return KAPSEL_ECUDA;
  particle_records(b, out);
  return *b->status_host;
}

int kapsel_gpu_set_particle_state(kapsel_ctx *ctx, const double *in) {
  if (!ctx || (!in && ctx->box->Np > 0)) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  std::vector<DPart> h(b->Np > 0 ? b->Np : 1);
  memset(h.data(), 0, sizeof(DPart) * h.size());
  for (int n = 0; n < b->Np; ++n) {
    const double *o = in + (size_t)KAPSEL_P_STRIDE * n;
    for (int i = 0; i < KAPSEL_P_STRIDE; ++i)
      if (!std::isfinite(o[i])) return KAPSEL_EINVAL;  // never send a NaN/Inf to the device
    DPart &a = h[n];
    for (int d = 0; d < 3; ++d) {
      a.x[d] = o[KAPSEL_P_X + d];
      if (!(a.x[d] >= 0.0 && a.x[d] < b->pp.L[d])) return KAPSEL_ERANGE;
      a.v[d] = o[KAPSEL_P_V + d];
      a.omega[d] = o[KAPSEL_P_OMEGA + d];
      a.f_hydro_prev[d] = o[KAPSEL_P_FHYDRO + d];
      a.t_hydro_prev[d] = o[KAPSEL_P_THYDRO + d];
      a.fr_prev[d] = o[KAPSEL_P_FR + d];
      a.x_nopbc[d] = o[KAPSEL_P_XNOPBC + d];
      a.v_old[d] = o[KAPSEL_P_VOLD + d];
      a.omega_old[d] = o[KAPSEL_P_OMEGAOLD + d];
    }
    for (int i = 0; i < 4; ++i) {
      a.q[i] = o[KAPSEL_P_Q + i];
      a.q_old[i] = o[KAPSEL_P_QOLD + i];
    }
  }
  if (cudaMemcpyAsync(b->parts, h.data(), sizeof(DPart) * h.size(), cudaMemcpyHostToDevice, b->stream) !=
          cudaSuccess ||
      cudaMemsetAsync(b->status, 0, sizeof(int), b->stream) != cudaSuccess ||
      cudaStreamSynchronize(b->stream) != cudaSuccess)
    return KAPSEL_ECUDA;
  b->particles_set = true;
  return 0;
}

int kapsel_gpu_get_time(kapsel_ctx *ctx, int *ts, double *time) {
  if (!ctx) return KAPSEL_EINVAL;
  if (ts) *ts = ctx->box->ts;
  if (time) *time = ctx->box->time;
  return 0;
}

int kapsel_gpu_get_dims(kapsel_ctx *ctx, int *dims) {
  if (!ctx || !dims) return KAPSEL_EINVAL;
  const BoxBase *b = ctx->box.get();
  dims[0] = b->g.NX;
  dims[1] = b->g.NY;
  dims[2] = b->g.NZ;
  dims[3] = b->g.NZ + 2;
  dims[4] = b->Np;
  dims[5] = b->S;
  return 0;
}

int kapsel_gpu_set_efield(kapsel_ctx *ctx, const double *e) {
  if (!ctx || !e) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (b->prm.eq != KAPSEL_EQ_ELECTROLYTE) return KAPSEL_EINVAL;
  for (int d = 0; d < 3; ++d) b->prm.e_ext[d] = e[d];
  // the field enters the step as launch arguments: re-capture the graphs
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return KAPSEL_ECUDA;
  for (int s = 0; s < 2; ++s)
    if (b->graph[s]) {
      cudaGraphExecDestroy(b->graph[s]);
      b->graph[s] = nullptr;
    }
  return 0;
}

int kapsel_gpu_get_concentration(kapsel_ctx *ctx, double *c) {
  if (!ctx || !c) return KAPSEL_EINVAL;
  if (ctx->box->prm.eq != KAPSEL_EQ_ELECTROLYTE) return KAPSEL_ESTATE;
  return ctx->box->conc_to_host(c);
}

int kapsel_gpu_check_bounded_wait(void) {
  int *st = nullptr, h = 0;
  if (cudaMalloc(&st, sizeof(int)) != cudaSuccess) return KAPSEL_ENOMEM;
  int rc = 0;
  if (cudaMemset(st, 0, sizeof(int)) != cudaSuccess) rc = KAPSEL_ECUDA;
  if (!rc) {
    nc::k_wait_selfcheck<<<1, 32>>>(st);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpy(&h, st, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = KAPSEL_ECUDA;
  }
  cudaFree(st);
  return rc ? rc : h;
}

int kapsel_gpu_set_concentration(kapsel_ctx *ctx, const double *c, const double *total_solute) {
  if (!ctx || !c) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (b->prm.eq != KAPSEL_EQ_ELECTROLYTE) return KAPSEL_ESTATE;
  int rc = b->conc_from_host(c);
  if (rc || !total_solute) return rc;
  return b->total_solute_from_host(total_solute);
}

int kapsel_gpu_A2a_k(kapsel_ctx *ctx, double *a) {
  if (!ctx || !a) return KAPSEL_EINVAL;
  return ctx->box->fft_fwd_host(a);
}
int kapsel_gpu_A_k2a(kapsel_ctx *ctx, double *a) {
  if (!ctx || !a) return KAPSEL_EINVAL;
  return ctx->box->fft_inv_host(a);
}
int kapsel_gpu_solenoidal_u(kapsel_ctx *ctx, double *u0, double *u1, double *u2) {
  if (!ctx || !u0 || !u1 || !u2) return KAPSEL_EINVAL;
  return ctx->box->solenoidal_host(u0, u1, u2);
}
int kapsel_gpu_make_phi_u(kapsel_ctx *ctx, double *phi, double *up0, double *up1, double *up2) {
  if (!ctx || !phi || !up0 || !up1 || !up2) return KAPSEL_EINVAL;
  const int rc = ctx->box->phi_up_host(phi, up0, up1, up2);
  return rc ? rc : check_status(ctx->box.get());
}
int kapsel_gpu_calc_f_hydro(kapsel_ctx *ctx, const double *u0, const double *u1, const double *u2, double *f,
                            double *t) {
  if (!ctx || !u0 || !u1 || !u2 || !f || !t) return KAPSEL_EINVAL;
  return ctx->box->fhydro_host(u0, u1, u2, f, t);
}

// Force (particle_solver.h:97-109) without the hydrodynamic part, on a
// scratch copy of the particle state: the particle kernel runs with no
// Sekibun points and no thermostat, and fr_prev after its velocity update is
// the LJ (+ gravity when `gravity`) force of the current positions.
static int calc_fr_impl(kapsel_ctx *ctx, double *fr, bool gravity) {
  if (!ctx || !fr) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (b->Np == 0) return 0;
  DPart *scratch = nullptr;
  if (cudaMalloc(&scratch, sizeof(DPart) * b->Np) != cudaSuccess) return KAPSEL_ENOMEM;
  cudaMemcpyAsync(scratch, b->parts, sizeof(DPart) * b->Np, cudaMemcpyDeviceToDevice, b->stream);
  b->launch_cells();
  PPar p = b->pp;
  p.S = 0;           // no hydro gather
  p.thermostat = 0;  // no kick
  p.frozen = 0;
  if (!gravity) p.grav = 0.0;
  // u is never read with S == 0
  if (b->prm.precision == KAPSEL_FP64)
    k_particles_hydro_velocity<double><<<b->Np * p.hyd_pcl, p.hyd_threads, 0, b->stream>>>(p, scratch, nullptr, b->cells, nullptr, 1,
                                                                           b->status, b->partial_p, b->arrivals);
  else
    k_particles_hydro_velocity<float><<<b->Np * p.hyd_pcl, p.hyd_threads, 0, b->stream>>>(p, scratch, nullptr, b->cells, nullptr, 1,
                                                                          b->status, b->partial_p, b->arrivals);
  std::vector<DPart> h(b->Np);
  cudaMemcpyAsync(h.data(), scratch, sizeof(DPart) * b->Np, cudaMemcpyDeviceToHost, b->stream);
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return KAPSEL_ECUDA;
  cudaFree(scratch);
  for (int n = 0; n < b->Np; ++n)
    for (int d = 0; d < 3; ++d) fr[3 * n + d] = h[n].fr_prev[d];
  return 0;
}

int kapsel_gpu_calc_fr(kapsel_ctx *ctx, double *fr) { return calc_fr_impl(ctx, fr, true); }

int kapsel_gpu_calc_lj(kapsel_ctx *ctx, double *fr) { return calc_fr_impl(ctx, fr, false); }

int kapsel_gpu_make_phi(kapsel_ctx *ctx, double *phi) {
  if (!ctx || !phi) return KAPSEL_EINVAL;
  const int rc = ctx->box->phi_only_host(phi);
  return rc ? rc : check_status(ctx->box.get());
}

int kapsel_gpu_ns_slaved_euler(kapsel_ctx *ctx, double *zeta, const double *uk_dc) {
  if (!ctx || !zeta || !uk_dc) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  int rc = b->slaved_euler_host(zeta, uk_dc);
  if (rc) return rc;
  b->initialised = true;
  return check_status(b);
}

// The Electrolyte routines behind their reference names: the context must
// be an Electrolyte one; its particle state (kapsel_gpu_set_particle_state)
// gives the positions.
static int el_routine_ready(kapsel_ctx *ctx) {
  BoxBase *b = ctx->box.get();
  if (b->prm.eq != KAPSEL_EQ_ELECTROLYTE) return KAPSEL_ESTATE;
  if (b->Np > 0 && !b->particles_set) return KAPSEL_ESTATE;
  return 0;
}

int kapsel_gpu_ns_solute_euler(kapsel_ctx *ctx, double *zeta, const double *uk_dc, double *conc_k) {
  if (!ctx || !zeta || !uk_dc || !conc_k) return KAPSEL_EINVAL;
  int rc = el_routine_ready(ctx);
  if (rc) return rc;
  BoxBase *b = ctx->box.get();
  if ((rc = b->ns_solute_host(zeta, uk_dc, conc_k))) return rc;
  b->initialised = true;
  return check_status(b);
}

int kapsel_gpu_rescale_solute(kapsel_ctx *ctx, const double *total_solute, double *conc_k, double *rescale_factor) {
  if (!ctx || !total_solute || !conc_k || !rescale_factor) return KAPSEL_EINVAL;
  int rc = el_routine_ready(ctx);
  if (rc) return rc;
  if ((rc = ctx->box->rescale_solute_host(total_solute, conc_k, rescale_factor))) return rc;
  return check_status(ctx->box.get());
}

int kapsel_gpu_coulomb_force(kapsel_ctx *ctx, const double *conc_k, double *f0, double *f1, double *f2) {
  if (!ctx || !conc_k || !f0 || !f1 || !f2) return KAPSEL_EINVAL;
  int rc = el_routine_ready(ctx);
  if (rc) return rc;
  if ((rc = ctx->box->coulomb_force_host(conc_k, f0, f1, f2))) return rc;
  return check_status(ctx->box.get());
}

int kapsel_gpu_md_position(kapsel_ctx *ctx, int euler) {
  if (!ctx) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (b->Np == 0) return 0;
  if (!b->particles_set) return KAPSEL_ESTATE;
  PPar p = b->pp;
  p.frozen = 0;
  k_particles_position<<<(b->Np + 127) / 128, 128, 0, b->stream>>>(p, b->parts, euler ? 1 : 0, b->status);
  if (cudaGetLastError() != cudaSuccess) return KAPSEL_ECUDA;
  return check_status(b);
}

int kapsel_gpu_md_velocity(kapsel_ctx *ctx, const double *f_hydro, const double *torque_hydro, int euler) {
  // the particle kernel with no Sekibun points: the given hydrodynamic force
  // and torque enter through its per-particle correction input (added to an
  // empty gather), then Force, the velocity update and reset_Forces
  if (!ctx || (ctx->box->Np > 0 && (!f_hydro || !torque_hydro))) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (b->Np == 0) return 0;
  if (!b->particles_set) return KAPSEL_ESTATE;
  std::vector<double> h(6 * (size_t)b->Np);
  for (int n = 0; n < b->Np; ++n)
    for (int d = 0; d < 3; ++d) {
      h[6 * n + d] = f_hydro[3 * n + d];
      h[6 * n + 3 + d] = torque_hydro[3 * n + d];
    }
  double *corr = nullptr;
  if (cudaMalloc(&corr, sizeof(double) * h.size()) != cudaSuccess) return KAPSEL_ENOMEM;
  int rc = 0;
  if (cudaMemcpyAsync(corr, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice, b->stream) != cudaSuccess)
    rc = KAPSEL_ECUDA;
  b->launch_cells();
  PPar p = b->pp;
  p.S = 0;
  p.thermostat = 0;
  p.frozen = 0;
  if (!rc) {
    if (b->prm.precision == KAPSEL_FP64)
      k_particles_hydro_velocity<double><<<b->Np * p.hyd_pcl, p.hyd_threads, 0, b->stream>>>(
          p, b->parts, nullptr, b->cells, nullptr, euler ? 1 : 0, b->status, b->partial_p, b->arrivals, corr);
    else
      k_particles_hydro_velocity<float><<<b->Np * p.hyd_pcl, p.hyd_threads, 0, b->stream>>>(
          p, b->parts, nullptr, b->cells, nullptr, euler ? 1 : 0, b->status, b->partial_p, b->arrivals, corr);
    if (cudaGetLastError() != cudaSuccess) rc = KAPSEL_ECUDA;
  }
  if (!rc) rc = check_status(b);
  cudaFree(corr);
  return rc;
}

int kapsel_gpu_set_time(kapsel_ctx *ctx, int ts, double time) {
  if (!ctx || ts < 0) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return KAPSEL_ECUDA;
  // normals already drawn for the next step stay the next step's: the
  // thermostat stream does not move with the step counter
  const int oslot = b->ts & 1, nslot = ts & 1;
  const bool pending = b->noise_pre_ts[oslot] == b->ts;
  b->drop_prefill();
  if (pending) {
    if (nslot != oslot) {
      if (cudaMemcpyAsync(b->noise_dev[nslot], b->noise_dev[oslot], sizeof(double) * 6 * b->Np,
                          cudaMemcpyDeviceToDevice, b->stream) != cudaSuccess ||
          cudaEventRecord(b->noise_ev[nslot], b->stream) != cudaSuccess ||
          cudaStreamSynchronize(b->stream) != cudaSuccess)
        return KAPSEL_ECUDA;
    }
    b->noise_pre_ts[nslot] = ts;
  }
  b->ts = ts;
  b->time = time;
  return 0;
}

static const char *kKernelNames[KAPSEL_N_STEP_KERNELS] = {
    "k_x_zeta_to_u",        "k_y_pass<inv>",        "k_z_products",       "k_y_pass<fwd>",
    "k_x_advect_update",    "k_y_pass<inv>",        "k_z_c2r",            "k_particles_position",
    "k_particles_hydro_velocity", "k_particles_scatter", "k_z_force",       "k_y_pass<fwd>",
    "k_x_force_to_zeta"};

int kapsel_thermostat_normals(unsigned int seed, long long skip, long long n, double *out) {
  // n normals of the reference thermostat stream: Gauss2 pairs from MT19937
  // seeded with init_genrand(seed), after `skip` normals (skip even).
  if (!out || n < 0 || skip < 0 || (skip & 1) || (n & 1)) return KAPSEL_EINVAL;
  MT19937 mt(seed);
  double pair[2];
  for (long long i = 0; i < skip; i += 2) mt.gauss2(pair);
  for (long long i = 0; i < n; i += 2) mt.gauss2(out + i);
  return 0;
}

int kapsel_sekibun_cells(double a, double a_xi, double dx, int *out, int cap) {
  if (!(a > 0.0) || !(a_xi > 0.0) || !(dx > 0.0)) return KAPSEL_EINVAL;
  std::vector<int> c = sekibun(a, a_xi, dx);
  const int n = (int)c.size() / 3;
  if (out) {
    if (cap < n) return KAPSEL_ERANGE;
    memcpy(out, c.data(), sizeof(int) * c.size());
  }
  return n;
}

int kapsel_gpu_get_stream(kapsel_ctx *ctx, void **stream) {
  if (!ctx || !stream) return KAPSEL_EINVAL;
  *stream = (void *)ctx->box->stream;
  return 0;
}

int kapsel_gpu_get_oblique(kapsel_ctx *ctx, double *out) {
  if (!ctx || !out || ctx->box->prm.eq != KAPSEL_EQ_SHEAR_LE) return KAPSEL_EINVAL;
  double h[4];
  const int rc = ctx->box->oblique_state(h);
  if (rc) return rc;
  out[0] = h[OB_DEG];
  out[1] = h[OB_SRATE];
  out[2] = h[OB_STRAIN];
  return 0;
}

int kapsel_gpu_set_oblique(kapsel_ctx *ctx, double degree_oblique, double shear_rate_eff) {
  if (!ctx || ctx->box->prm.eq != KAPSEL_EQ_SHEAR_LE || !std::isfinite(degree_oblique) ||
      !std::isfinite(shear_rate_eff))
    return KAPSEL_EINVAL;
  return ctx->box->set_oblique_state(degree_oblique, shear_rate_eff);
}

int kapsel_gpu_launches_per_step(kapsel_ctx *ctx) {
  if (!ctx) return KAPSEL_EINVAL;
  // Counted, not assumed: capture one step into a throwaway graph (nothing
  // runs) and count its kernel nodes.
  BoxBase *b = ctx->box.get();
  if (!b->initialised) return KAPSEL_ESTATE;
  cudaGraph_t gr = nullptr;
  if (cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return KAPSEL_ECUDA;
  b->launch_step(b->noise_dev[0], 0);
  if (cudaStreamEndCapture(b->stream, &gr) != cudaSuccess || !gr) return KAPSEL_ECUDA;
  size_t nn = 0;
  cudaGraphGetNodes(gr, nullptr, &nn);
  std::vector<cudaGraphNode_t> nodes(nn);
  if (nn) cudaGraphGetNodes(gr, nodes.data(), &nn);
  int nk = 0;
  for (size_t i = 0; i < nn; ++i) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++nk;
  }
  cudaGraphDestroy(gr);
  return nk;
}

const char *kapsel_gpu_kernel_name(int i) {
  return (i >= 0 && i < KAPSEL_N_STEP_KERNELS) ? kKernelNames[i] : "";
}

const char *kapsel_gpu_step_kernel_name(kapsel_ctx *ctx, int i) {
  if (i < 0 || i >= KAPSEL_N_STEP_KERNELS) return "";
  if (ctx && ctx->box->fused_yz()) {
    if (i == 5 || i == 11) return "";  // y passes inside the fused launches
    if (i == 6) return "k_yzw_c2r";
    if (i == 10) return "k_zyw_force";
  }
  return kKernelNames[i];
}

int kapsel_gpu_profile_step(kapsel_ctx *ctx, float *ms) {
  // A short timed gate kernel holds the stream while the host enqueues the
  // step with an event between consecutive launches, so on the device the
  // launches run back to back and each event delta is one kernel's duration
  // (not a host launch gap).
  if (!ctx || !ms) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (!b->initialised) return KAPSEL_ESTATE;
  const int slot = b->ts & 1;
  int rc = b->take_noise(slot);
  if (rc) return rc;
  cudaEvent_t ev[KAPSEL_N_STEP_KERNELS + 1];
  for (int i = 0; i <= KAPSEL_N_STEP_KERNELS; ++i)
    if (cudaEventCreate(&ev[i]) != cudaSuccess) return KAPSEL_ECUDA;
  k_time_gate<<<1, 32, 0, b->stream>>>(2000000ull);  // 2 ms
  b->launch_step(b->noise_dev[slot], b->ts == 0 ? 1 : 0, ev);
  b->u_spec_ready = false;
  b->ts += 1;
  b->time += b->prm.dt;
  if (cudaStreamSynchronize(b->stream) != cudaSuccess) return KAPSEL_ECUDA;
  const int nk = b->Np > 0 ? KAPSEL_N_STEP_KERNELS : 7;
  for (int i = 0; i < KAPSEL_N_STEP_KERNELS; ++i) ms[i] = 0.f;
  for (int i = 0; i < nk; ++i)
    if (cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]) != cudaSuccess) return KAPSEL_ECUDA;
  for (int i = 0; i <= KAPSEL_N_STEP_KERNELS; ++i) cudaEventDestroy(ev[i]);
  return check_status(b);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched ensemble: independent boxes advanced together, one CUDA graph
// launch per step.  The graph forks from a root stream to every box's stream,
// runs each box's step sequence as a parallel branch, and joins back.
struct kapsel_batch {
  std::vector<kapsel_ctx *> boxes;
  cudaStream_t root = nullptr;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  cudaEvent_t fork = nullptr, done = nullptr;
  std::vector<cudaEvent_t> ready, join;
  std::vector<std::vector<double>> x0;
  // the autotuner's choices: NX, NY, NZ, z variant, y variant, x split per shape
  std::vector<std::vector<int>> variants;
};

extern "C" {

int kapsel_batch_create(kapsel_ctx *const *boxes, int n, int autotune, kapsel_batch **out) {
  if (!boxes || n <= 0 || !out) return KAPSEL_EINVAL;
  *out = nullptr;
  std::unique_ptr<kapsel_batch> b(new (std::nothrow) kapsel_batch);
  if (!b) return KAPSEL_ENOMEM;
  const int ts0 = boxes[0]->box->ts;
  for (int i = 0; i < n; ++i) {
    if (!boxes[i] || !boxes[i]->box->initialised || boxes[i]->box->ts != ts0) return KAPSEL_ESTATE;
    b->boxes.push_back(boxes[i]);
  }
  if (cudaStreamCreateWithFlags(&b->root, cudaStreamNonBlocking) != cudaSuccess) return KAPSEL_ECUDA;
  if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) return KAPSEL_ECUDA;
  if (cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess) return KAPSEL_ECUDA;
  b->ready.resize(n);
  b->join.resize(n);
  for (int i = 0; i < n; ++i) {
    if (cudaEventCreateWithFlags(&b->ready[i], cudaEventDisableTiming) != cudaSuccess) return KAPSEL_ECUDA;
    if (cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming) != cudaSuccess) return KAPSEL_ECUDA;
  }
  // autotune: per box shape (and precision, particle count class), the z and
  // y pass variants, by timing whole steps of the first box of that shape on
  // a copy of its state
  if (autotune) {
    // per shape: {z variant, y variant, x radix split}
    std::vector<std::pair<std::vector<int>, std::vector<int>>> chosen;
    for (int i = 0; i < n; ++i) {
      BoxBase *x = b->boxes[i]->box.get();
      if (x->prm.eq != KAPSEL_EQ_NAVIER_STOKES || x->Np == 0) continue;
      std::vector<int> key = {x->g.NX, x->g.NY, x->g.NZ, x->prm.precision, x->Np > 1024 ? 1 : 0};
      int zp = -1, yp = -1, xp = 0;
      for (auto &c : chosen)
        if (c.first == key) zp = c.second[0], yp = c.second[1], xp = c.second[2];
      if (zp < 0) {
        float best = 0.f;
        for (int xs = 0; xs < 2; ++xs) {
          if (!x->xsplit_ok(xs)) continue;
          x->set_xsplit(xs);
          for (int zm = 0; zm < 2; ++zm)
            for (int ym = 0; ym < 4; ++ym) {
              if (!x->variant_ok(zm, ym)) continue;
              const float t = x->time_variant(zm, ym, 5);
              if (t > 0.f && (zp < 0 || t < best)) best = t, zp = zm, yp = ym, xp = xs;
            }
        }
        if (zp < 0) {
          x->set_xsplit(0);
          continue;
        }
        chosen.push_back({key, {zp, yp, xp}});
      }
      x->set_xsplit(xp);
      x->set_variant(zp, yp);
    }
    b->variants.clear();
    for (auto &c : chosen)
      b->variants.push_back({c.first[0], c.first[1], c.first[2], c.second[0], c.second[1], c.second[2]});
  }
  // initial unwrapped positions for the mean-square displacement
  for (int i = 0; i < n; ++i) {
    BoxBase *x = b->boxes[i]->box.get();
    std::vector<double> rec((size_t)KAPSEL_P_STRIDE * std::max(x->Np, 1));
    int rc = kapsel_gpu_get_particles(b->boxes[i], rec.data());
    if (rc) return rc;
    std::vector<double> p0(3 * (size_t)x->Np);
    for (int m = 0; m < x->Np; ++m)
      for (int d = 0; d < 3; ++d) p0[3 * m + d] = rec[(size_t)KAPSEL_P_STRIDE * m + KAPSEL_P_XNOPBC + d];
    b->x0.push_back(p0);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return KAPSEL_ECUDA;
  *out = b.release();
  return 0;
}

int kapsel_batch_step(kapsel_batch *b, int nsteps) {
  if (!b || nsteps < 0) return KAPSEL_EINVAL;
  const int n = (int)b->boxes.size();
  for (int s = 0; s < nsteps; ++s) {
    BoxBase *first = b->boxes[0]->box.get();
    const int slot = first->ts & 1;
    const int euler = first->ts == 0 ? 1 : 0;
    for (int i = 0; i < n; ++i) {
      BoxBase *x = b->boxes[i]->box.get();
      int rc = x->take_noise(slot);
      if (rc) return rc;
      x->ensure_u_spec();  // on the box's stream, before the graph's ready events
    }
    if (euler) {
      for (int i = 0; i < n; ++i) {
        BoxBase *x = b->boxes[i]->box.get();
        x->launch_step(x->noise_dev[slot], 1);
      }
    } else {
      if (!b->graph[slot]) {
        cudaGraph_t gr;
        if (cudaStreamBeginCapture(b->root, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return KAPSEL_ECUDA;
        cudaEventRecord(b->fork, b->root);
        for (int i = 0; i < n; ++i) {
          BoxBase *x = b->boxes[i]->box.get();
          cudaStreamWaitEvent(x->stream, b->fork, 0);
          x->launch_step(x->noise_dev[slot], 0);
          cudaEventRecord(b->join[i], x->stream);
          cudaStreamWaitEvent(b->root, b->join[i], 0);
        }
        if (cudaStreamEndCapture(b->root, &gr) != cudaSuccess) return KAPSEL_ECUDA;
        if (cudaGraphInstantiate(&b->graph[slot], gr, 0) != cudaSuccess) return KAPSEL_ECUDA;
        cudaGraphDestroy(gr);
      }
      // the graph reads each box's freshly copied noise: wait for the copies
      for (int i = 0; i < n; ++i) {
        BoxBase *x = b->boxes[i]->box.get();
        cudaEventRecord(b->ready[i], x->stream);
        cudaStreamWaitEvent(b->root, b->ready[i], 0);
      }
      if (cudaGraphLaunch(b->graph[slot], b->root) != cudaSuccess) return KAPSEL_ECUDA;
      // later work on the box streams (the next noise copies) follows the graph
      cudaEventRecord(b->done, b->root);
      for (int i = 0; i < n; ++i) cudaStreamWaitEvent(b->boxes[i]->box->stream, b->done, 0);
    }
    for (int i = 0; i < n; ++i) {
      BoxBase *x = b->boxes[i]->box.get();
      x->u_spec_ready = x->ends_with_u_spec();
      x->ts += 1;
      x->time += x->prm.dt;
    }
  }
  if (cudaStreamSynchronize(b->root) != cudaSuccess) return KAPSEL_ECUDA;
  for (int i = 0; i < n; ++i) {
    int rc = check_status(b->boxes[i]->box.get());
    if (rc) return rc;
  }
  return 0;
}

int kapsel_batch_msd(kapsel_batch *b, double *msd) {
  // mean over the particles of each box of |x_nopbc(t) - x_nopbc(t0)|^2
  // (the unwrapped R_raw of Output_udf, avs_output.cxx:361-363)
  if (!b || !msd) return KAPSEL_EINVAL;
  for (size_t i = 0; i < b->boxes.size(); ++i) {
    BoxBase *x = b->boxes[i]->box.get();
    std::vector<double> rec((size_t)KAPSEL_P_STRIDE * std::max(x->Np, 1));
    int rc = kapsel_gpu_get_particles(b->boxes[i], rec.data());
    if (rc) return rc;
    double acc = 0.0;
    for (int m = 0; m < x->Np; ++m)
      for (int d = 0; d < 3; ++d) {
        const double dd = rec[(size_t)KAPSEL_P_STRIDE * m + KAPSEL_P_XNOPBC + d] - b->x0[i][3 * m + d];
        acc += dd * dd;
      }
    msd[i] = x->Np > 0 ? acc / x->Np : 0.0;
  }
  return 0;
}

int kapsel_gpu_set_x_split(kapsel_ctx *ctx, int split) {
  if (!ctx) return KAPSEL_EINVAL;
  BoxBase *x = ctx->box.get();
  if (!x->xsplit_ok(split)) return KAPSEL_EINVAL;
  if (cudaStreamSynchronize(x->stream) != cudaSuccess) return KAPSEL_ECUDA;
  x->set_xsplit(split);
  return 0;
}

int kapsel_gpu_set_pass_variant(kapsel_ctx *ctx, int zmode, int ymode) {
  if (!ctx) return KAPSEL_EINVAL;
  BoxBase *x = ctx->box.get();
  if (!x->variant_ok(zmode, ymode)) return KAPSEL_EINVAL;
  if (cudaStreamSynchronize(x->stream) != cudaSuccess) return KAPSEL_ECUDA;
  x->set_variant(zmode, ymode);
  x->u_spec_ready = false;
  return 0;
}

int kapsel_batch_variants(kapsel_batch *b, int *out, int cap) {
  if (!b || cap < 0 || (cap > 0 && !out)) return KAPSEL_EINVAL;
  const int n = (int)b->variants.size();
  for (int i = 0; i < n && i < cap; ++i)
    for (int k = 0; k < 6; ++k) out[6 * i + k] = b->variants[i][k];
  return n;
}

int kapsel_batch_get_stream(kapsel_batch *b, void **stream) {
  if (!b || !stream) return KAPSEL_EINVAL;
  *stream = (void *)b->root;
  return 0;
}

int kapsel_batch_destroy(kapsel_batch *b) {
  if (!b) return KAPSEL_EINVAL;
  cudaStreamSynchronize(b->root);
  for (int s = 0; s < 2; ++s)
    if (b->graph[s]) cudaGraphExecDestroy(b->graph[s]);
  for (auto e : b->ready) cudaEventDestroy(e);
  for (auto e : b->join) cudaEventDestroy(e);
  cudaEventDestroy(b->fork);
  cudaEventDestroy(b->done);
  cudaStreamDestroy(b->root);
  delete b;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free Solenoidal_u on device arrays.
//
// Some callers cannot allocate device memory: code that runs while another
// component owns every allocation (a fixed memory pool or a host program
// whose allocator is not CUDA-aware), or code that must not call cudaMalloc
// because that call can synchronise the device or fail under memory
// pressure in the middle of a time step.  For them this entry point does the
// 2/3-truncated solenoidal projection of three real fields without
// allocating: its three spectra and its twiddle tables live in one
// file-scope device array of fixed size, which every GPU that loads this
// library holds until the process exits.
namespace {

// Largest grid the static scratch holds: NX*NY*(NZ/2+1) <= 64*64*33 complex
// values per component (any axis 16..128), i.e. 64^3 or an equal-size box.
constexpr size_t kNoAllocMaxModes = 64 * 64 * 33;
constexpr size_t kNoAllocMaxTwiddles = 128 + 128 + 64 + 128;
constexpr size_t kNoAllocScratchDoubles = 2 * (3 * kNoAllocMaxModes + kNoAllocMaxTwiddles);

static __device__ __align__(256) double kNoAllocScratch[kNoAllocScratchDoubles];

// The host-side name of kNoAllocScratch is only a stand-in for the device
// array; its device address comes from cudaGetSymbolAddress, looked up once
// per device with that device current and then reused.
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[kNoAllocMaxDevices] = {};

int noalloc_scratch(void **out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) return KAPSEL_ECUDA;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, kNoAllocScratch) != cudaSuccess || !p) return KAPSEL_ECUDA;
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return 0;
}

__global__ void k_noalloc_twiddles(Cx<double> *tw, int nx, int ny, int m, int nz) {
  const int n[4] = {nx, ny, m, nz};
  int off = 0;
  for (int t = 0; t < 4; ++t) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n[t]; j += gridDim.x * blockDim.x) {
      double s, c;
      sincospi(2.0 * (double)j / (double)n[t], &s, &c);
      tw[off + j] = {c, s};
    }
    off += n[t];
  }
}

}  // namespace

extern "C" int kapsel_gpu_solenoidal_u_noalloc(const int *np_xyz, double dx, const double *u0, const double *u1,
                                               const double *u2, double *o0, double *o1, double *o2, void *stream) {
  if (!np_xyz || !u0 || !u1 || !u2 || !o0 || !o1 || !o2 || !(dx > 0.0)) return KAPSEL_EINVAL;
  for (int d = 0; d < 3; ++d)
    if (np_xyz[d] < 4 || np_xyz[d] > 7) return KAPSEL_ERANGE;  // each axis 16..128
  Geo g;
  memset(&g, 0, sizeof(g));
  g.NX = 1 << np_xyz[0];
  g.NY = 1 << np_xyz[1];
  g.NZ = 1 << np_xyz[2];
  g.M = g.NZ / 2;
  const size_t modes = (size_t)g.NX * g.NY * (g.M + 1);
  if (modes > kNoAllocMaxModes) return KAPSEL_ERANGE;
  g.lx = ilog2(g.NX);
  g.ly = ilog2(g.NY);
  g.lm = ilog2(g.M);
  g.TX = (g.NX + 2) / 3;
  g.TY = (g.NY + 2) / 3;
  g.TZ = (g.NZ + 2) / 3;
  g.TS = (g.TZ + 3) & ~3;
  g.KXc = 2 * g.TX - 1;
  g.KYc = 2 * g.TY - 1;
  g.wave[0] = 2.0 * M_PI / (g.NX * dx);
  g.wave[1] = 2.0 * M_PI / (g.NY * dx);
  g.wave[2] = 2.0 * M_PI / (g.NZ * dx);
  g.inv_n = 1.0 / ((double)g.NX * g.NY * g.NZ);
  // an error left on this thread by earlier, unrelated work is not this
  // call's: report it without launching anything and leave it for its owner
  if (cudaPeekAtLastError() != cudaSuccess) return KAPSEL_ECUDA;
  void *base = nullptr;
  int rc = noalloc_scratch(&base);
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  Cx<double> *spec = reinterpret_cast<Cx<double> *>(base);
  Cx<double> *twb = spec + 3 * kNoAllocMaxModes;
  // the tables are rewritten on every call (the previous call may have used
  // another grid); the spectra need no clearing: the forward transform
  // writes every entry before anything reads it
  k_noalloc_twiddles<<<2, 128, 0, s>>>(twb, g.NX, g.NY, g.M, g.NZ);
  Twiddles<double> tw;
  tw.x = twb;
  tw.y = twb + g.NX;
  tw.m = twb + g.NX + g.NY;
  tw.z = twb + g.NX + g.NY + g.M;
  const int M1 = g.M + 1;
  const int gz = (g.NX * g.NY) / ZROWS;
  const size_t sm_z = sizeof(Cx<double>) * (g.M + g.NZ + (size_t)2 * g.M * ZROWS + (size_t)ZROWS * (g.M + 1));
  auto col = [&](Cx<double> *data, bool inv, int axis) {
    const int n = axis == 0 ? g.NX : g.NY;
    const int logn = axis == 0 ? g.lx : g.ly;
    const Cx<double> *twn = axis == 0 ? tw.x : tw.y;
    const size_t sm = sizeof(Cx<double>) * (n + (size_t)n * 16);
    // axis 0 (x): lines (y, kz) contiguous, element stride NY*M1; axis 1 (y):
    // lines (x, kz), kz contiguous within each x-plane, element stride M1
    const int nl = axis == 0 ? g.NY * M1 : g.NX * M1;
    const int lpp = axis == 0 ? nl : M1;
    const long long es = axis == 0 ? (long long)g.NY * M1 : M1, ps = axis == 0 ? 0 : (long long)g.NY * M1;
    if (inv)
      k_col_pass<double, true><<<(nl + 15) / 16, 256, sm, s>>>(g, twn, logn, n, data, data, 1, es, nl, lpp, ps);
    else
      k_col_pass<double, false><<<(nl + 15) / 16, 256, sm, s>>>(g, twn, logn, n, data, data, 1, es, nl, lpp, ps);
  };
  const double *in[3] = {u0, u1, u2};
  double *out[3] = {o0, o1, o2};
  for (int c = 0; c < 3; ++c) {
    Cx<double> *sc = spec + c * modes;
    k_z_r2c_full<double><<<gz, 256, sm_z, s>>>(g, tw, in[c], g.NZ, sc);
    col(sc, false, 1);
    col(sc, false, 0);
  }
  k_solenoidal_full<double><<<592, 256, 0, s>>>(g, spec, spec + modes, spec + 2 * modes);
  for (int c = 0; c < 3; ++c) {
    Cx<double> *sc = spec + c * modes;
    col(sc, true, 0);
    col(sc, true, 1);
    k_z_c2r_full<double><<<gz, 256, sm_z, s>>>(g, tw, sc, out[c], g.inv_n);
  }
  if (cudaGetLastError() != cudaSuccess) return KAPSEL_ECUDA;
  return 0;
}

// ---------------------------------------------------------------------------
// Learned near-contact correction: C ABI (no counterpart in the reference).
extern "C" {

int kapsel_nc_create(const float *params, kapsel_nc **out) {
  if (!params || !out) return KAPSEL_EINVAL;
  *out = nullptr;
  int rc = nc_smem_setup();
  if (rc) return rc;
  std::unique_ptr<kapsel_nc> h(new (std::nothrow) kapsel_nc());
  if (!h) return KAPSEL_ENOMEM;
  const size_t nb = sizeof(float) * nc::NPARAM;
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess) return KAPSEL_ECUDA;
  if (cudaMalloc(&h->params, nb) != cudaSuccess || cudaMalloc(&h->grad, nb) != cudaSuccess ||
      cudaMalloc(&h->m, nb) != cudaSuccess || cudaMalloc(&h->v, nb) != cudaSuccess ||
      cudaMalloc(&h->loss, sizeof(float)) != cudaSuccess || cudaMalloc(&h->status, sizeof(int)) != cudaSuccess)
    return KAPSEL_ENOMEM;
  KCHECK(cudaMemcpyAsync(h->params, params, nb, cudaMemcpyHostToDevice, h->stream));
  KCHECK(cudaMemsetAsync(h->grad, 0, nb, h->stream));
  KCHECK(cudaMemsetAsync(h->m, 0, nb, h->stream));
  KCHECK(cudaMemsetAsync(h->v, 0, nb, h->stream));
  KCHECK(cudaMemsetAsync(h->status, 0, sizeof(int), h->stream));
  KCHECK(cudaStreamSynchronize(h->stream));
  *out = h.release();
  return 0;
}

int kapsel_nc_destroy(kapsel_nc *nc) {
  if (!nc) return KAPSEL_EINVAL;
  cudaStreamSynchronize(nc->stream);
  cudaFree(nc->params);
  cudaFree(nc->grad);
  cudaFree(nc->m);
  cudaFree(nc->v);
  cudaFree(nc->loss);
  cudaFree(nc->status);
  cudaStreamDestroy(nc->stream);
  delete nc;
  return 0;
}

int kapsel_nc_get_params(kapsel_nc *nc, float *params) {
  if (!nc || !params) return KAPSEL_EINVAL;
  KCHECK(cudaMemcpyAsync(params, nc->params, sizeof(float) * nc::NPARAM, cudaMemcpyDeviceToHost, nc->stream));
  KCHECK(cudaStreamSynchronize(nc->stream));
  return 0;
}

int kapsel_nc_set_params(kapsel_nc *nc, const float *params) {
  if (!nc || !params) return KAPSEL_EINVAL;
  KCHECK(cudaMemcpyAsync(nc->params, params, sizeof(float) * nc::NPARAM, cudaMemcpyHostToDevice, nc->stream));
  KCHECK(cudaStreamSynchronize(nc->stream));
  return 0;
}

static int nc_status(kapsel_nc *nc) {
  int st = 0;
  KCHECK(cudaMemcpyAsync(&st, nc->status, sizeof(int), cudaMemcpyDeviceToHost, nc->stream));
  KCHECK(cudaStreamSynchronize(nc->stream));
  if (st) {
    cudaMemsetAsync(nc->status, 0, sizeof(int), nc->stream);
    cudaStreamSynchronize(nc->stream);
  }
  return st;
}

int kapsel_nc_forward(kapsel_nc *nc, const float *x, int n, float *y) {
  if (!nc || !x || !y || n < 0) return KAPSEL_EINVAL;
  if (n == 0) return 0;
  float *dx = nullptr, *dy = nullptr;
  if (cudaMallocAsync(&dx, sizeof(float) * nc::IN * n, nc->stream) != cudaSuccess ||
      cudaMallocAsync(&dy, sizeof(float) * nc::OUT * n, nc->stream) != cudaSuccess)
    return KAPSEL_ENOMEM;
  KCHECK(cudaMemcpyAsync(dx, x, sizeof(float) * nc::IN * n, cudaMemcpyHostToDevice, nc->stream));
  nc::TileIO io{};
  io.x = dx;
  io.n = n;
  io.out = dy;
  io.status = nc->status;
  nc::k_mlp_tile<false><<<(n + nc::TILE - 1) / nc::TILE, 256, nc::SMEM_ALLOC, nc->stream>>>(nc->params, io);
  KCHECK(cudaGetLastError());
  KCHECK(cudaMemcpyAsync(y, dy, sizeof(float) * nc::OUT * n, cudaMemcpyDeviceToHost, nc->stream));
  cudaFreeAsync(dx, nc->stream);
  cudaFreeAsync(dy, nc->stream);
  KCHECK(cudaStreamSynchronize(nc->stream));
  return nc_status(nc);
}

int kapsel_nc_gradient(kapsel_nc *nc, const float *x, const float *y, const float *colw, int n, float *grad,
                       float *loss) {
  if (!nc || !x || !y || !colw || !grad || !loss || n <= 0) return KAPSEL_EINVAL;
  float *dx = nullptr, *dy = nullptr, *dw = nullptr;
  if (cudaMallocAsync(&dx, sizeof(float) * nc::IN * n, nc->stream) != cudaSuccess ||
      cudaMallocAsync(&dy, sizeof(float) * nc::OUT * n, nc->stream) != cudaSuccess ||
      cudaMallocAsync(&dw, sizeof(float) * nc::OUT, nc->stream) != cudaSuccess)
    return KAPSEL_ENOMEM;
  KCHECK(cudaMemcpyAsync(dx, x, sizeof(float) * nc::IN * n, cudaMemcpyHostToDevice, nc->stream));
  KCHECK(cudaMemcpyAsync(dy, y, sizeof(float) * nc::OUT * n, cudaMemcpyHostToDevice, nc->stream));
  KCHECK(cudaMemcpyAsync(dw, colw, sizeof(float) * nc::OUT, cudaMemcpyHostToDevice, nc->stream));
  KCHECK(cudaMemsetAsync(nc->grad, 0, sizeof(float) * nc::NPARAM, nc->stream));
  KCHECK(cudaMemsetAsync(nc->loss, 0, sizeof(float), nc->stream));
  nc::TileIO io{};
  io.x = dx;
  io.y = dy;
  io.colw = dw;
  io.n = n;
  io.grad = nc->grad;
  io.loss = nc->loss;
  io.inv_n = 1.0f / (float)n;
  io.status = nc->status;
  nc::k_mlp_tile<true><<<(n + nc::TILE - 1) / nc::TILE, 128, nc::SMEM_ALLOC, nc->stream>>>(nc->params, io);
  KCHECK(cudaGetLastError());
  KCHECK(cudaMemcpyAsync(grad, nc->grad, sizeof(float) * nc::NPARAM, cudaMemcpyDeviceToHost, nc->stream));
  KCHECK(cudaMemcpyAsync(loss, nc->loss, sizeof(float), cudaMemcpyDeviceToHost, nc->stream));
  KCHECK(cudaMemsetAsync(nc->grad, 0, sizeof(float) * nc::NPARAM, nc->stream));
  cudaFreeAsync(dx, nc->stream);
  cudaFreeAsync(dy, nc->stream);
  cudaFreeAsync(dw, nc->stream);
  KCHECK(cudaStreamSynchronize(nc->stream));
  return nc_status(nc);
}

int kapsel_nc_train(kapsel_nc *nc, const float *x, const float *y, const float *colw, int n, int epochs, int batch,
                    float lr, unsigned int seed, float *loss_per_epoch) {
  if (!nc || !x || !y || !colw || n <= 0 || epochs <= 0 || batch <= 0 || !(lr > 0.f)) return KAPSEL_EINVAL;
  float *dx = nullptr, *dy = nullptr, *dw = nullptr;
  int *didx = nullptr;
  if (cudaMallocAsync(&dx, sizeof(float) * nc::IN * n, nc->stream) != cudaSuccess ||
      cudaMallocAsync(&dy, sizeof(float) * nc::OUT * n, nc->stream) != cudaSuccess ||
      cudaMallocAsync(&dw, sizeof(float) * nc::OUT, nc->stream) != cudaSuccess ||
      cudaMallocAsync(&didx, sizeof(int) * n * (size_t)epochs, nc->stream) != cudaSuccess)
    return KAPSEL_ENOMEM;
  KCHECK(cudaMemcpyAsync(dx, x, sizeof(float) * nc::IN * n, cudaMemcpyHostToDevice, nc->stream));
  KCHECK(cudaMemcpyAsync(dy, y, sizeof(float) * nc::OUT * n, cudaMemcpyHostToDevice, nc->stream));
  KCHECK(cudaMemcpyAsync(dw, colw, sizeof(float) * nc::OUT, cudaMemcpyHostToDevice, nc->stream));
  // one permutation per epoch (MT19937 stream of `seed`, Fisher-Yates)
  std::vector<int> perm((size_t)n * epochs);
  MT19937 mt(seed);
  for (int e = 0; e < epochs; ++e) {
    int *pe = perm.data() + (size_t)e * n;
    for (int i = 0; i < n; ++i) pe[i] = i;
    for (int i = n - 1; i > 0; --i) {
      const int j = (int)(mt.real3() * (i + 1));
      std::swap(pe[i], pe[j < i ? j : i]);
    }
  }
  KCHECK(cudaMemcpyAsync(didx, perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice, nc->stream));
  KCHECK(cudaMemsetAsync(nc->grad, 0, sizeof(float) * nc::NPARAM, nc->stream));
  std::vector<float> el(epochs, 0.f);
  const int nbatch = (n + batch - 1) / batch;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int e = 0; e < epochs; ++e) {
    KCHECK(cudaMemsetAsync(nc->loss, 0, sizeof(float), nc->stream));
    for (int b = 0; b < nbatch; ++b) {
      const int r0 = b * batch, nb = std::min(batch, n - r0);
      nc::TileIO io{};
      io.x = dx;
      io.y = dy;
      io.colw = dw;
      io.idx = didx + (size_t)e * n + r0;
      io.n = nb;
      io.grad = nc->grad;
      io.loss = nc->loss;
      io.inv_n = 1.0f / (float)nb;
      io.status = nc->status;
      nc::k_mlp_tile<true><<<(nb + nc::TILE - 1) / nc::TILE, 128, nc::SMEM_ALLOC, nc->stream>>>(nc->params, io);
      nc->adam_t += 1;
      const float c1 = 1.0f / (1.0f - powf(b1, (float)nc->adam_t)), c2 = 1.0f / (1.0f - powf(b2, (float)nc->adam_t));
      nc::k_adam<<<(nc::NPARAM + 255) / 256, 256, 0, nc->stream>>>(nc->params, nc->grad, nc->m, nc->v, nc::NPARAM,
                                                                   lr, b1, b2, eps, c1, c2);
    }
    KCHECK(cudaGetLastError());
    KCHECK(cudaMemcpyAsync(&el[e], nc->loss, sizeof(float), cudaMemcpyDeviceToHost, nc->stream));
  }
  cudaFreeAsync(dx, nc->stream);
  cudaFreeAsync(dy, nc->stream);
  cudaFreeAsync(dw, nc->stream);
  cudaFreeAsync(didx, nc->stream);
  KCHECK(cudaStreamSynchronize(nc->stream));
  if (loss_per_epoch)
    for (int e = 0; e < epochs; ++e) loss_per_epoch[e] = el[e] / (float)nbatch;
  return nc_status(nc);
}

int kapsel_nc_set_scaling(kapsel_nc *nc, const float *in_shift, const float *in_scale, const float *out_scale,
                          double a, double gap_lo, double gap_hi) {
  if (!nc || !in_shift || !in_scale || !out_scale || !(a > 0.0) || !(gap_lo > 0.0) || !(gap_hi > gap_lo))
    return KAPSEL_EINVAL;
  for (int i = 0; i < nc::IN; ++i) {
    nc->sc.in_shift[i] = in_shift[i];
    nc->sc.in_scale[i] = in_scale[i];
  }
  for (int i = 0; i < nc::OUT; ++i) nc->sc.out_scale[i] = out_scale[i];
  nc->sc.a = a;
  nc->sc.gap_lo = gap_lo;
  nc->sc.gap_hi = gap_hi;
  nc->scaled = true;
  return 0;
}

int kapsel_nc_pair_features(const kapsel_nc *nc, const double *rec_i, const double *rec_j, const double *box,
                            float *feat, float *frame, double *gap) {
  if (!nc || !nc->scaled || !rec_i || !rec_j || !box || !feat) return KAPSEL_EINVAL;
  double d[3];
  for (int k = 0; k < 3; ++k) {
    d[k] = rec_j[KAPSEL_P_X + k] - rec_i[KAPSEL_P_X + k];
    const double q = d[k] / box[k];
    d[k] -= (q >= 0.0 ? (double)(long long)(q + 0.5) : (double)(long long)(q - 0.5)) * box[k];
  }
  const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  const double h = r - 2.0 * nc->sc.a;
  if (gap) *gap = h;
  if (!(h > 0.0)) return KAPSEL_ERANGE;
  double e[9];
  nc::nc_frame(d, e);
  nc::nc_features(nc->sc, h, e, rec_i + KAPSEL_P_V, rec_j + KAPSEL_P_V, rec_i + KAPSEL_P_OMEGA,
                  rec_j + KAPSEL_P_OMEGA, feat);
  if (frame)
    for (int k = 0; k < 9; ++k) frame[k] = (float)e[k];
  return 0;
}

int kapsel_gpu_set_nearcontact(kapsel_ctx *ctx, const kapsel_nc *nc) {
  if (!ctx) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (nc && (!nc->scaled || b->prm.eq != KAPSEL_EQ_NAVIER_STOKES || b->Np < 2 ||
             std::fabs(b->pp.RADIUS - nc->sc.a) > 1e-12 * nc->sc.a))
    return KAPSEL_EINVAL;
  KCHECK(cudaStreamSynchronize(b->stream));
  for (int s = 0; s < 2; ++s)
    if (b->graph[s]) {
      cudaGraphExecDestroy(b->graph[s]);
      b->graph[s] = nullptr;
    }
  if (nc && !b->nc_feat) {
    int rc = nc_smem_setup();
    if (rc) return rc;
    // at most ~25 neighbours within a surface gap of 2a per sphere
    b->nc_cap = 32 * b->Np;
    if (cudaMalloc(&b->nc_feat, sizeof(float) * nc::IN * b->nc_cap) != cudaSuccess ||
        cudaMalloc(&b->nc_frames, sizeof(float) * 9 * b->nc_cap) != cudaSuccess ||
        cudaMalloc(&b->nc_pairs, sizeof(int2) * b->nc_cap) != cudaSuccess ||
        cudaMalloc(&b->nc_count, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&b->nc_corr, sizeof(double) * 6 * b->Np) != cudaSuccess)
      return KAPSEL_ENOMEM;
    KCHECK(cudaMemset(b->nc_count, 0, sizeof(int)));
    KCHECK(cudaMemset(b->nc_corr, 0, sizeof(double) * 6 * b->Np));
  }
  if (nc && b->cl_on) {
    // the lists must reach every pair in the trained gap range
    const int rc = b->setup_cells(std::max(b->cl_rlist, (2.0 * b->pp.RADIUS + nc->sc.gap_hi * nc->sc.a) * (1.0 + 1e-9)));
    if (rc) return rc;
  }
  b->nc = nc;
  return 0;
}

int kapsel_gpu_nearcontact_pairs(kapsel_ctx *ctx, int *n_pairs) {
  // pairs found by the last step's search (0 when no network is attached)
  if (!ctx || !n_pairs) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  *n_pairs = 0;
  if (!b->nc) return 0;
  KCHECK(cudaStreamSynchronize(b->stream));
  KCHECK(cudaMemcpy(n_pairs, b->nc_count, sizeof(int), cudaMemcpyDeviceToHost));
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Restart records: Save_Restart_udf / Force_restore_parameters
// (resume.cxx:10-78, 166-272, 274-365, 366-512) as `path = value` text lines
// with the reference's record paths (resume.CONTINUE.Saved_Data...).
namespace {

const char *const kRes = "resume.CONTINUE.Saved_Data.";

// per-particle vectors of Save_Particle_udf, in its order; n = 3 or 4
struct PField {
  const char *name;
  int n;
};
const PField kPFields[] = {{"R", 3},           {"v", 3},
                           {"v_old", 3},       {"q", 4},
                           {"q_old", 4},       {"f_hydro", 3},
                           {"f_hydro_previous", 3}, {"f_hydro1", 3},
                           {"f_slip", 3},      {"f_slip_previous", 3},
                           {"fr", 3},          {"fr_previous", 3},
                           {"omega", 3},       {"omega_old", 3},
                           {"torque_hydro", 3}, {"torque_hydro_previous", 3},
                           {"torque_hydro1", 3}, {"torque_slip", 3},
                           {"torque_slip_previous", 3}};
constexpr int kNPF = sizeof(kPFields) / sizeof(kPFields[0]);
const char *const kXYZ[3] = {"x", "y", "z"};
const char *const kQ[4] = {"q0", "q1", "q2", "q3"};

// record values of particle n for field f (from a KAPSEL_P_* record)
void pfield_values(const double *rec, int f, double *v) {
  const std::string nm = kPFields[f].name;
  for (int i = 0; i < 4; ++i) v[i] = 0.0;
  if (nm == "R") memcpy(v, rec + KAPSEL_P_X, 3 * sizeof(double));
  else if (nm == "v") memcpy(v, rec + KAPSEL_P_V, 3 * sizeof(double));
  else if (nm == "v_old") memcpy(v, rec + KAPSEL_P_VOLD, 3 * sizeof(double));
  else if (nm == "q") memcpy(v, rec + KAPSEL_P_Q, 4 * sizeof(double));
  else if (nm == "q_old") memcpy(v, rec + KAPSEL_P_QOLD, 4 * sizeof(double));
  else if (nm == "f_hydro_previous") memcpy(v, rec + KAPSEL_P_FHYDRO, 3 * sizeof(double));
  else if (nm == "fr_previous") memcpy(v, rec + KAPSEL_P_FR, 3 * sizeof(double));
  else if (nm == "omega") memcpy(v, rec + KAPSEL_P_OMEGA, 3 * sizeof(double));
  else if (nm == "omega_old") memcpy(v, rec + KAPSEL_P_OMEGAOLD, 3 * sizeof(double));
  else if (nm == "torque_hydro_previous") memcpy(v, rec + KAPSEL_P_THYDRO, 3 * sizeof(double));
  // f_hydro, fr and torque_hydro are zero after reset_Forces; the slip and
  // electrolyte-diagnostic terms are zero for the spherical particles here
}

}  // namespace

extern "C" {

int kapsel_gpu_save_restart(kapsel_ctx *ctx, const char *path) {
  if (!ctx || !path) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (!b->initialised) return KAPSEL_ESTATE;
  const int NX = b->g.NX, NY = b->g.NY, NZ_ = b->g.NZ + 2;
  const size_t plane = (size_t)NX * NY * NZ_;
  std::vector<double> z(2 * plane), uk(3), rec((size_t)KAPSEL_P_STRIDE * std::max(b->Np, 1));
  int rc = kapsel_gpu_get_zeta(ctx, z.data(), uk.data());
  if (rc) return rc;
  rc = kapsel_gpu_get_particles(ctx, rec.data());
  if (rc) return rc;
  const bool el = b->prm.eq == KAPSEL_EQ_ELECTROLYTE;
  std::vector<double> conc(el ? 2 * plane : 0);
  if (el && (rc = b->conc_to_host(conc.data()))) return rc;
  double obl[4] = {0.0, 0.0, 0.0, 0.0};
  if (b->prm.eq == KAPSEL_EQ_SHEAR_LE && (rc = b->oblique_state(obl))) return rc;
  FILE *f = fopen(path, "w");
  if (!f) return KAPSEL_EINVAL;
  fprintf(f, "resume.Calculation = CONTINUE\n");
  for (int i = 0; i < NX; ++i)
    for (int j = 0; j < NY; ++j)
      for (int k = 0; k < NZ_; ++k) {
        const size_t im = ((size_t)i * NY + j) * NZ_ + k;
        fprintf(f, "%sZeta[%d][%d][%d].zeta0 = %.17g\n", kRes, i, j, k, z[im]);
        fprintf(f, "%sZeta[%d][%d][%d].zeta1 = %.17g\n", kRes, i, j, k, z[plane + im]);
        if (el)
          for (int n = 0; n < 2; ++n)
            fprintf(f, "%sConcentration[%d][%d][%d][%d].ck = %.17g\n", kRes, n, i, j, k, conc[n * plane + im]);
      }
  for (int d = 0; d < 3; ++d) fprintf(f, "%suk_dc.%s = %.17g\n", kRes, kXYZ[d], uk[d]);
  for (int n = 0; n < b->Np; ++n)
    for (int fi = 0; fi < kNPF; ++fi) {
      double v[4];
      pfield_values(rec.data() + (size_t)KAPSEL_P_STRIDE * n, fi, v);
      for (int c = 0; c < kPFields[fi].n; ++c)
        fprintf(f, "%sParticles[%d].%s.%s = %.17g\n", kRes, n, kPFields[fi].name,
                kPFields[fi].n == 4 ? kQ[c] : kXYZ[c], v[c]);
    }
  // jikan.ts is the index of the step just completed (the reference saves
  // inside its step loop, sp_3d_ns.cxx:606-616)
  fprintf(f, "%sjikan.ts = %d\n", kRes, b->ts - 1);
  fprintf(f, "%sjikan.time = %.17g\n", kRes, b->time);
  fprintf(f, "%soblique.degree_oblique = %.17g\n", kRes, obl[OB_DEG]);
  const bool ok = !ferror(f);
  fclose(f);
  return ok ? 0 : KAPSEL_EINVAL;
}

int kapsel_gpu_load_restart(kapsel_ctx *ctx, const char *path) {
  if (!ctx || !path) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (!b->initialised) return KAPSEL_ESTATE;
  const int NX = b->g.NX, NY = b->g.NY, NZ_ = b->g.NZ + 2, Np = b->Np;
  const size_t plane = (size_t)NX * NY * NZ_;
  const bool el = b->prm.eq == KAPSEL_EQ_ELECTROLYTE;
  std::vector<double> z(2 * plane, 0.0), conc(el ? 2 * plane : 0, 0.0), uk(3, 0.0);
  std::vector<double> pv((size_t)std::max(Np, 1) * kNPF * 4, 0.0);
  std::vector<unsigned char> seen((size_t)std::max(Np, 1) * kNPF, 0);
  size_t nz_seen = 0;
  int ts = -1, have_time = 0, nuk = 0, have_deg = 0;
  double time = 0.0, deg = 0.0;
  FILE *f = fopen(path, "r");
  if (!f) return KAPSEL_EINVAL;
  std::vector<char> line(1 << 12);
  const size_t lr = strlen(kRes);
  int bad = 0;
  while (fgets(line.data(), (int)line.size(), f)) {
    char *s = line.data();
    // the reference's record writer prefixes "record <n> "
    if (!strncmp(s, "record ", 7)) {
      s += 7;
      while (*s && *s != ' ') ++s;
      while (*s == ' ') ++s;
    }
    if (strncmp(s, kRes, lr)) continue;
    s += lr;
    char *eq = strchr(s, '=');
    if (!eq) continue;
    const double val = strtod(eq + 1, nullptr);
    int i, j, k, n, c;
    char name[128], comp[16];
    if (sscanf(s, "Zeta[%d][%d][%d].zeta%d", &i, &j, &k, &c) == 4) {
      if (i < 0 || i >= NX || j < 0 || j >= NY || k < 0 || k >= NZ_ || c < 0 || c > 1) { bad = 1; continue; }
      z[c * plane + ((size_t)i * NY + j) * NZ_ + k] = val;
      ++nz_seen;
    } else if (sscanf(s, "Concentration[%d][%d][%d][%d].ck", &n, &i, &j, &k) == 4) {
      if (!el) continue;
      if (n < 0 || n > 1 || i < 0 || i >= NX || j < 0 || j >= NY || k < 0 || k >= NZ_) { bad = 1; continue; }
      conc[n * plane + ((size_t)i * NY + j) * NZ_ + k] = val;
    } else if (sscanf(s, "uk_dc.%15[a-z]", comp) == 1) {
      for (int d = 0; d < 3; ++d)
        if (!strcmp(comp, kXYZ[d])) { uk[d] = val; ++nuk; }
    } else if (sscanf(s, "Particles[%d].%127[A-Za-z0-9_].%15[a-z0-9]", &n, name, comp) == 3) {
      if (n < 0 || n >= Np) continue;
      for (int fi = 0; fi < kNPF; ++fi)
        if (!strcmp(name, kPFields[fi].name))
          for (int cc = 0; cc < kPFields[fi].n; ++cc)
            if (!strcmp(comp, kPFields[fi].n == 4 ? kQ[cc] : kXYZ[cc])) {
              pv[((size_t)n * kNPF + fi) * 4 + cc] = val;
              seen[(size_t)n * kNPF + fi] |= (unsigned char)(1u << cc);
            }
    } else if (!strncmp(s, "jikan.ts", 8) && (s[8] == ' ' || s[8] == '=')) {
      ts = (int)strtol(eq + 1, nullptr, 10);
    } else if (!strncmp(s, "jikan.time", 10)) {
      time = val;
      have_time = 1;
    } else if (!strncmp(s, "oblique.degree_oblique", 22)) {
      deg = val;
      have_deg = 1;
    }
  }
  fclose(f);
  if (bad || nz_seen != 2 * plane || nuk != 3 || ts < 0 || !have_time) return KAPSEL_EINVAL;
  for (int n = 0; n < Np; ++n)
    for (int fi = 0; fi < kNPF; ++fi) {
      const std::string nm = kPFields[fi].name;
      const bool needed = nm == "R" || nm == "v" || nm == "v_old" || nm == "q" || nm == "q_old" ||
                          nm == "omega" || nm == "omega_old" || nm == "fr_previous";
      if (needed && seen[(size_t)n * kNPF + fi] != (1u << kPFields[fi].n) - 1) return KAPSEL_EINVAL;
    }
  // Read_Particle_udf (resume.cxx:366-512): quaternions normalised, the
  // unwrapped position restarts at the position
  std::vector<double> rec((size_t)KAPSEL_P_STRIDE * std::max(Np, 1), 0.0);
  auto fld = [&](int n, const char *nm) -> const double * {
    for (int fi = 0; fi < kNPF; ++fi)
      if (!strcmp(kPFields[fi].name, nm)) return &pv[((size_t)n * kNPF + fi) * 4];
    return nullptr;
  };
  for (int n = 0; n < Np; ++n) {
    double *o = rec.data() + (size_t)KAPSEL_P_STRIDE * n;
    memcpy(o + KAPSEL_P_X, fld(n, "R"), 3 * sizeof(double));
    memcpy(o + KAPSEL_P_XNOPBC, fld(n, "R"), 3 * sizeof(double));
    memcpy(o + KAPSEL_P_V, fld(n, "v"), 3 * sizeof(double));
    memcpy(o + KAPSEL_P_VOLD, fld(n, "v_old"), 3 * sizeof(double));
    memcpy(o + KAPSEL_P_OMEGA, fld(n, "omega"), 3 * sizeof(double));
    memcpy(o + KAPSEL_P_OMEGAOLD, fld(n, "omega_old"), 3 * sizeof(double));
    memcpy(o + KAPSEL_P_FHYDRO, fld(n, "f_hydro_previous"), 3 * sizeof(double));
    memcpy(o + KAPSEL_P_THYDRO, fld(n, "torque_hydro_previous"), 3 * sizeof(double));
    memcpy(o + KAPSEL_P_FR, fld(n, "fr_previous"), 3 * sizeof(double));
    for (int which = 0; which < 2; ++which) {
      const double *q = fld(n, which ? "q_old" : "q");
      const double nq = std::sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
      if (!(nq > 0.0)) return KAPSEL_EINVAL;
      for (int i = 0; i < 4; ++i) o[(which ? KAPSEL_P_QOLD : KAPSEL_P_Q) + i] = q[i] * (1.0 / nq);
    }
  }
  int rc = 0;
  const bool le = b->prm.eq == KAPSEL_EQ_SHEAR_LE;
  if (le && (!have_deg || !std::isfinite(deg))) return KAPSEL_EINVAL;
  if (le && b->ts == 0) {
    // A resumed Lees-Edwards run takes its first step (at jikan.ts = the
    // saved ts, so AB2 unless that is 0) from the fresh state before the
    // restore (sp_3d_ns.cxx:547-627) and keeps that step's Shear_rate_eff,
    // which the record does not hold: a fresh context takes the same
    // discarded step.
    if ((rc = b->fill_noise(0))) return rc;
    b->launch_step(b->noise_dev[0], ts == 0 ? 1 : 0);
    if ((rc = check_status(b))) return rc;
  }
  rc = kapsel_gpu_set_zeta(ctx, z.data(), uk.data());
  if (rc) return rc;
  if (el && (rc = b->conc_from_host(conc.data()))) return rc;
  if (Np > 0 && (rc = kapsel_gpu_set_particle_state(ctx, rec.data()))) return rc;
  if (le) {
    // degree_oblique is restored (resume.cxx:333-360; K2 is formed from it on
    // the fly); Shear_rate_eff keeps its current value (above)
    double obl[4];
    if ((rc = b->oblique_state(obl))) return rc;
    if ((rc = b->set_oblique_state(deg, obl[OB_SRATE]))) return rc;
  }
  b->ts = ts + 1;
  b->time = time;
  // The reference's resumed run seeds the thermostat stream afresh
  // (MT_seed(GIVEN_SEED, 0), sp_3d_ns.cxx:477) and takes one step before the
  // restore overwrites the state (sp_3d_ns.cxx:547-627), which draws one
  // step of normals: the stream continues after those.
  b->mt.reset(new MT19937(b->prm.mt_seed));
  b->drop_prefill();
  if (b->pp.thermostat) {
    double pair[2];
    for (int n = 0; n < 3 * Np; ++n) b->mt->gauss2(pair);
  }
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// AVS/Express field snapshots: Init_avs, Add_field_description and the
// binary branches of Output_avs (avs_output.cxx:20-109, 162-342; Navier_Stokes
// columns "ux uy uz phi pressure tau_xy tau_yz tau_zx tau_xx tau_yy") and
// Output_avs_charge (avs_output.cxx:451-549; Electrolyte columns "ux uy uz
// phi surface_charge rho e_potential").
namespace {

void avs_binary_write(FILE *f, const double *a, int NX, int NY, int NZ) {
  // Binary_write (avs_output.cxx:162-175): i fastest, then j, then k
  const int NZ_ = NZ + 2;
  std::vector<float> row((size_t)NX);
  for (int k = 0; k < NZ; ++k)
    for (int j = 0; j < NY; ++j) {
      for (int i = 0; i < NX; ++i) row[i] = (float)a[((size_t)i * NY + j) * NZ_ + k];
      fwrite(row.data(), sizeof(float), row.size(), f);
    }
}

// Output_avs_p (avs_output_p.cxx:13-142, BINARY): per snapshot the particle
// positions (<pfx><ts>.cod: z, y, x blocks) and the radius and body axes
// (<pfx><ts>.dat: radius block, then the columns of the rotation matrix of
// each orientation quaternion) as float32, and their description in the
// particle .fld file.  The rotation matrix of a unit quaternion (s, v) is
// (s^2 - v.v) I + 2 v v^T + 2 s [v]x, the matrix rqtn_rm builds
// (quaternion.h:432-449).
int avs_write_particles(const std::string &dir, const std::string &name, const double *rec, int np, double radius,
                        int ts, double time, int nstep, bool init) {
  const std::string pfld = dir + "/" + name + "p.fld", ppfx = "avs/" + name + "p_";
  const int veclen = 10;
  if (init) {
    FILE *f = fopen(pfld.c_str(), "w");
    if (!f) return KAPSEL_EINVAL;
    fprintf(f, "# AVS field file\nndim=%d\ndim1=%d\nnspace=%d\nveclen=%d\ndata=float\nfield=irregular\n", 1, np, 3,
            veclen);
    fprintf(f, "nstep=%d\nlabel = %s\n", nstep, "Radius x1 x2 x3 y1 y2 y3 z1 z2 z3");
    fclose(f);
  }
  FILE *f = fopen(pfld.c_str(), "a");
  if (!f) return KAPSEL_EINVAL;
  const int data_size = (int)sizeof(float) * np;
  fprintf(f, "time value = \"step%dtime%g\"\n", ts, time);
  for (int n = 0; n < 3; ++n)
    fprintf(f, "coord %d file = %s%d.cod filetype = binary skip = %d\n", 3 - n, ppfx.c_str(), ts, n * data_size);
  for (int n = 0; n < veclen; ++n)
    fprintf(f, "variable %d file = %s%d.dat filetype = binary skip = %d\n", n + 1, ppfx.c_str(), ts, n * data_size);
  fprintf(f, "EOT\n");
  fclose(f);
  std::vector<float> col((size_t)np);
  f = fopen((dir + "/" + ppfx + std::to_string(ts) + ".cod").c_str(), "wb");
  if (!f) return KAPSEL_EINVAL;
  for (int d = 0; d < 3; ++d) {
    for (int n = 0; n < np; ++n) col[n] = (float)rec[(size_t)KAPSEL_P_STRIDE * n + KAPSEL_P_X + 2 - d];
    fwrite(col.data(), sizeof(float), col.size(), f);
  }
  bool ok = !ferror(f);
  fclose(f);
  f = fopen((dir + "/" + ppfx + std::to_string(ts) + ".dat").c_str(), "wb");
  if (!f) return KAPSEL_EINVAL;
  for (int n = 0; n < np; ++n) col[n] = (float)radius;
  fwrite(col.data(), sizeof(float), col.size(), f);
  // R[a][b] for each particle, written column by column (b outer, a inner)
  for (int b = 0; b < 3; ++b)
    for (int a = 0; a < 3; ++a) {
      for (int n = 0; n < np; ++n) {
        const double *q = rec + (size_t)KAPSEL_P_STRIDE * n + KAPSEL_P_Q;  // s, v0, v1, v2
        const double qs = q[0], v[3] = {q[1], q[2], q[3]};
        double r = 2.0 * v[a] * v[b];
        if (a == b) r += qs * qs - (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        // 2 s [v]x: [v]x[a][b] = -eps_abc v_c
        if (a != b) {
          const int c = 3 - a - b;
          const double sgn = ((b - a + 3) % 3 == 1) ? -1.0 : 1.0;
          r += 2.0 * qs * sgn * v[c];
        }
        col[n] = (float)r;
      }
      fwrite(col.data(), sizeof(float), col.size(), f);
    }
  ok = ok && !ferror(f);
  fclose(f);
  return ok ? 0 : KAPSEL_EINVAL;
}

}  // namespace

extern "C" {

int kapsel_gpu_write_avs(kapsel_ctx *ctx, const char *out_dir, const char *out_name, int nstep, int init) {
  if (!ctx || !out_dir || !out_name || nstep < 1) return KAPSEL_EINVAL;
  BoxBase *b = ctx->box.get();
  if (!b->initialised) return KAPSEL_ESTATE;
  const bool el = b->prm.eq == KAPSEL_EQ_ELECTROLYTE;
  if (b->prm.eq != KAPSEL_EQ_NAVIER_STOKES && !el) return KAPSEL_EINVAL;
  const int NX = b->g.NX, NY = b->g.NY, NZ = b->g.NZ, NZ_ = NZ + 2;
  const double DX = b->prm.dx, ETA = b->prm.eta;
  const size_t plane = (size_t)NX * NY * NZ_;
  const std::string dir(out_dir), name(out_name);
  const std::string fld = dir + "/" + name + ".fld", cod = name + ".cod";
  // Veclen / Label, Veclen_charge / Label_charge (avs_output.cxx:14-19)
  const int veclen = el ? 7 : 10;
  const char *label = el ? "ux uy uz phi surface_charge rho e_potential"
                         : "ux uy uz phi pressure tau_xy tau_yz tau_zx tau_xx tau_yy";
  if (init) {
    mkdir((dir + "/avs").c_str(), 0755);
    FILE *f = fopen(fld.c_str(), "w");
    if (!f) return KAPSEL_EINVAL;
    fprintf(f, "# AVS field file\nndim=%d\ndim1=%d\ndim2=%d\ndim3=%d\nnspace=%d\nveclen=%d\n", 3, NX, NY, NZ, 3,
            veclen);
    fprintf(f, "data=float\nfield=uniform\nnstep=%d\n", nstep);
    fprintf(f, "label = %s\n", label);
    fclose(f);
    f = fopen((dir + "/" + cod).c_str(), "wb");
    if (!f) return KAPSEL_EINVAL;
    fprintf(f, "%g\n%g\n%g\n%g\n%g\n%g\n", 0.0, (double)(NX - 1) * DX, 0.0, (double)(NY - 1) * DX, 0.0,
            (double)(NZ - 1) * DX);
    fclose(f);
  }
  // fields in the Ooura real layout [NX][NY][NZ_]
  std::vector<double> u(3 * plane), phi(plane), strain(el ? 0 : 5 * plane, 0.0);
  std::vector<double> surf(el ? plane : 0), conc(el ? 2 * plane : 0), pot(el ? plane : 0);
  int rc = b->velocity_to_host(u.data());
  if (rc) return rc;
  if (el) {
    // Output_avs_charge (avs_output.cxx:451-549)
    if ((rc = b->el_snapshot_host(phi.data(), surf.data(), conc.data(), pot.data()))) return rc;
  } else {
    if ((rc = b->phi_only_host(phi.data()))) return rc;
    // viscous strain tensor eta*(d_i u_j + d_j u_i)/2 of the velocity, by the
    // spectral formula of Zeta_k2Strain_k (fft_wrapper.cxx:201-257)
    std::vector<double> uk(u);
    for (int c = 0; c < 3; ++c)
      if ((rc = b->fft_fwd_host(uk.data() + c * plane))) return rc;
    const double wx = 2.0 * M_PI / (NX * DX), wy = 2.0 * M_PI / (NY * DX), wz = 2.0 * M_PI / (NZ * DX);
    for (int i = 0; i < NX; ++i)
      for (int j = 0; j < NY; ++j)
        for (int k = 0; k < NZ_ / 2; ++k) {
          const size_t im0 = ((size_t)i * NY + j) * NZ_ + 2 * k, im1 = im0 + 1;
          const double ks[3] = {(i > NX / 2 ? i - NX : i) * wx * .5, (j > NY / 2 ? j - NY : j) * wy * .5,
                                k * wz * .5};
          double ud[3][2];
          for (int d = 0; d < 3; ++d) {
            ud[d][0] = ETA * uk[d * plane + im0];
            ud[d][1] = ETA * uk[d * plane + im1];
          }
          double *s0 = strain.data();
          s0[0 * plane + im0] = ks[0] * ud[0][1] * 2.;
          s0[0 * plane + im1] = -ks[0] * ud[0][0] * 2.;
          s0[1 * plane + im0] = ks[0] * ud[1][1] + ks[1] * ud[0][1];
          s0[1 * plane + im1] = -ks[0] * ud[1][0] - ks[1] * ud[0][0];
          s0[2 * plane + im0] = ks[0] * ud[2][1] + ks[2] * ud[0][1];
          s0[2 * plane + im1] = -ks[0] * ud[2][0] - ks[2] * ud[0][0];
          s0[3 * plane + im0] = ks[1] * ud[1][1] * 2.;
          s0[3 * plane + im1] = -ks[1] * ud[1][0] * 2.;
          s0[4 * plane + im0] = ks[1] * ud[2][1] + ks[2] * ud[1][1];
          s0[4 * plane + im1] = -ks[1] * ud[2][0] - ks[2] * ud[1][0];
        }
    for (int c = 0; c < 5; ++c)
      if ((rc = b->fft_inv_host(strain.data() + c * plane))) return rc;
  }
  // Add_field_description (BINARY, uniform field)
  const size_t data_size = sizeof(float) * (size_t)NX * NY * NZ;
  const std::string pfx = "avs/" + name + "_";
  FILE *f = fopen(fld.c_str(), "a");
  if (!f) return KAPSEL_EINVAL;
  fprintf(f, "time value = \"step%dtime%g\"\n", b->ts, b->time);
  for (int n = 0; n < 3; ++n) fprintf(f, "coord %d file = %s filetype = ascii skip = %d\n", n + 1, cod.c_str(), n * 2);
  for (int n = 0; n < veclen; ++n)
    fprintf(f, "variable %d file = %s%d.dat filetype = binary skip = %d\n", n + 1, pfx.c_str(), b->ts,
            (int)(n * data_size));
  fprintf(f, "EOT\n");
  fclose(f);
  const std::string dat = dir + "/" + pfx + std::to_string(b->ts) + ".dat";
  f = fopen(dat.c_str(), "wb");
  if (!f) return KAPSEL_EINVAL;
  for (int c = 0; c < 3; ++c) avs_binary_write(f, u.data() + c * plane, NX, NY, NZ);
  avs_binary_write(f, phi.data(), NX, NY, NZ);
  if (el) {
    // surface charge * 4 pi a^2, rho = (1 - phi) sum_n e z_n c_n summed in
    // float as the reference does, then the potential (avs_output.cxx:490-513)
    const double area = 4.0 * M_PI * (b->prm.a * DX) * (b->prm.a * DX);
    const double val[2] = {b->prm.valency_p, b->prm.valency_n};
    std::vector<float> row((size_t)NX);
    for (int k = 0; k < NZ; ++k)
      for (int j = 0; j < NY; ++j) {
        for (int i = 0; i < NX; ++i) row[i] = (float)(surf[((size_t)i * NY + j) * NZ_ + k] * area);
        fwrite(row.data(), sizeof(float), row.size(), f);
      }
    for (int k = 0; k < NZ; ++k)
      for (int j = 0; j < NY; ++j) {
        for (int i = 0; i < NX; ++i) {
          const size_t im = ((size_t)i * NY + j) * NZ_ + k;
          float q = 0.f;
          for (int n = 0; n < 2; ++n) q += (float)(1.0 * val[n] * conc[n * plane + im]);  // Elementary_charge = 1
          q = (float)((double)q * (1. - phi[im]));
          row[i] = q;
        }
        fwrite(row.data(), sizeof(float), row.size(), f);
      }
    avs_binary_write(f, pot.data(), NX, NY, NZ);
  } else {
    // the Navier_Stokes step computes no pressure field
    std::vector<double> zero(plane, 0.0);
    avs_binary_write(f, zero.data(), NX, NY, NZ);
    const int order[5] = {1, 4, 2, 0, 3};  // xy, yz, zx, xx, yy
    for (int c = 0; c < 5; ++c) avs_binary_write(f, strain.data() + order[c] * plane, NX, NY, NZ);
  }
  const bool ok = !ferror(f);
  fclose(f);
  if (!ok) return KAPSEL_EINVAL;
  if (b->Np == 0) return 0;
  // the particle snapshot the main loop writes beside it (sp_3d_ns.cxx:557-559)
  std::vector<double> rec((size_t)KAPSEL_P_STRIDE * b->Np);
  if ((rc = kapsel_gpu_get_particles(ctx, rec.data()))) return rc;
  return avs_write_particles(dir, name, rec.data(), b->Np, b->prm.a * DX, b->ts, b->time, nstep, init != 0);
}

}  // extern "C"
