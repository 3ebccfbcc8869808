// Fused y and z passes over one (component, x) plane per block.
//
// Two pass pairs of the Navier-Stokes step act on each velocity component
// on its own: the inverse to u* (inverse y, then the z c2r; as k_yw_pass
// followed by k_zw_c2r) and the rigidity force (z forward, then forward y;
// as k_zw_force followed by k_yw_pass).  Between the two passes of a pair a
// (component, x) plane is NY rows of TZ retained kz values, 45 KB in FP32
// at 128^3, so one block keeps it in shared memory: the intermediate never
// goes through global memory and the pair is one launch.  The per-line
// transforms, packings, force expressions and store orders are those of the
// separate kernels, so the results are bitwise the same.
//
// Plane rows have the stride PS = TZ rounded up to 4 mod 8 elements: the
// column accesses of the y phases (four kz columns of eight consecutive rows
// per warp instruction) then fall on distinct banks for 8- and 16-byte
// elements, and the z phases read and write rows contiguously.
#pragma once

#include "particle_kernels.cuh"
#include "zwarp_kernels.cuh"

namespace kapsel {

template <typename R, int LY, int LM>
struct YZ {
  using Y = ZL<LY>;
  using Z = ZL<LM>;
  using YL = YLines<R, LY>;
  static constexpr int NY = Y::M;
  static constexpr int PS = ((Z::TZ + 3) / 8) * 8 + 4;  // plane row stride, PS % 8 == 4
  static constexpr int SLOT_Y = Y::RW * YL::LS, SLOT_Z = Z::RW * Z::LS;
  static constexpr int SLOT = SLOT_Y > SLOT_Z ? SLOT_Y : SLOT_Z;  // per-warp lines
  static constexpr int NB = (Z::TZ + Y::RW - 1) / Y::RW;          // kz column batches
  static constexpr int NG = NY / Z::RW;                           // z row groups
  static size_t smem(int nw) { return sizeof(Cx<R>) * ((size_t)NY * PS + (size_t)nw * SLOT); }
};

// Inverse y, then z c2r, of planes (c, x) = blockIdx.x < nplanes:
//   in [c][NX][KYc][TS] (x real, ky compact) -> out[c * out_cstride +
//   (x NY + y) out_pitch + z] (A_k2a-scaled reals).
// Blocks at or past nplanes run the particle position update, as in
// k_zw_c2r.
template <typename R, int LY, int LM, bool FULLY, int NW>
__global__ void __launch_bounds__(NW * 32) k_yzw_c2r(Geo g, Twiddles<R> tw, const Cx<R> *__restrict__ in,
                                                     R *__restrict__ out, size_t out_cstride, int out_pitch,
                                                     int nplanes, PPar pp, DPart *__restrict__ parts, int euler,
                                                     int *__restrict__ status) {
  using P = YZ<R, LY, LM>;
  using Y = typename P::Y;
  using Z = typename P::Z;
  using YL = typename P::YL;
  using V2 = typename Vec2<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  pdl_begin();
  if ((int)blockIdx.x >= nplanes) {
    const int n = ((int)blockIdx.x - nplanes) * blockDim.x + threadIdx.x;
    if (parts && n < pp.Np) position_update_one(pp, parts, n, euler, status);
    return;
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Cx<R> *plane = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *slot = plane + P::NY * P::PS + warp * P::SLOT;
  const int pl = blockIdx.x;  // c * NX + x
  const int c = pl / g.NX;
  {
    Cx<R> w[Y::N1];
    wfft_twiddles<R, LY, -1>(tw.y, w);
    // the warp's next batch of kz columns is loaded into registers while the
    // current one is transformed (the elements of yw_issue, same placement)
    constexpr int TYc = FULLY ? P::NY / 2 + 1 : (P::NY + 2) / 3, KYc = FULLY ? P::NY : 2 * TYc - 1;
    constexpr int NL = (KYc * Y::RW + 31) / 32;
    const Cx<R> zero = {R(0), R(0)};
    Cx<R> pre[NL];
    auto load_batch = [&](int b) {
      const int col0 = b * Y::RW, ncols = min(Y::RW, Z::TZ - col0);
      const Cx<R> *src = in + (size_t)pl * KYc * g.TS + col0;
#pragma unroll
      for (int q = 0; q < NL; ++q) {
        const int i = lane + 32 * q, r = i >> Y::LR, col = i & (Y::RW - 1);
        pre[q] = (i < KYc * Y::RW && col < ncols) ? src[(size_t)r * g.TS + col] : zero;
      }
    };
    if (warp < P::NB) load_batch(warp);
    for (int b = warp; b < P::NB; b += NW) {
#pragma unroll
      for (int q = 0; q < NL; ++q) {
        const int i = lane + 32 * q, r = i >> Y::LR, col = i & (Y::RW - 1);
        const int j = r < TYc ? r : P::NY + r - KYc;
        if (i < KYc * Y::RW) slot[YL::template base<LY>(col) + zpos<LY>(j)] = pre[q];
      }
      for (int i = lane; i < (P::NY - KYc) * Y::RW; i += 32) {
        const int j = TYc + (i >> Y::LR), col = i & (Y::RW - 1);
        slot[YL::template base<LY>(col) + zpos<LY>(j)] = zero;
      }
      if (b + NW < P::NB) load_batch(b + NW);
      __syncwarp();
      wfft<R, LY, -1, YL>(slot, w);
      const int col0 = b * Y::RW, ncols = min(Y::RW, Z::TZ - col0);
      for (int i = lane; i < P::NY * Y::RW; i += 32) {
        const int r = i >> Y::LR, col = i & (Y::RW - 1);
        if (col < ncols) plane[r * P::PS + col0 + col] = slot[YL::template base<LY>(col) + zpos<LY>(r)];
      }
      __syncwarp();
    }
  }
  __syncthreads();
  Cx<R> wi[Z::N1], wk[Z::KW];
  wfft_twiddles<R, LM, -1>(tw.m, wi);
  wpre_twiddles<R, LM>(tw.z, wk);
  const R sc = R(g.inv_n);
  const size_t row_base = (size_t)(pl - c * g.NX) * P::NY;
  for (int grp = warp; grp < P::NG; grp += NW) {
    for (int rr = 0; rr < Z::RW; ++rr) wpack_c2r<R, LM>(plane + (grp * Z::RW + rr) * P::PS, slot + rr * Z::LS, wk);
    __syncwarp();
    wfft<R, LM, -1>(slot, wi);
    R *dst = out + c * out_cstride + (row_base + grp * Z::RW) * (size_t)out_pitch;
    for (int i = lane; i < Z::RW * Z::M; i += 32) {
      const int rr = i >> LM, n = i & (Z::M - 1);
      const Cx<R> v = slot[rr * Z::LS + zpos<LM>(n)];
      V2 o;
      o.x = v.x * sc;
      o.y = v.y * sc;
      *reinterpret_cast<V2 *>(dst + rr * (size_t)out_pitch + 2 * n) = o;
    }
    __syncwarp();
  }
}

// Rigidity force of component c = blockIdx.x / NX on plane x, z forward, then
// forward y: f_c = up_c' - phi' u*_c with the phi > 1 clamp (as k_zw_force),
// out [c][NX][KYc][TS].  up_c is cleared where phi is non-zero by the
// component's own block; phi, which the blocks of all three components of
// the plane read, by the last of them to finish reading (plane_count[x],
// zero between launches), from the bit mask of non-zero element pairs that
// every block gathers while it reads phi.
template <typename R, int LY, int LM, bool FULLY, int NW>
__global__ void __launch_bounds__(NW * 32) k_zyw_force(Geo g, Twiddles<R> tw, R *__restrict__ phiup,
                                                       const R *__restrict__ ustar, Cx<R> *__restrict__ out,
                                                       unsigned *__restrict__ plane_count) {
  using P = YZ<R, LY, LM>;
  using Y = typename P::Y;
  using Z = typename P::Z;
  using YL = typename P::YL;
  using V2 = typename Vec2<R>::T;
  constexpr int NI = Z::RW * Z::M / 32;           // element pairs per lane and row group
  constexpr int MASKW = P::NY * Z::M / 32;        // mask words of the plane
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ unsigned nzmask[MASKW];
  __shared__ int last_reader;
  pdl_begin();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  Cx<R> *plane = reinterpret_cast<Cx<R> *>(smem_raw);
  Cx<R> *slot = plane + P::NY * P::PS + warp * P::SLOT;
  const int pl = blockIdx.x;  // c * NX + x
  const int c = pl / g.NX, x = pl - c * g.NX;
  const size_t npts = (size_t)g.NX * P::NY * Z::NZ;
  const size_t row_base = (size_t)x * P::NY;
  R *upc = phiup + (size_t)(1 + c) * npts;
  const R *usc = ustar + (size_t)c * npts;
  {
    Cx<R> wf[Z::N1];
    wfft_twiddles<R, LM, 1>(tw.m, wf);
    // phi of the warp's next row group is loaded while the current one is
    // transformed
    V2 ph_next[NI];
    if (warp < P::NG)
#pragma unroll
      for (int h = 0; h < NI; ++h)
        ph_next[h] = *reinterpret_cast<const V2 *>(phiup + (row_base + (size_t)warp * Z::RW) * Z::NZ +
                                                   2 * (size_t)(lane + 32 * h));
    for (int grp = warp; grp < P::NG; grp += NW) {
      const size_t row0 = row_base + (size_t)grp * Z::RW;
      // all of the lane's loads first (up and u* where phi is non-zero), so
      // that they are in flight together
      V2 ph[NI], up[NI], us[NI];
#pragma unroll
      for (int h = 0; h < NI; ++h) ph[h] = ph_next[h];
      if (grp + NW < P::NG)
#pragma unroll
        for (int h = 0; h < NI; ++h)
          ph_next[h] = *reinterpret_cast<const V2 *>(phiup + (row0 + (size_t)NW * Z::RW) * Z::NZ +
                                                     2 * (size_t)(lane + 32 * h));
#pragma unroll
      for (int h = 0; h < NI; ++h) {
        const size_t o = row0 * Z::NZ + 2 * (size_t)(lane + 32 * h);
        up[h] = us[h] = V2{R(0), R(0)};
        if (ph[h].x != R(0) || ph[h].y != R(0)) {
          up[h] = *reinterpret_cast<const V2 *>(upc + o);
          us[h] = *reinterpret_cast<const V2 *>(usc + o);
        }
      }
#pragma unroll
      for (int h = 0; h < NI; ++h) {
        const int i = lane + 32 * h, rr = i >> LM, n = i & (Z::M - 1);
        const size_t o = row0 * Z::NZ + 2 * (size_t)i;
        const bool nz = ph[h].x != R(0) || ph[h].y != R(0);
        const unsigned bits = __ballot_sync(0xffffffffu, nz);
        if (lane == 0) nzmask[grp * NI + h] = bits;
        R p0 = ph[h].x, p1 = ph[h].y;
        if (p0 > R(1)) {
          const R inv = R(1) / p0;
          up[h].x *= inv;
          p0 = R(1);
        }
        if (p1 > R(1)) {
          const R inv = R(1) / p1;
          up[h].y *= inv;
          p1 = R(1);
        }
        slot[rr * Z::LS + zpos<LM>(n)] = {up[h].x - p0 * us[h].x, up[h].y - p1 * us[h].y};
        if (nz) *reinterpret_cast<V2 *>(upc + o) = V2{R(0), R(0)};
      }
      __syncwarp();
      wfft<R, LM, 1>(slot, wf);
      for (int i = lane; i < Z::RW * Z::TZ; i += 32) {
        const int rr = i / Z::TZ, k = i - rr * Z::TZ;
        plane[(grp * Z::RW + rr) * P::PS + k] = wunpack_r2c<R, LM>(slot + rr * Z::LS, k, tw.z);
      }
      __syncwarp();
    }
  }
  __syncthreads();
  // every phi value of this block has been read (and used) above
  if (threadIdx.x == 0) {
    __threadfence();
    last_reader = atomicAdd(plane_count + x, 1u) == 2u;
  }
  {
    Cx<R> w[Y::N1];
    wfft_twiddles<R, LY, 1>(tw.y, w);
    const Cx<R> zero = {R(0), R(0)};
    for (int b = warp; b < P::NB; b += NW) {
      const int col0 = b * Y::RW, ncols = min(Y::RW, Z::TZ - col0);
      for (int i = lane; i < P::NY * Y::RW; i += 32) {
        const int r = i >> Y::LR, col = i & (Y::RW - 1);
        slot[YL::template base<LY>(col) + zpos<LY>(r)] = col < ncols ? plane[r * P::PS + col0 + col] : zero;
      }
      __syncwarp();
      wfft<R, LY, 1, YL>(slot, w);
      Cx<R> *dst = out + (size_t)pl * g.KYc * g.TS + col0;
      for (int i = lane; i < g.KYc * Y::RW; i += 32) {
        const int r = i >> Y::LR, col = i & (Y::RW - 1);
        const int j = full_from_compact(r, g.TY, g.KYc, P::NY);
        if (col < ncols) dst[(size_t)r * g.TS + col] = slot[YL::template base<LY>(col) + zpos<LY>(j)];
      }
      __syncwarp();
    }
  }
  __syncthreads();
  if (last_reader) {
    __threadfence();
    // element pair q of the plane (row q / M, pair q % M) is mask bit q
    R *phi = phiup + row_base * Z::NZ;
    for (int wd = warp; wd < MASKW; wd += NW)
      if ((nzmask[wd] >> lane) & 1u) *reinterpret_cast<V2 *>(phi + 2 * (size_t)(wd * 32 + lane)) = V2{R(0), R(0)};
    if (threadIdx.x == 0) plane_count[x] = 0u;
  }
}

}  // namespace kapsel
