// Cell lists and per-particle neighbour lists for large particle counts.
//
// The reference finds LJ pairs with a head/linked-list cell list of
// 16-grid-unit cells and a 27-cell scan (md_force.cxx:23-134).  Here the
// same idea serves every pair search of the step at once: after the
// position update the particles are binned into cells at least as wide as
// the longest pair range in use (the LJ cutoff, the overlap of two profile
// supports 2(RADIUS+HXI), and the near-contact range when a correction
// network is attached), and each particle gets the list of the particles
// within that range, in increasing index order.  The LJ force, the
// deterministic phi/up scatter and the near-contact pair search then read
// the lists instead of scanning all particles.  The LJ force keeps the
// reference's pair multiplicity of its own 16-unit cells (the kernel
// computes it per pair), so results do not depend on the cells used here.
//
// Five launches: count, scan, fill, sort (each cell's members by index, so
// the lists do not depend on atomic ordering) and the neighbour lists.
#pragma once

#include <cuda_runtime.h>

#include "particle_kernels.cuh"

namespace kapsel {

struct CellPar {
  int lc[3];         // cells per axis
  double inv_cl[3];  // 1 / cell length
  int ncell;
  double r2list;     // squared neighbour range
};

__device__ __forceinline__ void cell_coords(const double *x, const CellPar &c, int ci[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int k = (int)(x[d] * c.inv_cl[d]);
    ci[d] = k < 0 ? 0 : (k >= c.lc[d] ? c.lc[d] - 1 : k);
  }
}

__global__ void k_cell_count(PPar p, CellPar c, const DPart *__restrict__ parts, int *__restrict__ cellof,
                             int *__restrict__ count) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= p.Np) return;
  int ci[3];
  cell_coords(parts[n].x, c, ci);
  const int cell = (ci[0] * c.lc[1] + ci[1]) * c.lc[2] + ci[2];
  cellof[n] = cell;
  atomicAdd(count + cell, 1);
}

// Exclusive scan of the per-cell counts (one block of 1024 threads): start
// and cursor, and the counts cleared for the next build.
__global__ void __launch_bounds__(1024) k_cell_scan(CellPar c, int *__restrict__ count, int *__restrict__ start,
                                                    int *__restrict__ cursor) {
  __shared__ int wsum[32];
  __shared__ int carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < c.ncell; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int v = i < c.ncell ? count[i] : 0;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int before = carry;
    for (int w = 0; w < warp; ++w) before += wsum[w];
    if (i < c.ncell) {
      const int ex = before + incl - v;
      start[i] = ex;
      cursor[i] = ex;
      count[i] = 0;
    }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) carry += wsum[w];
    __syncthreads();
  }
  if (threadIdx.x == 0) start[c.ncell] = carry;
}

__global__ void k_cell_fill(PPar p, const int *__restrict__ cellof, int *__restrict__ cursor, int *__restrict__ list) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= p.Np) return;
  list[atomicAdd(cursor + cellof[n], 1)] = n;
}

// Members of each cell in increasing particle index (a cell holds a few).
__global__ void k_cell_sort(CellPar c, const int *__restrict__ start, int *__restrict__ list) {
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= c.ncell) return;
  const int b = start[cell], e = start[cell + 1];
  for (int i = b + 1; i < e; ++i) {
    const int v = list[i];
    int k = i - 1;
    while (k >= b && list[k] > v) {
      list[k + 1] = list[k];
      --k;
    }
    list[k + 1] = v;
  }
}

// Neighbour list of each particle: count, then up to NBL_MAX indices in
// increasing order, of the particles within the list range (minimum image).
// More neighbours than NBL_MAX: KAPSEL_ERANGE in the status word.  One warp
// per particle: the lanes test a cell's members together and append the
// hits in cell order (ballot), then each lane places its entries by rank.
constexpr int NBL_WARPS = 4;  // particles per block
__global__ void __launch_bounds__(NBL_WARPS * 32) k_neighbor_lists(PPar p, CellPar c, const DPart *__restrict__ parts,
                                                                   const int *__restrict__ start,
                                                                   const int *__restrict__ list, int *__restrict__ nbl,
                                                                   int *__restrict__ status) {
  __shared__ int cand[NBL_WARPS][NBL_MAX];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = blockIdx.x * NBL_WARPS + warp;
  if (n >= p.Np) return;  // a whole warp: no later block-wide barrier
  int *cw = cand[warp];
  const double xn[3] = {parts[n].x[0], parts[n].x[1], parts[n].x[2]};
  int ci[3];
  cell_coords(xn, c, ci);
  int cnt = 0;
  for (int ox = -1; ox <= 1; ++ox) {
    // each distinct neighbouring cell once (fewer than 3 cells on an axis)
    if ((c.lc[0] == 1 && ox != 0) || (c.lc[0] == 2 && ox == -1)) continue;
    const int cx = (ci[0] + ox + c.lc[0]) % c.lc[0];
    for (int oy = -1; oy <= 1; ++oy) {
      if ((c.lc[1] == 1 && oy != 0) || (c.lc[1] == 2 && oy == -1)) continue;
      const int cy = (ci[1] + oy + c.lc[1]) % c.lc[1];
      for (int oz = -1; oz <= 1; ++oz) {
        if ((c.lc[2] == 1 && oz != 0) || (c.lc[2] == 2 && oz == -1)) continue;
        const int cz = (ci[2] + oz + c.lc[2]) % c.lc[2];
        const int cell = (cx * c.lc[1] + cy) * c.lc[2] + cz;
        const int b = start[cell], e = start[cell + 1];
        for (int k0 = b; k0 < e; k0 += 32) {
          const int k = k0 + lane;
          int j = -1;
          bool hit = false;
          if (k < e) {
            j = list[k];
            if (j != n) {
              double s = 0.0;
#pragma unroll
              for (int d = 0; d < 3; ++d) {
                double dd = parts[j].x[d] - xn[d];
                dd -= nint_d(dd * p.invL[d]) * p.L[d];
                s += dd * dd;
              }
              hit = s < c.r2list;
            }
          }
          const unsigned bal = __ballot_sync(0xffffffffu, hit);
          const int pos = cnt + __popc(bal & ((1u << lane) - 1u));
          if (hit && pos < NBL_MAX) cw[pos] = j;
          cnt += __popc(bal);
        }
      }
    }
  }
  __syncwarp();
  if (cnt > NBL_MAX) {
    if (lane == 0) atomicExch(status, -6);
    cnt = NBL_MAX;
  }
  // increasing index order: each entry's rank among the distinct indices
  int *out = nbl + (size_t)n * (NBL_MAX + 1);
  for (int q = lane; q < cnt; q += 32) {
    const int v = cw[q];
    int r = 0;
    for (int t = 0; t < cnt; ++t) r += cw[t] < v;
    out[1 + r] = v;
  }
  if (lane == 0) out[0] = cnt;
}

}  // namespace kapsel
