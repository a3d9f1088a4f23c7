// rbx_cells.cu -- cell binning, cell-sorted atom order, candidate (Verlet)
// lists and the velocity-Verlet integration kernels for sm_100a.
//
// Binning replaces LinkedCell::AssignAtomsToCell / SortAtomsByCellKey /
// ComputeCellRangesIndices (src/neighbor_list/src/linked_cell/linked_cell.cpp:428-670,
// src/neighbor_list/src/op/rocm/linked_cell_op.hip.cu:57-164) with a counting
// sort: atomic histogram, one-block scan, atomic scatter, then a per-cell
// bitonic sort.  Inside a cell atoms are ordered by a 4x4x4 Morton sub-cell
// code, then by old index (deterministic), so consecutive atoms are close in
// space: 32-atom chunks have small bounding boxes for the list builder.
//
// The candidate list replaces Estimate/GenerateFullNeighborListOp
// (src/neighbor_list/src/op/rocm/full_neighbor_list_op.hip.cu:177-288): one
// warp per 32 centre atoms (one per lane) streams the chunks of the 27
// stencil cells that survive a bounding-box cull through shared memory and
// screens them in FP32; only pairs inside a guard band around the cutoff are
// settled with the reference's FP64 predicate, so the list is bit-identical
// (as a set) to the FP64 reference list.  Rows come out in stencil order,
// then in cell order.
#include <math.h>

#include "rbx_common.cuh"
#include "rbx_kernels.h"

namespace rbx {

constexpr int SEG_MAX = 2048;  // atoms per cell handled by the segment sort

__device__ __forceinline__ int cell_coord(double v, double lo, double inv_edge, int dim) {
  int c = (int)floor((v - lo) * inv_edge);
  c = c < 0 ? 0 : c;
  return c > dim - 1 ? dim - 1 : c;
}

// Morton interleave of three 2-bit sub-cell coordinates.
__device__ __forceinline__ unsigned morton2(unsigned a, unsigned b, unsigned c) {
  unsigned m = 0;
#pragma unroll
  for (int bit = 0; bit < 2; ++bit)
    m |= ((a >> bit) & 1u) << (3 * bit) | ((b >> bit) & 1u) << (3 * bit + 1) |
         ((c >> bit) & 1u) << (3 * bit + 2);
  return m;
}

constexpr int SUB_SHIFT = 26;  // key = sub-cell code << 26 | old index (n < 2^26)

// Cell edge and its reciprocal per dimension, formed on the host as LinkedCell
// does (edge = box length / cells, reciprocal = 1 / edge).
struct CellGeom {
  double edge[3], inv[3];
};

// AssignAtomsToCell (linked_cell_op.hip.cu:57-138, no halo): floor((p - lo) *
// 1/edge) clamped, then, for a point outside that cell's bounds
// [lo + c edge, lo + (c + 1) edge) (products and sums rounded separately), a
// move of one cell per dimension that is kept only if the point lies inside
// the corrected cell.
__device__ __forceinline__ void assign_cell(const DBox& b, const CellGeom& g, const int dims[3],
                                            const double p[3], int c[3]) {
  bool inside = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    c[d] = cell_coord(p[d], b.lo[d], g.inv[d], dims[d]);
    const double cmin = __dadd_rn(__dmul_rn((double)c[d], g.edge[d]), b.lo[d]);
    const double cmax = __dadd_rn(__dmul_rn((double)(c[d] + 1), g.edge[d]), b.lo[d]);
    inside = inside && cmin <= p[d] && p[d] < cmax;
  }
  if (inside) return;
  int cc[3];
  bool ok = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double cmin = __dadd_rn(__dmul_rn((double)c[d], g.edge[d]), b.lo[d]);
    const double cmax = __dadd_rn(__dmul_rn((double)(c[d] + 1), g.edge[d]), b.lo[d]);
    cc[d] = c[d] + (p[d] < cmin ? -1 : (p[d] >= cmax ? 1 : 0));
    cc[d] = cc[d] < 0 ? 0 : (cc[d] > dims[d] - 1 ? dims[d] - 1 : cc[d]);
    const double nmin = __dadd_rn(__dmul_rn((double)cc[d], g.edge[d]), b.lo[d]);
    const double nmax = __dadd_rn(__dmul_rn((double)(cc[d] + 1), g.edge[d]), b.lo[d]);
    ok = ok && nmin <= p[d] && p[d] < nmax;
  }
  if (ok)
    for (int d = 0; d < 3; ++d) c[d] = cc[d];
}

__global__ void k_cell_assign(DBox b, CellGeom g, int dx, int dy, int dz, int n,
                              const double* __restrict__ x, const double* __restrict__ y,
                              const double* __restrict__ z, int* __restrict__ cell,
                              unsigned* __restrict__ sub, int* __restrict__ counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double fx = (x[i] - b.lo[0]) * (dx / b.len[0]);
  const double fy = (y[i] - b.lo[1]) * (dy / b.len[1]);
  const double fz = (z[i] - b.lo[2]) * (dz / b.len[2]);
  const int dims[3] = {dx, dy, dz};
  const double p[3] = {x[i], y[i], z[i]};
  int cc[3];
  assign_cell(b, g, dims, p, cc);
  const int cx = cc[0], cy = cc[1], cz = cc[2];
  const int c = (cz * dy + cy) * dx + cx;
  cell[i] = c;
  auto sub4 = [](double f, int c0) {
    int v = (int)floor((f - c0) * 4.0);
    return (unsigned)(v < 0 ? 0 : (v > 3 ? 3 : v));
  };
  sub[i] = n < (1 << SUB_SHIFT) ? morton2(sub4(fx, cx), sub4(fy, cy), sub4(fz, cz)) : 0u;
  // atoms still in the order of the last sort share cells along a warp: one
  // atomic per distinct cell of the warp
  const unsigned same = __match_any_sync(__activemask(), c);
  if ((threadIdx.x & 31) == __ffs(same) - 1) atomicAdd(counts + c, __popc(same));
}

// Exclusive scan of counts into start[0..ncell] (one block of 1024 threads).
__global__ void __launch_bounds__(1024)
k_cell_scan(int ncell, const int* __restrict__ counts, int* __restrict__ start,
            int* __restrict__ fill) {
  __shared__ int s_warp[32];
  __shared__ int s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int base = 0; base < ncell; base += 1024) {
    const int c = base + threadIdx.x;
    const int v = c < ncell ? counts[c] : 0;
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) s_warp[w] = incl;
    __syncthreads();
    if (w == 0) {
      int ws = s_warp[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, ws, o);
        if (lane >= o) ws += t;
      }
      s_warp[lane] = ws;
    }
    __syncthreads();
    const int excl = s_carry + (w > 0 ? s_warp[w - 1] : 0) + incl - v;
    if (c < ncell) {
      start[c] = excl;
      fill[c] = excl;
    }
    __syncthreads();
    if (threadIdx.x == 1023) s_carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0) start[ncell] = s_carry;
}

__global__ void k_cell_scatter(int n, const int* __restrict__ cell,
                               const unsigned* __restrict__ sub, int* __restrict__ fill,
                               unsigned* __restrict__ tmp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  // one atomic per distinct cell of the warp; the order inside a cell is set
  // by the segment sort that follows
  const int c = cell[i];
  const unsigned same = __match_any_sync(__activemask(), c);
  const int lane = threadIdx.x & 31, leader = __ffs(same) - 1;
  int base = 0;
  if (lane == leader) base = atomicAdd(fill + c, __popc(same));
  base = __shfl_sync(same, base, leader);
  tmp[base + __popc(same & ((1u << lane) - 1u))] = (sub[i] << SUB_SHIFT) | (unsigned)i;
}

// One block per cell: bitonic sort of the cell's keys (sub-cell, old index).
__global__ void __launch_bounds__(512)
k_cell_segsort(int ncell, int n, const int* __restrict__ start, const unsigned* __restrict__ tmp,
               int* __restrict__ perm, int* __restrict__ cell_of_sorted, int* __restrict__ status) {
  __shared__ unsigned s[SEG_MAX];
  const int c = blockIdx.x;
  const int a = start[c], cnt = start[c + 1] - a;
  const unsigned mask = n < (1 << SUB_SHIFT) ? (1u << SUB_SHIFT) - 1u : 0xffffffffu;
  if (cnt > SEG_MAX) {  // reported; the cell keeps a valid, unsorted permutation
    if (threadIdx.x == 0) atomicOr(status, 2);
    for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
      perm[a + t] = (int)(tmp[a + t] & mask);
      cell_of_sorted[a + t] = c;
    }
    return;
  }
  int p2 = 1;
  while (p2 < cnt) p2 <<= 1;
  for (int t = threadIdx.x; t < p2; t += blockDim.x) s[t] = t < cnt ? tmp[a + t] : 0xffffffffu;
  __syncthreads();
  for (int k = 2; k <= p2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = threadIdx.x; t < p2; t += blockDim.x) {
        const int u = t ^ j;
        if (u > t) {
          const bool up = (t & k) == 0;
          const unsigned va = s[t], vb = s[u];
          if ((va > vb) == up) {
            s[t] = vb;
            s[u] = va;
          }
        }
      }
      __syncthreads();
    }
  }
  for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
    perm[a + t] = (int)(s[t] & mask);
    cell_of_sorted[a + t] = c;
  }
}

// ---------------------------------------------------------------------------
// Candidate list.  Atoms of a cell are cut into 32-atom chunks; chunk k of
// cell c sits at table index (cell_start[c] >> 5) + c + k, which is unique
// and needs no scan (the indices of consecutive cells never overlap), and the
// few indices between two cells are marked empty.  k_chunk_boxes writes each
// chunk's bounding box, rounded outwards to FP32, and its cell.
//
// k_full_list runs one warp per chunk of centre atoms, one centre atom per
// lane.  For each of the 27 stencil cells it culls the cell's chunks against
// the group's box (directed rounding: a lower bound of the true box distance,
// so no pair within the cutoff is ever culled), then streams each surviving
// chunk through a 32-slot shared buffer as {v, |v|^2}, FP32 coordinates
// relative to the centre cell's centre with the periodic image applied.
// Lane u tests slot v as |v|^2 - 2 u.v < C - |u|^2: three FMAs per pair.
// Pairs inside a guard band around the cutoff are settled with the
// reference's FP64 predicate, so the list equals the FP64 reference list as a
// set; rows come out in stencil order, then in cell order.
//
// Split rows (RBL engines in the mixed form): a pair whose build distance is
// certainly at least r_near = r_core + skin cannot come within r_core before
// the next rebuild (no atom moves more than skin/2 before one), so the fused
// RBL kernel tests it with its batch hash first.  Such far pairs are written from the end of the
// row backwards; every other candidate from the front.  count[i] is the
// number of candidates (above cap: overflow), far[i] the number written to
// the back; the front holds min(count, cap) - far[i] entries, all written.
// ---------------------------------------------------------------------------
constexpr int NL_BLOCK = 128;
constexpr int NL_WARPS = NL_BLOCK / 32;

__device__ __forceinline__ int chunk_base(int c, int cs) { return (cs >> 5) + c; }

int full_list_table_size(int n, int ncell) { return (n >> 5) + ncell; }

__global__ void __launch_bounds__(128)
k_chunk_boxes(const double* __restrict__ x, const double* __restrict__ y,
              const double* __restrict__ z, const int* __restrict__ cell_start,
              float4* __restrict__ box_lo, float4* __restrict__ box_hi, int* __restrict__ cell_of) {
  const int c = blockIdx.x;
  const int cs = cell_start[c], ce = cell_start[c + 1];
  const int nch = (ce - cs + 31) >> 5;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int base = chunk_base(c, cs);
  for (int k = warp; k < nch; k += 4) {
    const int a = cs + 32 * k + lane;
    const bool ok = a < ce;
    float lo[3], hi[3];
    const double* p[3] = {x, y, z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const double v = ok ? p[d][a] : 0.0;
      lo[d] = ok ? __double2float_rd(v) : INFINITY;
      hi[d] = ok ? __double2float_ru(v) : -INFINITY;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
        hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
      }
    if (lane == 0) {
      box_lo[base + k] = make_float4(lo[0], lo[1], lo[2], 0.f);
      box_hi[base + k] = make_float4(hi[0], hi[1], hi[2], 0.f);
      cell_of[base + k] = c;
    }
  }
  const int next = chunk_base(c + 1, ce);  // first index of the next cell
  for (int t = base + nch + threadIdx.x; t < next; t += blockDim.x) cell_of[t] = -1;
}

// SPLIT: RBL rows with a far segment; without it (Verlet lists) no far test.
template <bool SPLIT>
__global__ void __launch_bounds__(NL_BLOCK, 5)
k_full_list(DBox b, int dimx, int dimy, int dimz, double cut2, float cut2_up, float lo_band,
            float hi_band, int nidx, const double* __restrict__ x, const double* __restrict__ y,
            const double* __restrict__ z, const int* __restrict__ cell_start,
            const float4* __restrict__ box_lo, const float4* __restrict__ box_hi,
            const int* __restrict__ cell_of, int cap, int* __restrict__ count,
            int* __restrict__ nbrs, int* __restrict__ overflow, float near2,
            int* __restrict__ far, long long* __restrict__ total) {
  __shared__ float4 buf[NL_WARPS][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int w = blockIdx.x * NL_WARPS + warp;
  if (w >= nidx) return;
  const int c = cell_of[w];
  if (c < 0) return;  // an index between two cells
  const int cs = cell_start[c], ce = cell_start[c + 1];
  const int g = w - chunk_base(c, cs);
  const int cz = c / (dimx * dimy), cy = (c / dimx) % dimy, cx = c % dimx;
  const double ox = b.lo[0] + (cx + 0.5) * (b.len[0] / dimx);
  const double oy = b.lo[1] + (cy + 0.5) * (b.len[1] / dimy);
  const double oz = b.lo[2] + (cz + 0.5) * (b.len[2] / dimz);
  const bool live = cs + g * 32 + lane < ce;
  const int i = live ? cs + g * 32 + lane : cs + g * 32;
  const double xi = x[i], yi = y[i], zi = z[i];
  const float ux = (float)(xi - ox), uy = (float)(yi - oy), uz = (float)(zi - oz);
  const float uu = fmaf(ux, ux, fmaf(uy, uy, uz * uz));
  const float ax = live ? -2.f * ux : 0.f, ay = live ? -2.f * uy : 0.f,
              az = live ? -2.f * uz : 0.f;
  const float lo_i = live ? lo_band - uu : -INFINITY;
  const float hi_i = live ? hi_band - uu : -INFINITY;
  // far pairs: d above this
  const float near_i = live ? near2 - uu : INFINITY;
  // box of the group's centre atoms relative to the cell centre, rounded outwards
  float glo[3], ghi[3];
  {
    const double p[3] = {xi, yi, zi}, o[3] = {ox, oy, oz};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      glo[d] = live ? __double2float_rd(__dsub_rd(p[d], o[d])) : INFINITY;
      ghi[d] = live ? __double2float_ru(__dsub_ru(p[d], o[d])) : -INFINITY;
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1)
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        glo[d] = fminf(glo[d], __shfl_xor_sync(0xffffffffu, glo[d], s));
        ghi[d] = fmaxf(ghi[d], __shfl_xor_sync(0xffffffffu, ghi[d], s));
      }
  }
  int cnt = 0, nback = 0;  // candidates found, entries written to the back
  int* row = nbrs + (size_t)i * cap;
  for (int s = 0; s < 27; ++s) {
    // stencil order of ComputeFullNeighborStencilCellOnTheFly:
    // offsets (s%3-1, (s/3)%3-1, s/9-1)
    int nx = cx + s % 3 - 1, ny = cy + (s / 3) % 3 - 1, nz = cz + s / 9 - 1;
    double shx = 0.0, shy = 0.0, shz = 0.0;
    if (nx < 0) { nx += dimx; shx = -b.len[0]; } else if (nx >= dimx) { nx -= dimx; shx = b.len[0]; }
    if (ny < 0) { ny += dimy; shy = -b.len[1]; } else if (ny >= dimy) { ny -= dimy; shy = b.len[1]; }
    if (nz < 0) { nz += dimz; shz = -b.len[2]; } else if (nz >= dimz) { nz -= dimz; shz = b.len[2]; }
    const int nc = (nz * dimy + ny) * dimx + nx;
    const int ncs = cell_start[nc], nce = cell_start[nc + 1];
    const int nch = (nce - ncs + 31) >> 5;
    const int nb = chunk_base(nc, ncs);
    const double dx = shx - ox, dy = shy - oy, dz = shz - oz;
    const double dxl = __dsub_rd(shx, ox), dyl = __dsub_rd(shy, oy), dzl = __dsub_rd(shz, oz);
    const double dxh = __dsub_ru(shx, ox), dyh = __dsub_ru(shy, oy), dzh = __dsub_ru(shz, oz);
    for (int kb = 0; kb < nch; kb += 32) {
      bool near = false;
      if (kb + lane < nch) {  // lower bound of the box-box distance
        const float4 bl = box_lo[nb + kb + lane], bh = box_hi[nb + kb + lane];
        const float clx = __double2float_rd(__dadd_rd((double)bl.x, dxl));
        const float cly = __double2float_rd(__dadd_rd((double)bl.y, dyl));
        const float clz = __double2float_rd(__dadd_rd((double)bl.z, dzl));
        const float chx = __double2float_ru(__dadd_ru((double)bh.x, dxh));
        const float chy = __double2float_ru(__dadd_ru((double)bh.y, dyh));
        const float chz = __double2float_ru(__dadd_ru((double)bh.z, dzh));
        const float gx = fmaxf(0.f, fmaxf(__fsub_rd(clx, ghi[0]), __fsub_rd(glo[0], chx)));
        const float gy = fmaxf(0.f, fmaxf(__fsub_rd(cly, ghi[1]), __fsub_rd(glo[1], chy)));
        const float gz = fmaxf(0.f, fmaxf(__fsub_rd(clz, ghi[2]), __fsub_rd(glo[2], chz)));
        const float d2 = __fadd_rd(__fadd_rd(__fmul_rd(gx, gx), __fmul_rd(gy, gy)), __fmul_rd(gz, gz));
        near = d2 < cut2_up;
      }
      unsigned m = __ballot_sync(0xffffffffu, near);
      while (m) {
        const int k = kb + __ffs(m) - 1;
        m &= m - 1;
        const int first = ncs + 32 * k;
        float4 v = make_float4(0.f, 0.f, INFINITY, INFINITY);  // empty slot: never a hit
        if (first + lane < nce) {
          const int a = first + lane;
          v.x = (float)(x[a] + dx);
          v.y = (float)(y[a] + dy);
          v.z = (float)(z[a] + dz);
          v.w = fmaf(v.x, v.x, fmaf(v.y, v.y, v.z * v.z));
        }
        __syncwarp();  // the previous chunk's readers are done
        buf[warp][lane] = v;
        __syncwarp();
        unsigned acc = 0, maybe = 0, farm = 0;  // farm: build distance certainly >= r_near
#pragma unroll
        for (int t = 0; t < 32; ++t) {
          const float4 q = buf[warp][t];  // broadcast
          const float d = fmaf(ax, q.x, fmaf(ay, q.y, fmaf(az, q.z, q.w)));
          acc |= d < lo_i ? 1u << t : 0u;
          maybe |= d < hi_i ? 1u << t : 0u;
          if (SPLIT) farm |= d > near_i ? 1u << t : 0u;
        }
        if (nc == c && k == g) {  // the centre atom itself
          acc &= ~(1u << lane);
          maybe &= ~(1u << lane);
        }
        unsigned unsure = maybe & ~acc;
        if (__any_sync(0xffffffffu, unsure != 0)) {  // rare: the FP64 predicate decides
          while (unsure) {
            const int t = __ffs(unsure) - 1;
            unsure &= unsure - 1;
            const int j = first + t;
            if (dist2_list(b, xi, yi, zi, x[j], y[j], z[j]) < cut2) acc |= 1u << t;
          }
        }
        if (cnt + __popc(acc) <= cap) {
          // every hit of the chunk fits: next front and back slots as offsets,
          // the counts recovered after the loop
          int foff = cnt - nback, boff = cap - 1 - nback;
          while (acc) {  // hits in cell order, each lane into its own row
            const int t = __ffs(acc) - 1;
            acc &= acc - 1;
            const bool to_back = SPLIT && ((farm >> t) & 1u);
            row[to_back ? boff : foff] = first + t;
            boff -= to_back;
            foff += !to_back;
          }
          nback = cap - 1 - boff;
          cnt = foff + nback;
        }
        while (acc) {  // the row fills up: stop storing at cap entries
          const int t = __ffs(acc) - 1;
          acc &= acc - 1;
          // one store to the front or the back of the row (no branch)
          const bool to_back = SPLIT && ((farm >> t) & 1u);
          if (cnt < cap) row[to_back ? cap - 1 - nback : cnt - nback] = first + t;
          nback += (cnt < cap) & to_back;
          ++cnt;
        }
      }
    }
  }
  if (live) {
    count[i] = cnt;
    if (SPLIT) far[i] = nback;
    if (cnt > cap) atomicOr(overflow, 1);
  }
  if (total) {  // the warp's rows (cnt is 0 on lanes without a centre atom)
    const int s = __reduce_add_sync(0xffffffffu, cnt);
    if (lane == 0) atomicAdd((unsigned long long*)total, (unsigned long long)s);
  }
}

// ---------------------------------------------------------------------------
// Candidate rows for boxes with fewer than three cells of edge cut_off + skin
// along some axis (edge between two and three times cut_off + skin): every
// atom j != i is tested with the reference's FP64 predicate (CaculateDistance:
// i minus j, single-shift minimum image, no FMA), so each pair is listed once.
// (The reference's cells have edge (cut_off + skin) / c, c = 1 for a Verlet
// list and ceil((cut_off + skin) / r_core) for RBL (linked_cell_locator.cpp:
// 26-40), and its (2c + 1)^3 stencil wraps onto the same cell more than once
// along an axis with fewer than 2c + 1 cells, WrapFullNeighborStencilIndex in
// full_neighbor_list_op.hip.cu:9-80, listing those pairs repeatedly.)  A warp
// per atom; hits are appended in index order through a ballot prefix, far
// pairs (see FarSplit) to the back.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128)
k_full_list_small(DBox b, double cut2, double near2, int n, const double* __restrict__ x,
                  const double* __restrict__ y, const double* __restrict__ z, int cap,
                  int* __restrict__ count, int* __restrict__ nbrs, int* __restrict__ overflow,
                  int* __restrict__ far, long long* __restrict__ total) {
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * 4 + (threadIdx.x >> 5);
  if (i >= n) return;
  const unsigned lt = (1u << lane) - 1u;
  const double xi = x[i], yi = y[i], zi = z[i];
  int nf = 0, nb = 0;  // near (front) and far (back) entries found
  int* row = nbrs + (size_t)i * cap;
  for (int j0 = 0; j0 < n; j0 += 32) {
    const int j = j0 + lane;
    double d2 = INFINITY;
    if (j < n && j != i) d2 = dist2_list(b, xi, yi, zi, x[j], y[j], z[j]);
    const bool hit = d2 < cut2;
    const bool is_far = hit && !(d2 < near2);
    const unsigned mh = __ballot_sync(0xffffffffu, hit && !is_far);
    const unsigned mf = __ballot_sync(0xffffffffu, is_far);
    if (hit && !is_far) {
      const int pos = nf + __popc(mh & lt);
      if (pos < cap) row[pos] = j;
    } else if (is_far) {
      const int k = nb + __popc(mf & lt);
      if (k < cap) row[cap - 1 - k] = j;
    }
    nf += __popc(mh);
    nb += __popc(mf);
  }
  if (lane == 0) {
    count[i] = nf + nb;
    if (far) far[i] = nb;
    if (nf + nb > cap) atomicOr(overflow, 1);
    if (total) atomicAdd((unsigned long long*)total, (unsigned long long)(nf + nb));
  }
}

int launch_full_list_small(const DBox& b, double cutoff, int n, const double* x, const double* y,
                           const double* z, int cap, int* count, int* nbrs, int* overflow,
                           cudaStream_t st, const FarSplit* split, long long* total) {
  if (n <= 0) return RBX_OK;
  // near threshold raised by 1e-9 relative: FP64 rounding never moves a pair
  // that could come within r_core before the next rebuild to the far segment
  const double near2 =
      split ? split->r_near * split->r_near * (1.0 + 1e-9) : (double)INFINITY;
  k_full_list_small<<<(n + 3) / 4, 128, 0, st>>>(b, cutoff * cutoff, near2, n, x, y, z, cap,
                                                 count, nbrs, overflow,
                                                 split ? split->far : nullptr, total);
  count_launch();
  return check_launch("full_list_small");
}

// ---------------------------------------------------------------------------
// Gathers / scatters and integration.
// ---------------------------------------------------------------------------
__global__ void k_fill_i32(int n, int* __restrict__ p, int v) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// Zero the cell counts; with book (an engine rebuild), also its flags and
// candidate total, and count the rebuild.
__global__ void k_cells_reset(int ncell, int* __restrict__ counts, RebuildBook book) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < ncell; i += gridDim.x * blockDim.x)
    counts[i] = 0;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (book.flags) book.flags[0] = book.flags[1] = 0;
    if (book.total) *book.total = 0;
    if (book.counter) *book.counter += 1;
  }
}

// One pass over a set of per-atom arrays: dst[a][i] = src[a][perm[i]] (perm
// null: a plain copy).  The set's pointers are kernel parameters, so one
// launch moves every array of the rebuild.
__global__ void k_move_set(int n, const int* __restrict__ perm, ArraySet s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = perm ? perm[i] : i;
#pragma unroll
  for (int a = 0; a < ArraySet::kMaxF64; ++a)
    if (a < s.nf64) s.dst_f64[a][i] = s.src_f64[a][p];
#pragma unroll
  for (int a = 0; a < ArraySet::kMaxI32; ++a)
    if (a < s.ni32) s.dst_i32[a][i] = s.src_i32[a][p];
#pragma unroll
  for (int a = 0; a < ArraySet::kMaxU64; ++a)
    if (a < s.nu64) s.dst_u64[a][i] = s.src_u64[a][p];
}

// Per-step decision inside the step graph: advance the device epoch and take
// the rebuild branch when some atom moved more than skin / 2 since the last
// rebuild (max_d2 holds the bits of a non-negative double).
__global__ void k_step_decide(const unsigned long long* __restrict__ max_d2, double thr2,
                              int* __restrict__ epoch, cudaGraphConditionalHandle rebuild) {
  *epoch += 1;
  cudaGraphSetConditional(rebuild, __longlong_as_double((long long)*max_d2) > thr2 ? 1u : 0u);
}

__global__ void k_zero_u64(unsigned long long* __restrict__ p) { *p = 0ULL; }

__global__ void k_add_i32(int* __restrict__ p, int v) { *p += v; }

template <typename T>
__global__ void k_gather(int n, const int* __restrict__ perm, const T* __restrict__ src,
                         T* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[perm[i]];
}
template <typename T>
__global__ void k_scatter(int n, const int* __restrict__ idx, const T* __restrict__ src,
                          T* __restrict__ dst) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[idx[i]] = src[i];
}

// UpdateVelocity (update_velocity_op.hip.cu:5-28), fmt2v folded into inv_mass.
__global__ void k_kick(int n, const double* __restrict__ fx, const double* __restrict__ fy,
                       const double* __restrict__ fz, const int* __restrict__ type,
                       const double* __restrict__ inv_mass, double half_dt,
                       double* __restrict__ vx, double* __restrict__ vy,
                       double* __restrict__ vz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double s = inv_mass[type[i]] * half_dt;
  vx[i] += fx[i] * s;
  vy[i] += fy[i] * s;
  vz[i] += fz[i] * s;
}

// UpdatePositionFlag + ApplyPBC (update_position_op.hip.cu:22-46, box.h:133-169),
// fused with the skin check DisplacementSq (base_neighbor_list_builder.cpp:102-116)
// and, for the mixed form, the fixed-point record {ux, uy, uz, q_f32}.  With
// kick.fx the first half kick of the step comes first (k_kick's arithmetic).
// With decide.ctr (inside a step graph) the last block to finish takes the
// step's rebuild decision as k_step_decide does, then clears the maximum and
// the block counter for the next step.
struct DriftArgs {
  DBox b;
  int n;
  double dt;
  double *x, *y, *z, *vx, *vy, *vz;
  const double *x0, *y0, *z0;
  unsigned long long* max_d2;
  uint4* atoms;
  const double* q;
  ImageRefs img;
  Pos3 old;
  KickArgs kick;
  DecideArgs decide;
};

// Block bx of a grid of gx blocks.
__device__ __forceinline__ void drift_body(const DriftArgs& A, int bx, int gx) {
  const DBox& b = A.b;
  const int n = A.n;
  const double dt = A.dt;
  double* __restrict__ x = A.x;
  double* __restrict__ y = A.y;
  double* __restrict__ z = A.z;
  double* __restrict__ vx = A.vx;
  double* __restrict__ vy = A.vy;
  double* __restrict__ vz = A.vz;
  const double* __restrict__ x0 = A.x0;
  const double* __restrict__ y0 = A.y0;
  const double* __restrict__ z0 = A.z0;
  unsigned long long* __restrict__ max_d2 = A.max_d2;
  uint4* __restrict__ atoms = A.atoms;
  const double* __restrict__ q = A.q;
  const ImageRefs& img = A.img;
  const Pos3& old = A.old;
  const KickArgs& kick = A.kick;
  const DecideArgs& decide = A.decide;
  const int i = bx * blockDim.x + threadIdx.x;
  double d2 = 0.0;
  if (i < n) {
    if (old.x) {  // positions before the drift, for SHAKE
      old.x[i] = x[i];
      old.y[i] = y[i];
      old.z[i] = z[i];
    }
    double v[3] = {vx[i], vy[i], vz[i]};
    if (kick.fx) {
      const double s = kick.inv_mass[kick.type[i]] * kick.half_dt;
      v[0] += kick.fx[i] * s;
      v[1] += kick.fy[i] * s;
      v[2] += kick.fz[i] * s;
      vx[i] = v[0];
      vy[i] = v[1];
      vz[i] = v[2];
    }
    double p[3] = {x[i] + v[0] * dt, y[i] + v[1] * dt, z[i] + v[2] * dt};
    for (int d = 0; d < 3; ++d) {  // periodic wrap, counted in the image flags
      int w = 0;
      if (p[d] >= b.lo[d] + b.len[d]) {
        p[d] -= b.len[d];
        w = 1;
      }
      if (p[d] < b.lo[d]) {
        p[d] += b.len[d];
        w = -1;
      }
      if (w && img.c[d]) img.c[d][i] += w;
    }
    x[i] = p[0];
    y[i] = p[1];
    z[i] = p[2];
    if (max_d2) {
      const double ddx = min_image1(p[0] - x0[i], b.len[0], b.half[0]);
      const double ddy = min_image1(p[1] - y0[i], b.len[1], b.half[1]);
      const double ddz = min_image1(p[2] - z0[i], b.len[2], b.half[2]);
      d2 = ddx * ddx + ddy * ddy + ddz * ddz;
    }
    if (atoms) {
      uint4 a;
      a.x = to_fixed(p[0], b.lo[0], 4294967296.0 / b.len[0]);
      a.y = to_fixed(p[1], b.lo[1], 4294967296.0 / b.len[1]);
      a.z = to_fixed(p[2], b.lo[2], 4294967296.0 / b.len[2]);
      a.w = __float_as_uint((float)q[i]);
      atoms[i] = a;
    }
  }
  if (max_d2) {  // block maximum, then one atomic per block
    __shared__ unsigned long long s_max[32];
    unsigned long long bits = (unsigned long long)__double_as_longlong(d2);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long t = __shfl_xor_sync(0xffffffffu, bits, o);
      bits = t > bits ? t : bits;
    }
    if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = bits;
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 1; w < (int)(blockDim.x >> 5); ++w) bits = s_max[w] > bits ? s_max[w] : bits;
      atomicMax(max_d2, bits);
    }
  }
  if (decide.ctr) {
    __syncthreads();  // the block's maximum is folded in (by thread 0, below)
    if (threadIdx.x == 0) {
      __threadfence();
      if (atomicAdd(decide.ctr, 1u) == (unsigned)gx - 1) {  // the last block
        __threadfence();
        const unsigned long long m = atomicAdd(max_d2, 0ULL);
        *decide.epoch += 1;
        cudaGraphSetConditional(decide.cond,
                                __longlong_as_double((long long)m) > decide.thr2 ? 1u : 0u);
        *max_d2 = 0ULL;
        *decide.ctr = 0u;
      }
    }
  }
}

__global__ void __launch_bounds__(256) k_drift(DriftArgs a) {
  drift_body(a, blockIdx.x, gridDim.x);
}

__global__ void __launch_bounds__(256)
k_drift_batch(const DriftArgs* __restrict__ a, const int* __restrict__ start, int nrep) {
  const int r = batch_replica(start, nrep, blockIdx.x);
  const int b0 = __ldg(start + r);
  drift_body(a[r], blockIdx.x - b0, __ldg(start + r + 1) - b0);
}

__global__ void k_to_fixed(DBox b, int n, const double* __restrict__ x,
                           const double* __restrict__ y, const double* __restrict__ z,
                           const double* __restrict__ q, uint4* __restrict__ atoms) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint4 a;
  a.x = to_fixed(x[i], b.lo[0], 4294967296.0 / b.len[0]);
  a.y = to_fixed(y[i], b.lo[1], 4294967296.0 / b.len[1]);
  a.z = to_fixed(z[i], b.lo[2], 4294967296.0 / b.len[2]);
  a.w = __float_as_uint((float)q[i]);
  atoms[i] = a;
}

__global__ void k_max_disp(DBox b, int n, const double* __restrict__ x,
                           const double* __restrict__ y, const double* __restrict__ z,
                           const double* __restrict__ x0, const double* __restrict__ y0,
                           const double* __restrict__ z0, unsigned long long* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double d2 = 0.0;
  if (i < n) {
    double dx = x[i] - x0[i], dy = y[i] - y0[i], dz = z[i] - z0[i];
    // MinImageDistance_while (box.h:75-97) as one bounded step: the nearest
    // image by rint, so a non-finite coordinate cannot spin the loop.
    dx -= b.len[0] * rint(dx / b.len[0]);
    dy -= b.len[1] * rint(dy / b.len[1]);
    dz -= b.len[2] * rint(dz / b.len[2]);
    d2 = dx * dx + dy * dy + dz * dz;
  }
  warp_max_atomic(d2, out);
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
size_t cells_scratch_bytes(int n, int ncell) {
  // counts[ncell] + fill[ncell] + cell[n] + sub[n] + tmp[n], 256-byte aligned pieces
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  return al(sizeof(int) * (size_t)ncell) * 2 + al(sizeof(int) * (size_t)n) * 3;
}

int launch_cells_sort(const DBox& b, const int dims[3], int n, const double* x, const double* y,
                      const double* z, int* perm, int* cell_of_sorted, int* cell_start,
                      void* scratch, int* status, cudaStream_t st, const RebuildBook* book) {
  const int ncell = dims[0] * dims[1] * dims[2];
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  char* p = (char*)scratch;
  int* counts = (int*)p;
  p += al(sizeof(int) * (size_t)ncell);
  int* fill = (int*)p;
  p += al(sizeof(int) * (size_t)ncell);
  int* cell = (int*)p;
  p += al(sizeof(int) * (size_t)n);
  unsigned* sub = (unsigned*)p;
  p += al(sizeof(int) * (size_t)n);
  unsigned* tmp = (unsigned*)p;
  k_cells_reset<<<grid_for(ncell, 256, sm_count() * 4), 256, 0, st>>>(
      ncell, counts, book ? *book : RebuildBook{nullptr, nullptr, nullptr});
  count_launch();
  if (n > 0) {
    CellGeom g;
    for (int d = 0; d < 3; ++d) {
      g.edge[d] = b.len[d] / dims[d];
      g.inv[d] = 1.0 / g.edge[d];
    }
    k_cell_assign<<<(n + 255) / 256, 256, 0, st>>>(b, g, dims[0], dims[1], dims[2], n, x, y, z,
                                                   cell, sub, counts);
    count_launch();
  }
  k_cell_scan<<<1, 1024, 0, st>>>(ncell, counts, cell_start, fill);
  count_launch();
  if (n > 0) {
    k_cell_scatter<<<(n + 255) / 256, 256, 0, st>>>(n, cell, sub, fill, tmp);
    count_launch();
  }
  k_cell_segsort<<<ncell, 512, 0, st>>>(ncell, n, cell_start, tmp, perm, cell_of_sorted, status);
  count_launch();
  return check_launch("cells_sort");
}

size_t full_list_scratch_bytes(int n, int ncell) {
  const size_t t = (size_t)full_list_table_size(n, ncell);
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  return al(sizeof(float4) * t) * 2 + al(sizeof(int) * t);
}

int launch_full_list(const DBox& b, const int dims[3], double cutoff, int n, const double* x,
                     const double* y, const double* z, const int* cell_start, int cap,
                     int* count, int* nbrs, int* overflow, void* scratch, cudaStream_t st,
                     const FarSplit* split, long long* total) {
  const int ncell = dims[0] * dims[1] * dims[2];
  if (n <= 0) return RBX_OK;
  if (dims[0] < 3 || dims[1] < 3 || dims[2] < 3)
    return launch_full_list_small(b, cutoff, n, x, y, z, cap, count, nbrs, overflow, st, split,
                                  total);
  const double cut2 = cutoff * cutoff;
  double emax = 0.0;
  for (int d = 0; d < 3; ++d) emax = fmax(emax, b.len[d] / dims[d]);
  // FP32 screening error of |v|^2 - 2 u.v against C - |u|^2, with u (|u_d| <=
  // e/2) and v (|v_d| <= 3e/2) rounded once to FP32 relative to the centre
  // cell's centre: coordinate rounding moves |d|^2 by at most
  // 4 sqrt(3) r e 2^-24, and the roundings of |v|^2, the three FMAs, |u|^2 and
  // C - |u|^2 by at most (60 e^2 + 3 r^2) 2^-24 (e = largest cell edge,
  // r = cutoff).  Pairs within twice that of the cutoff take the FP64 path.
  const double err =
      (4.0 * sqrt(3.0) * cutoff * emax + 60.0 * emax * emax + 3.0 * cut2) / 16777216.0;
  const double band = 2.0 * err;
  const float lo_band = (float)(cut2 - band), hi_band = (float)(cut2 + band);
  float cut2_up = (float)cut2;  // rounded up
  if ((double)cut2_up < cut2) cut2_up = nextafterf(cut2_up, INFINITY);
  const int t = full_list_table_size(n, ncell);
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  char* p = (char*)scratch;
  float4* box_lo = (float4*)p;
  float4* box_hi = (float4*)(p + al(sizeof(float4) * t));
  int* cell_of = (int*)(p + 2 * al(sizeof(float4) * t));
  k_chunk_boxes<<<ncell, 128, 0, st>>>(x, y, z, cell_start, box_lo, box_hi, cell_of);
  count_launch();
  // far threshold in r^2, raised by the FP32 error of the test value
  const float near2 = split ? (float)(split->r_near * split->r_near + band) : INFINITY;
  if (split)
    k_full_list<true><<<(t + NL_WARPS - 1) / NL_WARPS, NL_BLOCK, 0, st>>>(
        b, dims[0], dims[1], dims[2], cut2, cut2_up, lo_band, hi_band, t, x, y, z, cell_start,
        box_lo, box_hi, cell_of, cap, count, nbrs, overflow, near2, split->far, total);
  else
    k_full_list<false><<<(t + NL_WARPS - 1) / NL_WARPS, NL_BLOCK, 0, st>>>(
        b, dims[0], dims[1], dims[2], cut2, cut2_up, lo_band, hi_band, t, x, y, z, cell_start,
        box_lo, box_hi, cell_of, cap, count, nbrs, overflow, near2, nullptr, total);
  count_launch();
  return check_launch("full_list");
}

// dst[a][idx[i]] = src[a][i] for every array of the set (one launch).
__global__ void k_scatter_set(int n, const int* __restrict__ idx, ArraySet s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int p = idx[i];
#pragma unroll
  for (int a = 0; a < ArraySet::kMaxF64; ++a)
    if (a < s.nf64) s.dst_f64[a][p] = s.src_f64[a][i];
#pragma unroll
  for (int a = 0; a < ArraySet::kMaxI32; ++a)
    if (a < s.ni32) s.dst_i32[a][p] = s.src_i32[a][i];
#pragma unroll
  for (int a = 0; a < ArraySet::kMaxU64; ++a)
    if (a < s.nu64) s.dst_u64[a][p] = s.src_u64[a][i];
}

int launch_scatter_set(int n, const int* idx, const ArraySet& set, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_scatter_set<<<(n + 255) / 256, 256, 0, st>>>(n, idx, set);
  count_launch();
  return check_launch("scatter_set");
}

int launch_move_set(int n, const int* perm, const ArraySet& set, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_move_set<<<(n + 255) / 256, 256, 0, st>>>(n, perm, set);
  count_launch();
  return check_launch("move_set");
}

int launch_fill_i32(int n, int* p, int v, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_fill_i32<<<grid_for(n, 256, sm_count() * 4), 256, 0, st>>>(n, p, v);
  count_launch();
  return check_launch("fill_i32");
}

int launch_zero_u64(unsigned long long* p, cudaStream_t st) {
  k_zero_u64<<<1, 1, 0, st>>>(p);
  count_launch();
  return check_launch("zero_u64");
}

int launch_add_i32(int* p, int v, cudaStream_t st) {
  k_add_i32<<<1, 1, 0, st>>>(p, v);
  count_launch();
  return check_launch("add_i32");
}

int launch_step_decide(const unsigned long long* max_d2, double thr2, int* epoch,
                       cudaGraphConditionalHandle rebuild, cudaStream_t st) {
  k_step_decide<<<1, 1, 0, st>>>(max_d2, thr2, epoch, rebuild);
  count_launch();
  return check_launch("step_decide");
}

int launch_gather_f64(int n, const int* perm, const double* src, double* dst, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_gather<double><<<(n + 255) / 256, 256, 0, st>>>(n, perm, src, dst);
  count_launch();
  return check_launch("gather_f64");
}
int launch_gather_i32(int n, const int* perm, const int* src, int* dst, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_gather<int><<<(n + 255) / 256, 256, 0, st>>>(n, perm, src, dst);
  count_launch();
  return check_launch("gather_i32");
}
int launch_gather_u64(int n, const int* perm, const unsigned long long* src,
                      unsigned long long* dst, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_gather<unsigned long long><<<(n + 255) / 256, 256, 0, st>>>(n, perm, src, dst);
  count_launch();
  return check_launch("gather_u64");
}
int launch_scatter_f64(int n, const int* idx, const double* src, double* dst, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_scatter<double><<<(n + 255) / 256, 256, 0, st>>>(n, idx, src, dst);
  count_launch();
  return check_launch("scatter_f64");
}
int launch_scatter_i32(int n, const int* idx, const int* src, int* dst, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_scatter<int><<<(n + 255) / 256, 256, 0, st>>>(n, idx, src, dst);
  count_launch();
  return check_launch("scatter_i32");
}

int launch_kick(int n, const double* fx, const double* fy, const double* fz, const int* type,
                const double* inv_mass, double half_dt, double* vx, double* vy, double* vz,
                cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_kick<<<(n + 255) / 256, 256, 0, st>>>(n, fx, fy, fz, type, inv_mass, half_dt, vx, vy, vz);
  count_launch();
  return check_launch("kick");
}

int launch_drift(const DBox& b, int n, double dt, double* x, double* y, double* z,
                 double* vx, double* vy, double* vz, const double* x0,
                 const double* y0, const double* z0, unsigned long long* max_d2_bits,
                 uint4* atoms, const double* q, ImageRefs img, Pos3 old, cudaStream_t st,
                 const KickArgs* kick, const DecideArgs* decide) {
  if (n <= 0) return RBX_OK;
  DriftArgs a;
  a.b = b;
  a.n = n;
  a.dt = dt;
  a.x = x;
  a.y = y;
  a.z = z;
  a.vx = vx;
  a.vy = vy;
  a.vz = vz;
  a.x0 = x0;
  a.y0 = y0;
  a.z0 = z0;
  a.max_d2 = max_d2_bits;
  a.atoms = atoms;
  a.q = q;
  a.img = img;
  a.old = old;
  a.kick = kick ? *kick : KickArgs{nullptr, nullptr, nullptr, nullptr, nullptr, 0.0};
  a.decide = decide ? *decide : DecideArgs{nullptr, 0.0, nullptr, {}};
  const int grid = (n + 255) / 256;
  if (batch_recorder()) return record_phase(PH_DRIFT, 0, grid, 256, 0, &a, sizeof a);
  k_drift<<<grid, 256, 0, st>>>(a);
  count_launch();
  return check_launch("drift");
}

int launch_drift_batch(const void* args, const int* start, int nrep, int total, cudaStream_t st) {
  k_drift_batch<<<total, 256, 0, st>>>(static_cast<const DriftArgs*>(args), start, nrep);
  count_launch();
  return check_launch("drift_batch");
}

int launch_to_fixed(const DBox& b, int n, const double* x, const double* y, const double* z,
                    const double* q, uint4* atoms, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_to_fixed<<<(n + 255) / 256, 256, 0, st>>>(b, n, x, y, z, q, atoms);
  count_launch();
  return check_launch("to_fixed");
}

int launch_max_disp(const DBox& b, int n, const double* x, const double* y, const double* z,
                    const double* x0, const double* y0, const double* z0,
                    unsigned long long* max_d2_bits, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_max_disp<<<(n + 255) / 256, 256, 0, st>>>(b, n, x, y, z, x0, y0, z0, max_d2_bits);
  count_launch();
  return check_launch("max_disp");
}

}  // namespace rbx
