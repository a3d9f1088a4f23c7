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
// CTA per cell stages the 27 stencil cells in shared memory as FP32
// coordinates relative to the centre cell (periodic images pre-shifted), one
// warp per centre atom screens them in FP32 and settles only the pairs inside
// a guard band around the cutoff with the reference's FP64 predicate, so the
// list is bit-identical (as a set) to the FP64 reference list.
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

__global__ void k_cell_assign(DBox b, int dx, int dy, int dz, int n, const double* __restrict__ x,
                              const double* __restrict__ y, const double* __restrict__ z,
                              int* __restrict__ cell, unsigned* __restrict__ sub,
                              int* __restrict__ counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double fx = (x[i] - b.lo[0]) * (dx / b.len[0]);
  const double fy = (y[i] - b.lo[1]) * (dy / b.len[1]);
  const double fz = (z[i] - b.lo[2]) * (dz / b.len[2]);
  const int cx = cell_coord(x[i], b.lo[0], dx / b.len[0], dx);
  const int cy = cell_coord(y[i], b.lo[1], dy / b.len[1], dy);
  const int cz = cell_coord(z[i], b.lo[2], dz / b.len[2], dz);
  const int c = (cz * dy + cy) * dx + cx;
  cell[i] = c;
  auto sub4 = [](double f, int c0) {
    int v = (int)floor((f - c0) * 4.0);
    return (unsigned)(v < 0 ? 0 : (v > 3 ? 3 : v));
  };
  sub[i] = n < (1 << SUB_SHIFT) ? morton2(sub4(fx, cx), sub4(fy, cy), sub4(fz, cz)) : 0u;
  atomicAdd(counts + c, 1);
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
  tmp[atomicAdd(fill + cell[i], 1)] = (sub[i] << SUB_SHIFT) | (unsigned)i;
}

// One block per cell: bitonic sort of the cell's keys (sub-cell, old index).
__global__ void __launch_bounds__(512)
k_cell_segsort(int ncell, int n, const int* __restrict__ start, const unsigned* __restrict__ tmp,
               int* __restrict__ perm, int* __restrict__ cell_of_sorted, int* __restrict__ status) {
  __shared__ unsigned s[SEG_MAX];
  const int c = blockIdx.x;
  const int a = start[c], cnt = start[c + 1] - a;
  if (cnt > SEG_MAX) {
    if (threadIdx.x == 0) atomicOr(status, 2);
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
  const unsigned mask = n < (1 << SUB_SHIFT) ? (1u << SUB_SHIFT) - 1u : 0xffffffffu;
  for (int t = threadIdx.x; t < cnt; t += blockDim.x) {
    perm[a + t] = (int)(s[t] & mask);
    cell_of_sorted[a + t] = c;
  }
}

// ---------------------------------------------------------------------------
// Candidate list: CTA per cell.  Stencil cells are staged in shared memory,
// each padded to whole 32-atom chunks; every chunk gets a bounding box, and a
// centre atom tests only the chunks whose box comes within the cutoff.
// ---------------------------------------------------------------------------
constexpr int NL_BLOCK = 256;
constexpr int NL_WARPS = NL_BLOCK / 32;
constexpr int NL_STAGE = 2048;   // staged stencil slots per pass (multiple of 32)
constexpr int NL_CHUNKS = NL_STAGE / 32;
constexpr int NL_CENTER = 1024;  // centre-cell atoms tracked per CTA

__global__ void __launch_bounds__(NL_BLOCK)
k_full_list(DBox b, int dimx, int dimy, int dimz, double cut2, float lo_band, float hi_band,
            int n, const double* __restrict__ x, const double* __restrict__ y,
            const double* __restrict__ z, const int* __restrict__ cell_start, int cap,
            int* __restrict__ count, int* __restrict__ nbrs, int* __restrict__ overflow) {
  __shared__ float sx[NL_STAGE], sy[NL_STAGE], sz[NL_STAGE];
  __shared__ int sj[NL_STAGE];
  __shared__ float bb[6][NL_CHUNKS];  // chunk boxes: min xyz, max xyz
  __shared__ int s_cnt[NL_CENTER];
  __shared__ int s_cbeg[27], s_ccnt[27];
  __shared__ double s_shift[27][3];
  const int c = blockIdx.x;
  const int cz = c / (dimx * dimy), cy = (c / dimx) % dimy, cx = c % dimx;
  const double ex = b.len[0] / dimx, ey = b.len[1] / dimy, ez = b.len[2] / dimz;
  const double ox = b.lo[0] + cx * ex, oy = b.lo[1] + cy * ey, oz = b.lo[2] + cz * ez;
  const int cs = cell_start[c], ce = cell_start[c + 1];
  const int ncen = ce - cs;
  if (ncen > NL_CENTER) {
    if (threadIdx.x == 0) atomicOr(overflow, 2);
    return;
  }
  if (threadIdx.x < 27) {
    // stencil order of ComputeFullNeighborStencilCellOnTheFly:
    // offsets (s%3-1, (s/3)%3-1, s/9-1)
    const int s = threadIdx.x;
    const int o[3] = {s % 3 - 1, (s / 3) % 3 - 1, s / 9 - 1};
    const int cc[3] = {cx, cy, cz};
    const int dims[3] = {dimx, dimy, dimz};
    int nc[3];
    for (int d = 0; d < 3; ++d) {
      int v = cc[d] + o[d];
      double sh = 0.0;
      if (v < 0) {
        v += dims[d];
        sh = -b.len[d];
      } else if (v >= dims[d]) {
        v -= dims[d];
        sh = b.len[d];
      }
      nc[d] = v;
      s_shift[s][d] = sh;
    }
    const int cell = (nc[2] * dimy + nc[1]) * dimx + nc[0];
    s_cbeg[s] = cell_start[cell];
    s_ccnt[s] = cell_start[cell + 1] - cell_start[cell];
  }
  for (int t = threadIdx.x; t < ncen; t += NL_BLOCK) s_cnt[t] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  int s0 = 0;
  while (s0 < 27) {
    // greedy group of stencil cells whose padded sizes fit the stage
    int s1 = s0, tot = 0;
    while (s1 < 27 && tot + ((s_ccnt[s1] + 31) & ~31) <= NL_STAGE) {
      tot += (s_ccnt[s1] + 31) & ~31;
      ++s1;
    }
    if (s1 == s0) {  // a single cell larger than the stage
      if (threadIdx.x == 0) atomicOr(overflow, 2);
      return;
    }
    int off = 0;
    for (int s = s0; s < s1; ++s) {
      const int beg = s_cbeg[s], cnt = s_ccnt[s], pad = (cnt + 31) & ~31;
      const double shx = s_shift[s][0] - ox, shy = s_shift[s][1] - oy, shz = s_shift[s][2] - oz;
      for (int t = threadIdx.x; t < pad; t += NL_BLOCK) {
        if (t < cnt) {
          const int j = beg + t;
          sx[off + t] = (float)(x[j] + shx);
          sy[off + t] = (float)(y[j] + shy);
          sz[off + t] = (float)(z[j] + shz);
          sj[off + t] = j;
        } else {  // padding slot: never within the cutoff
          sx[off + t] = 1e30f;
          sy[off + t] = 1e30f;
          sz[off + t] = 1e30f;
          sj[off + t] = -1;
        }
      }
      off += pad;
    }
    __syncthreads();
    const int nch = tot / 32;
    for (int ch = warp; ch < nch; ch += NL_WARPS) {
      const int t = ch * 32 + lane;
      const bool real = sj[t] >= 0;
      float lo[3] = {real ? sx[t] : 1e30f, real ? sy[t] : 1e30f, real ? sz[t] : 1e30f};
      float hi[3] = {real ? sx[t] : -1e30f, real ? sy[t] : -1e30f, real ? sz[t] : -1e30f};
#pragma unroll
      for (int o = 16; o > 0; o >>= 1)
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          lo[d] = fminf(lo[d], __shfl_xor_sync(0xffffffffu, lo[d], o));
          hi[d] = fmaxf(hi[d], __shfl_xor_sync(0xffffffffu, hi[d], o));
        }
      if (lane < 3) {
        bb[lane][ch] = lo[lane];
        bb[3 + lane][ch] = hi[lane];
      }
    }
    __syncthreads();
    for (int li = warp; li < ncen; li += NL_WARPS) {
      const int i = cs + li;
      const double xi = x[i], yi = y[i], zi = z[i];
      const float fxi = (float)(xi - ox), fyi = (float)(yi - oy), fzi = (float)(zi - oz);
      int cnt = s_cnt[li];
      for (int cb = 0; cb < nch; cb += 32) {
        const int ch = cb + lane;
        bool near = false;
        if (ch < nch) {
          const float gx = fmaxf(0.f, fmaxf(bb[0][ch] - fxi, fxi - bb[3][ch]));
          const float gy = fmaxf(0.f, fmaxf(bb[1][ch] - fyi, fyi - bb[4][ch]));
          const float gz = fmaxf(0.f, fmaxf(bb[2][ch] - fzi, fzi - bb[5][ch]));
          near = gx * gx + gy * gy + gz * gz < hi_band;
        }
        unsigned m = __ballot_sync(0xffffffffu, near);
        while (m) {
          const int chunk = cb + __ffs(m) - 1;
          m &= m - 1;
          const int t = chunk * 32 + lane;
          const int j = sj[t];
          bool in = false;
          if (j >= 0 && j != i) {
            const float dxf = sx[t] - fxi, dyf = sy[t] - fyi, dzf = sz[t] - fzi;
            const float d2f = dxf * dxf + dyf * dyf + dzf * dzf;
            if (d2f < lo_band)
              in = true;
            else if (d2f < hi_band)
              in = dist2_list(b, xi, yi, zi, x[j], y[j], z[j]) < cut2;
          }
          const unsigned mm = __ballot_sync(0xffffffffu, in);
          if (in) {
            const int pos = cnt + __popc(mm & lt);
            if (pos < cap) nbrs[(size_t)i * cap + pos] = j;
          }
          cnt += __popc(mm);
        }
      }
      if (lane == 0) s_cnt[li] = cnt;
      __syncwarp();
    }
    __syncthreads();
    s0 = s1;
  }
  for (int t = threadIdx.x; t < ncen; t += NL_BLOCK) {
    const int cnt = s_cnt[t];
    count[cs + t] = cnt;
    if (cnt > cap) atomicOr(overflow, 1);
  }
}

// ---------------------------------------------------------------------------
// Gathers / scatters and integration.
// ---------------------------------------------------------------------------
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

__device__ __forceinline__ unsigned to_fixed(double v, double lo, double scale) {
  return (unsigned)(unsigned long long)__double2ll_rd((v - lo) * scale);
}

__device__ __forceinline__ void warp_max_atomic(double d2, unsigned long long* out) {
  unsigned long long bits = (unsigned long long)__double_as_longlong(d2);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long t = __shfl_xor_sync(0xffffffffu, bits, o);
    bits = t > bits ? t : bits;
  }
  if ((threadIdx.x & 31) == 0) atomicMax(out, bits);
}

// UpdatePositionFlag + ApplyPBC (update_position_op.hip.cu:22-46, box.h:133-169),
// fused with the skin check DisplacementSq (base_neighbor_list_builder.cpp:102-116)
// and, for the mixed form, the fixed-point record {ux, uy, uz, q_f32}.
__global__ void k_drift(DBox b, int n, double dt, double* __restrict__ x, double* __restrict__ y,
                        double* __restrict__ z, const double* __restrict__ vx,
                        const double* __restrict__ vy, const double* __restrict__ vz,
                        const double* __restrict__ x0, const double* __restrict__ y0,
                        const double* __restrict__ z0, unsigned long long* __restrict__ max_d2,
                        uint4* __restrict__ atoms, const double* __restrict__ q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double d2 = 0.0;
  if (i < n) {
    double p[3] = {x[i] + vx[i] * dt, y[i] + vy[i] * dt, z[i] + vz[i] * dt};
    for (int d = 0; d < 3; ++d) {
      if (p[d] >= b.lo[d] + b.len[d]) p[d] -= b.len[d];
      if (p[d] < b.lo[d]) p[d] += b.len[d];
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
  if (max_d2) warp_max_atomic(d2, max_d2);
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
                      void* scratch, int* status, cudaStream_t st) {
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
  if (cudaMemsetAsync(counts, 0, sizeof(int) * (size_t)ncell, st) != cudaSuccess) {
    set_error("cudaMemsetAsync failed in cells_sort");
    return RBX_ERR_CUDA;
  }
  if (n > 0) {
    k_cell_assign<<<(n + 255) / 256, 256, 0, st>>>(b, dims[0], dims[1], dims[2], n, x, y, z, cell,
                                                   sub, counts);
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

int launch_full_list(const DBox& b, const int dims[3], double cutoff, int n, const double* x,
                     const double* y, const double* z, const int* cell_start, int cap,
                     int* count, int* nbrs, int* overflow, cudaStream_t st) {
  const int ncell = dims[0] * dims[1] * dims[2];
  const double cut2 = cutoff * cutoff;
  double emax = 0.0;
  for (int d = 0; d < 3; ++d) emax = fmax(emax, b.len[d] / dims[d]);
  // FP32 screening error is far below 1e-5 of (cutoff^2 + (2 edge)^2); guard band 1e-4 of it.
  const double band = 1e-4 * (cut2 + 4.0 * emax * emax);
  const float lo_band = (float)(cut2 - band), hi_band = (float)(cut2 + band);
  k_full_list<<<ncell, NL_BLOCK, 0, st>>>(b, dims[0], dims[1], dims[2], cut2, lo_band, hi_band, n,
                                          x, y, z, cell_start, cap, count, nbrs, overflow);
  count_launch();
  return check_launch("full_list");
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

int launch_kick(int n, const double* fx, const double* fy, const double* fz, const int* type,
                const double* inv_mass, double half_dt, double* vx, double* vy, double* vz,
                cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_kick<<<(n + 255) / 256, 256, 0, st>>>(n, fx, fy, fz, type, inv_mass, half_dt, vx, vy, vz);
  count_launch();
  return check_launch("kick");
}

int launch_drift(const DBox& b, int n, double dt, double* x, double* y, double* z,
                 const double* vx, const double* vy, const double* vz, const double* x0,
                 const double* y0, const double* z0, unsigned long long* max_d2_bits,
                 uint4* atoms, const double* q, cudaStream_t st) {
  if (n <= 0) return RBX_OK;
  k_drift<<<(n + 255) / 256, 256, 0, st>>>(b, n, dt, x, y, z, vx, vy, vz, x0, y0, z0, max_d2_bits,
                                           atoms, q);
  count_launch();
  return check_launch("drift");
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
