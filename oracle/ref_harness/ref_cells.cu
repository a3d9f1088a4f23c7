/* Reference-kernel harness, linked cells and the full candidate list: RBMD's
 * own op functors from src/neighbor_list/src/op/rocm/linked_cell_op.hip.cu
 * (InitializeCell, AssignAtomsToCell, ComputeCellRangesIndices) and
 * full_neighbor_list_op.hip.cu (EstimateFullNeighborListNoWarp,
 * GenerateFullNeighborListNoWarp), compiled in place.  The host steps around
 * them follow LinkedCell::Build / SortAtomsByCellKey / ComputeCellRangesIndices
 * (linked_cell.cpp:251-411, 443-455, 485-663) for one process without MPI
 * (no halo cells).  Test infrastructure only. */
#include <thrust/device_vector.h>
#include <thrust/fill.h>
#include <thrust/scan.h>
#include <thrust/sequence.h>
#include <thrust/sort.h>

#include <cmath>
#include <vector>

#include "neighbor_list/src/op/rocm/linked_cell_op.hip.cu"
#include "neighbor_list/src/op/rocm/full_neighbor_list_op.hip.cu"
#include "ref_common.h"

/* full_neighbor_list_op.hip.cu also defines ComputeFullNeighborsOp, whose host
 * side reaches the LinkedCell singleton.  The harness never calls it; these
 * definitions only give the linker the symbols it names. */
LinkedCellLocator& LinkedCellLocator::GetInstance() {
  static LinkedCellLocator instance;
  return instance;
}
std::shared_ptr<LinkedCell> LinkedCellLocator::GetLinkedCell() { return _linked_cell; }
LinkedCellDeviceDataPtr* LinkedCell::GetDataPtr() { return nullptr; }

namespace {
struct Grid {
  int dims[3];
  rbmd::Real length[3], recip[3];
};

/* LinkedCell::Build without MPI: cells of edge neighbor_cutoff / c per axis,
 * floor(extent / that) of them, the edge then stretched to fill the box. */
Grid ref_grid(const double* lo, const double* hi, double neighbor_cutoff, int c) {
  Grid g{};
  const rbmd::Real per_cell = (rbmd::Real)neighbor_cutoff / static_cast<rbmd::Real>(c);
  for (int d = 0; d < 3; ++d) {
    const rbmd::Real diff = (rbmd::Real)hi[d] - (rbmd::Real)lo[d];
    g.dims[d] = (int)std::floor(static_cast<double>(diff) / static_cast<double>(per_cell));
    g.length[d] = diff / g.dims[d];
    g.recip[d] = 1.0 / g.length[d];
  }
  return g;
}
}  // namespace

extern "C" {

int ref_cell_dims(const double* lo, const double* hi, double neighbor_cutoff, int c, int* dims) {
  const Grid g = ref_grid(lo, hi, neighbor_cutoff, c);
  for (int d = 0; d < 3; ++d) dims[d] = g.dims[d];
  return 0;
}

/* Cells and the full list of every atom within sqrt(cutoff2) (positions in
 * host order, device pointers).  Outputs, host arrays: per-atom cell id
 * [n]; cell start / end [total cells] over the stably sorted atoms; per-atom
 * neighbour count [n] and the neighbours of atom 0, 1, ... concatenated into
 * nbr_out (capacity nbr_cap).  Returns 0, a CUDA error code, or -(entries
 * needed) when nbr_cap is too small.  *realloc_out is the kernel's overflow
 * flag. */
int ref_cells_full_list(const double* lo, const double* hi, double neighbor_cutoff, int c,
                        double cutoff2, int n, const rbmd::Real* x, const rbmd::Real* y,
                        const rbmd::Real* z, int* cell_out, int* start_out, int* end_out,
                        int* count_out, int* nbr_out, long long nbr_cap, int* realloc_out) {
  const Grid g = ref_grid(lo, hi, neighbor_cutoff, c);
  const int total = g.dims[0] * g.dims[1] * g.dims[2];
  Box box = ref_make_box(lo, hi);
  for (int d = 0; d < 3; ++d) {
    box._halo_coord_min[d] = box._coord_min[d];
    box._halo_coord_max[d] = box._coord_max[d];
    box._box_width_as_cell_units[d] = g.dims[d];
    box._halo_width_as_cell_units[d] = 0;
  }
  LinkedCellDeviceDataPtr lc{};
  lc._d_total_cells = total;
  lc._d_cutoff = (rbmd::Real)neighbor_cutoff;
  for (int d = 0; d < 3; ++d) {
    lc._d_per_dimension_cells[d] = g.dims[d];
    lc._d_cell_length[d] = g.length[d];
    lc._d_cell_length_reciprocal[d] = g.recip[d];
    lc._d_nativate_cells_dims[d] = g.dims[d];
    lc._d_nativate_cells_start[d] = 0;
    lc._d_covers_whole_domain[d] = true;
  }
  Box* d_box = nullptr;
  LinkedCellDeviceDataPtr* d_lc = nullptr;
  if (cudaMalloc(&d_box, sizeof(Box)) != cudaSuccess ||
      cudaMalloc(&d_lc, sizeof(LinkedCellDeviceDataPtr)) != cudaSuccess)
    return (int)cudaGetLastError();
  cudaMemcpy(d_box, &box, sizeof(Box), cudaMemcpyHostToDevice);
  cudaMemcpy(d_lc, &lc, sizeof(LinkedCellDeviceDataPtr), cudaMemcpyHostToDevice);
  int rc = 0;
  {
    thrust::device_vector<Cell> cells(total);
    thrust::device_vector<rbmd::Id> cell_id(n > 0 ? n : 1), sorted_id(n > 0 ? n : 1),
        sorted_idx(n > 0 ? n : 1), start(total), end(total), num(n > 0 ? n : 1),
        maxnum(n > 0 ? n : 1), nstart(n > 0 ? n : 1), nend(n > 0 ? n : 1), realloc_flag(1, 0);
    op::InitializeCellOp<device::DEVICE_GPU>()(d_lc, d_box, thrust::raw_pointer_cast(cells.data()),
                                              total);
    op::AssignAtomsToCellOp<device::DEVICE_GPU>()(
        const_cast<rbmd::Real*>(x), const_cast<rbmd::Real*>(y), const_cast<rbmd::Real*>(z),
        d_box, d_lc, thrust::raw_pointer_cast(cells.data()),
        thrust::raw_pointer_cast(cell_id.data()), n);
    thrust::copy(cell_id.begin(), cell_id.begin() + n, sorted_id.begin());
    thrust::sequence(sorted_idx.begin(), sorted_idx.begin() + n, 0);
    thrust::stable_sort_by_key(sorted_id.begin(), sorted_id.begin() + n, sorted_idx.begin());
    thrust::fill(start.begin(), start.end(), rbmd::Id(0));
    thrust::fill(end.begin(), end.end(), rbmd::Id(0));
    op::ComputeCellRangesIndicesOp<device::DEVICE_GPU>()(
        thrust::raw_pointer_cast(sorted_id.data()), thrust::raw_pointer_cast(start.data()),
        thrust::raw_pointer_cast(end.data()), n);
    const int stencil = (2 * c + 1) * (2 * c + 1) * (2 * c + 1);
    op::EstimateFullNeighborListOp<device::DEVICE_GPU>()(
        thrust::raw_pointer_cast(cell_id.data()), thrust::raw_pointer_cast(start.data()),
        thrust::raw_pointer_cast(end.data()), (rbmd::Real)cutoff2, n,
        const_cast<rbmd::Real*>(x), const_cast<rbmd::Real*>(y), const_cast<rbmd::Real*>(z),
        thrust::raw_pointer_cast(sorted_idx.data()), thrust::raw_pointer_cast(num.data()),
        thrust::raw_pointer_cast(maxnum.data()), box, d_lc, stencil, c);
    thrust::exclusive_scan(maxnum.begin(), maxnum.begin() + n, nstart.begin());
    const long long room =
        n > 0 ? (long long)nstart[n - 1] + (long long)maxnum[n - 1] : 0;
    thrust::device_vector<rbmd::Id> nbrs(room > 0 ? room : 1);
    op::GenerateFullNeighborListOp<device::DEVICE_GPU>()(
        thrust::raw_pointer_cast(cell_id.data()), thrust::raw_pointer_cast(start.data()),
        thrust::raw_pointer_cast(end.data()), (rbmd::Real)cutoff2, n,
        const_cast<rbmd::Real*>(x), const_cast<rbmd::Real*>(y), const_cast<rbmd::Real*>(z),
        thrust::raw_pointer_cast(sorted_idx.data()), thrust::raw_pointer_cast(maxnum.data()),
        thrust::raw_pointer_cast(nstart.data()), thrust::raw_pointer_cast(nend.data()),
        thrust::raw_pointer_cast(nbrs.data()), box, thrust::raw_pointer_cast(realloc_flag.data()),
        d_lc, stencil, c);
    rc = ref_sync();
    if (rc == 0) {
      std::vector<rbmd::Id> h_cell(n), h_s(n), h_e(n), h_nb(room > 0 ? room : 0);
      thrust::copy(cell_id.begin(), cell_id.begin() + n, h_cell.begin());
      thrust::copy(nstart.begin(), nstart.begin() + n, h_s.begin());
      thrust::copy(nend.begin(), nend.begin() + n, h_e.begin());
      if (room > 0) thrust::copy(nbrs.begin(), nbrs.begin() + room, h_nb.begin());
      thrust::copy(start.begin(), start.end(), start_out);
      thrust::copy(end.begin(), end.end(), end_out);
      *realloc_out = realloc_flag[0];
      long long used = 0;
      for (int i = 0; i < n; ++i) {
        cell_out[i] = h_cell[i];
        count_out[i] = h_e[i] - h_s[i];
        used += count_out[i];
      }
      if (used > nbr_cap) {
        rc = (int)-used;
      } else {
        long long o = 0;
        for (int i = 0; i < n; ++i)
          for (int k = h_s[i]; k < h_e[i]; ++k) nbr_out[o++] = h_nb[k];
      }
    }
  }
  cudaFree(d_box);
  cudaFree(d_lc);
  return rc;
}

}  // extern "C"
