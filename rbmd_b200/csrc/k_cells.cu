// k_cells.cu -- cell-list binning by counting sort (replaces ContPointLocator::Build,
// framework/locator/ContPointLocator.cxx:70-92: BinPointsWorklet + SortByKey + Upper/LowerBounds).
//
// count (atomics) -> exclusive scan (one block per system) -> scatter (atomics) -> per-cell sort
// by atom id (the stable order of the reference's sort of fresh 0..N-1 point ids) fused with the
// gather of cell-ordered positions, charges and metadata that the pair kernel streams.
#include <climits>

#include "kernels.h"

namespace rbmd {

__global__ void k_cells_zero(const SysDev* __restrict__ S, const int2* __restrict__ work) {
  const int2 w = work[blockIdx.x];
  const SysDev& s = S[w.x];
  const int c = w.y + threadIdx.x;
  if (c < s.ncell) s.cell_count[c] = 0;
  if (c == 0) {  // a new cell list: nothing has moved since
    s.st->shake_disp_bits = 0u;
    s.st->out_bits = 0u;
    s.st->mig_n = 0;
  }
}

__global__ void k_cells_count(const SysDev* __restrict__ S, const int2* __restrict__ work) {
  const int2 w = work[blockIdx.x];
  const SysDev& s = S[w.x];
  const int i = w.y + threadIdx.x;
  if (i >= s.n) return;
  const double4 p = s.x[i];
  const double pc[3] = {p.x, p.y, p.z};
  int ijk[3];
  double out = 0.0;  // how far the atom lies outside the cell it is binned into
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    long long c = (long long)((pc[k] - s.lo[k]) / s.d[k]);  // truncation, as vtkm::Id3(Vec3f)
    c = c < 0 ? 0 : c;
    c = c > s.dims[k] - 1 ? s.dims[k] - 1 : c;
    ijk[k] = (int)c;
    out = fmax(out, fmax(s.lo[k] + (double)c * s.d[k] - pc[k], pc[k] - (s.lo[k] + (double)(c + 1) * s.d[k])));
  }
  if (out > 0.0) atomicMax(&s.st->out_bits, __float_as_uint(__double2float_ru(out)));  // non-negative: bits order as values
  // internal numbering is z fastest so that the 2 nc + 1 cells of a traversal row (fixed x and y
  // offsets) are contiguous in cell order; get_cells reports the reference's x-fastest ids
  const int cell = ijk[2] + s.dims[2] * (ijk[1] + s.dims[1] * ijk[0]);
  s.cell_of_atom[i] = cell;
  atomicAdd(&s.cell_count[cell], 1);
}

// One block (1024 threads) per system: exclusive scan of the cell counts.
__global__ void __launch_bounds__(1024) k_cells_scan(const SysDev* __restrict__ S,
                                                     const int* __restrict__ slots) {
  const SysDev& s = S[slots[blockIdx.x]];
  const int nt = blockDim.x, t = threadIdx.x;
  const int chunk = (s.ncell + nt - 1) / nt;
  const int c0 = t * chunk, c1 = min(c0 + chunk, s.ncell);
  int local = 0;
  for (int c = c0; c < c1; ++c) local += s.cell_count[c];
  __shared__ int wsum[32];
  const int lane = t & 31, wid = t >> 5;
  int incl = warp_incl_scan(local, lane);
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int vsum = (lane < (nt >> 5)) ? wsum[lane] : 0;
    int winc = warp_incl_scan(vsum, lane);
    wsum[lane] = winc - vsum;
  }
  __syncthreads();
  int run = wsum[wid] + incl - local;
  for (int c = c0; c < c1; ++c) {
    s.cell_start[c] = run;
    s.cell_fill[c] = run;
    run += s.cell_count[c];
  }
  if (t == nt - 1) s.cell_start[s.ncell] = s.n;
}

__global__ void k_cells_scatter(const SysDev* __restrict__ S, const int2* __restrict__ work) {
  const int2 w = work[blockIdx.x];
  const SysDev& s = S[w.x];
  const int i = w.y + threadIdx.x;
  if (i >= s.n) return;
  const int slot = atomicAdd(&s.cell_fill[s.cell_of_atom[i]], 1);
  s.sorted[slot] = i;
}

// One warp per cell (kSortWarps warps per block, each taking kCellBlock / kSortWarps cells of the
// block's range): the cell's atom ids ranked by value with shuffles (cells of more than 32 atoms,
// rare, are sorted by lane 0), then the cell-ordered copies of positions and metadata written by
// consecutive lanes.  The order is the ids' ascending order, as before.
constexpr int kSortWarps = 32;

__global__ void __launch_bounds__(kSortWarps * 32) k_cells_sort_gather(const SysDev* __restrict__ S,
                                                                     const int2* __restrict__ work) {
  const int2 w = work[blockIdx.x];
  const SysDev& s = S[w.x];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const unsigned FULL = 0xffffffffu;
  int* ids = s.sorted;
  for (int cc = wid; cc < kCellBlock; cc += kSortWarps) {
    const int c = w.y + cc;
    if (c >= s.ncell) break;  // warp-uniform
    const int b = s.cell_start[c], e = s.cell_start[c + 1], cnt = e - b;
    if (cnt <= 32) {
      const int id = lane < cnt ? ids[b + lane] : INT_MAX;
      int rank = 0;
      for (int j = 0; j < cnt; ++j) rank += __shfl_sync(FULL, id, j) < id ? 1 : 0;
      __syncwarp();
      if (lane < cnt) ids[b + rank] = id;
      __syncwarp();
    } else {
      if (lane == 0)
        for (int k = b + 1; k < e; ++k) {
          const int key = ids[k];
          int j = k - 1;
          while (j >= b && ids[j] > key) {
            ids[j + 1] = ids[j];
            --j;
          }
          ids[j + 1] = key;
        }
      __syncwarp();
    }
    for (int k = b + lane; k < e; k += 32) {
      const int i = ids[k];
      s.rank[i] = k;
      const double4 p = s.x[i];
      s.sx[k] = p;
      s.sxf[k] = make_float4((float)p.x, (float)p.y, (float)p.z, (float)p.w);
      const int4 m = s.meta[i];
      s.smeta[k] = make_int4(i, m.x, m.y, m.z);
    }
  }
}

void launch_cells(const Batch& b, cudaStream_t st) {
  k_cells_zero<<<b.cell.n, kCellBlock, 0, st>>>(b.sys, b.cell.d);
  k_cells_count<<<b.atom.n, kAtomBlock, 0, st>>>(b.sys, b.atom.d);
  k_cells_scan<<<b.nsys, 1024, 0, st>>>(b.sys, b.d_slots);
  k_cells_scatter<<<b.atom.n, kAtomBlock, 0, st>>>(b.sys, b.atom.d);
  k_cells_sort_gather<<<b.cell.n, kSortWarps * 32, 0, st>>>(b.sys, b.cell.d);
  note_launch(5);
}

}  // namespace rbmd
