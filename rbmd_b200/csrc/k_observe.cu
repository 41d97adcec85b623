// k_observe.cu -- trajectory observables on the device: mean square displacement and velocity
// autocorrelation against a reference configuration, and radial-distribution pair counts.
//
// None of these kernels is on the step path: they run between steps, on the context stream, when
// an output asks for them (output/MSDOutput.cpp, output/VACFOutput.cpp, output/RDFOutput.cpp).
#include "kernels.h"

namespace rbmd {

// ------------------------------------------------------------------------------------ MSD, VACF
// Reference configuration: positions, velocities and image counters at the start step
// (MSDOutput.cpp:58-66, VACFOutput.cpp:54-57).  The reference zeroes the image counters there
// instead; the counters are kept and their values at the start step subtracted, which gives the
// same unwrapped displacement without changing the state.
// which: bit 0 positions and image counters (MSD), bit 1 velocities (VACF).
__global__ void k_obs_snapshot(const SysDev* __restrict__ sys, int slot, int which, double4* __restrict__ x0,
                               double4* __restrict__ v0, int4* __restrict__ img0) {
  const SysDev& D = sys[slot];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.n; i += gridDim.x * blockDim.x) {
    if (which & 1) {
      x0[i] = D.x[i];
      img0[i] = make_int4(D.image[3 * i], D.image[3 * i + 1], D.image[3 * i + 2], 0);
    }
    if (which & 2) v0[i] = D.v[i];
  }
}

// Per-block sums of (dx^2, dy^2, dz^2, |d|^2) and (v0x vx, v0y vy, v0z vz, v0.v) over the atoms
// of a fixed grid (ComputeMSDWorklet, OutPutWorklet.cpp:326-362: the unwrapped position
// x + (image - image0) L less the start position; ComputeVACFWorklet, OutPutWorklet.cpp:406-428).
__global__ void __launch_bounds__(kObsThreads) k_obs_msd_vacf(const SysDev* __restrict__ sys, int slot,
                                                              const double4* __restrict__ x0,
                                                              const double4* __restrict__ v0,
                                                              const int4* __restrict__ img0,
                                                              double* __restrict__ part) {
  const SysDev& D = sys[slot];
  const double L0 = D.L[0], L1 = D.L[1], L2 = D.L[2];
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < D.n; i += gridDim.x * blockDim.x) {
    const double4 x = D.x[i], a = x0[i], v = D.v[i], w = v0[i];
    const int4 m = img0[i];
    const int* im = D.image + 3 * i;
    const double dx = __dsub_rn(__dadd_rn(x.x, __dmul_rn((double)(im[0] - m.x), L0)), a.x);
    const double dy = __dsub_rn(__dadd_rn(x.y, __dmul_rn((double)(im[1] - m.y), L1)), a.y);
    const double dz = __dsub_rn(__dadd_rn(x.z, __dmul_rn((double)(im[2] - m.z), L2)), a.z);
    const double sx = __dmul_rn(dx, dx), sy = __dmul_rn(dy, dy), sz = __dmul_rn(dz, dz);
    acc[0] += sx;
    acc[1] += sy;
    acc[2] += sz;
    acc[3] += __dadd_rn(__dadd_rn(sx, sy), sz);
    const double cx = __dmul_rn(w.x, v.x), cy = __dmul_rn(w.y, v.y), cz = __dmul_rn(w.z, v.z);
    acc[4] += cx;
    acc[5] += cy;
    acc[6] += cz;
    acc[7] += __dadd_rn(__dadd_rn(cx, cy), cz);
  }
  __shared__ double s[kObsThreads / 32][8];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double t = acc[k];
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) s[warp][k] = t;
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    double t = 0.0;
    for (int w = 0; w < kObsThreads / 32; ++w) t += s[w][threadIdx.x];
    part[blockIdx.x * 8 + threadIdx.x] = t;
  }
}

// Fixed-order sum of the block partials, divided by the atom count (MSDOutput.cpp:130-131,
// VACFOutput.cpp:115-116): out = (msd x, y, z, total, vacf x, y, z, total).
__global__ void k_obs_finish(const SysDev* __restrict__ sys, int slot, const double* __restrict__ part,
                             int nblocks, double* __restrict__ out) {
  const int k = threadIdx.x;
  if (k >= 8) return;
  double t = 0.0;
  for (int b = 0; b < nblocks; ++b) t += part[b * 8 + k];
  out[k] = t / (double)sys[slot].n;
}

void launch_obs_snapshot(const SysDev* sys, int slot, int n, int which, double4* x0, double4* v0, int4* img0,
                         cudaStream_t s) {
  const int blocks = (int)((n + kObsThreads - 1) / kObsThreads);
  k_obs_snapshot<<<blocks > 0 ? blocks : 1, kObsThreads, 0, s>>>(sys, slot, which, x0, v0, img0);
  note_launch();
}

int obs_blocks(int n) {
  const int b = (n + kObsThreads - 1) / kObsThreads;
  return b < 1 ? 1 : (b > kObsMaxBlocks ? kObsMaxBlocks : b);
}

void launch_obs_msd_vacf(const SysDev* sys, int slot, int n, const double4* x0, const double4* v0, const int4* img0,
                         double* part, double* out, cudaStream_t s) {
  const int blocks = obs_blocks(n);
  k_obs_msd_vacf<<<blocks, kObsThreads, 0, s>>>(sys, slot, x0, v0, img0, part);
  k_obs_finish<<<1, 32, 0, s>>>(sys, slot, part, blocks, out);
  note_launch(2);
}

// ------------------------------------------------------------------------------------------ RDF
// Pair counts of the radial distribution function (ComputeRDFWorklet, OutPutWorklet.cpp:230-310
// and its inbuild twin at :578-640): for every bin b and every (center, target) pair, counted
// once per periodic image, whether r_b < |x_t + n L - x_c| < u_b with u_b = r_b + 0.01 r_b, the
// pair skipped when both atoms share a molecule (exclude_mol).  The reference enumerates the
// images a cell stencil of +-(r / cell + 1) cells reaches; here every image inside u_max counts.
//
// One thread per center atom, the block's slice of targets staged through shared memory 256 at a
// time.  The displacement of an image is (x_t - x_c) + n L, each component rounded once; its
// length is the correctly rounded square root of dx^2 + dy^2 + dz^2 summed left to right, so the
// counts are reproducible bit for bit on any IEEE-754 FP64 host.  Bins are found from the
// distance and tested against the tables exactly; the bin counters live in shared memory when
// they fit.
__global__ void __launch_bounds__(kObsThreads) k_rdf_count(const SysDev* __restrict__ sys, int slot,
                                                           const int* __restrict__ centers, int nc,
                                                           const int* __restrict__ targets, int nt,
                                                           const double* __restrict__ radii,
                                                           const double* __restrict__ upper, int nb,
                                                           double inv_dr, int exclude_mol, int hist_shared,
                                                           unsigned long long* __restrict__ counts) {
  extern __shared__ unsigned int s_hist[];
  __shared__ double s_x[kObsThreads], s_y[kObsThreads], s_z[kObsThreads];
  __shared__ int s_m[kObsThreads];
  const SysDev& D = sys[slot];
  const double Lx = D.L[0], Ly = D.L[1], Lz = D.L[2];
  const double ix = __drcp_rn(Lx), iy = __drcp_rn(Ly), iz = __drcp_rn(Lz);
  const double R = upper[nb - 1];
  const double R2 = R * R * (1.0 + 1e-9);  // a filter only: never rejects a pair below R
  if (hist_shared)
    for (int k = threadIdx.x; k < nb; k += blockDim.x) s_hist[k] = 0u;

  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  double xc = 0, yc = 0, zc = 0;
  int mc = -1;
  if (c < nc) {
    const int a = centers[c];
    const double4 p = D.x[a];
    xc = p.x;
    yc = p.y;
    zc = p.z;
    mc = D.meta[a].y;
  }
  const int t_begin = blockIdx.y * kRdfTargetsPerBlock;
  const int t_end = min(nt, t_begin + kRdfTargetsPerBlock);
  for (int t0 = t_begin; t0 < t_end; t0 += kObsThreads) {
    __syncthreads();
    const int t = t0 + threadIdx.x;
    if (t < t_end) {
      const int a = targets[t];
      const double4 p = D.x[a];
      s_x[threadIdx.x] = p.x;
      s_y[threadIdx.x] = p.y;
      s_z[threadIdx.x] = p.z;
      s_m[threadIdx.x] = D.meta[a].y;
    }
    __syncthreads();
    if (c >= nc) continue;
    const int cnt = min(kObsThreads, t_end - t0);
    for (int j = 0; j < cnt; ++j) {
      if (exclude_mol && s_m[j] == mc) continue;
      const double bx = __dsub_rn(s_x[j], xc), by = __dsub_rn(s_y[j], yc), bz = __dsub_rn(s_z[j], zc);
      // images whose component can lie inside R, one more on each side against rounding
      const int x0 = (int)ceil((-R - bx) * ix) - 1, x1 = (int)floor((R - bx) * ix) + 1;
      const int y0 = (int)ceil((-R - by) * iy) - 1, y1 = (int)floor((R - by) * iy) + 1;
      const int z0 = (int)ceil((-R - bz) * iz) - 1, z1 = (int)floor((R - bz) * iz) + 1;
      for (int nx = x0; nx <= x1; ++nx) {
        const double dx = __dadd_rn(bx, __dmul_rn((double)nx, Lx));
        if (fabs(dx) >= R) continue;
        const double sx = __dmul_rn(dx, dx);
        for (int ny = y0; ny <= y1; ++ny) {
          const double dy = __dadd_rn(by, __dmul_rn((double)ny, Ly));
          if (fabs(dy) >= R) continue;
          const double sxy = __dadd_rn(sx, __dmul_rn(dy, dy));
          for (int nz = z0; nz <= z1; ++nz) {
            const double dz = __dadd_rn(bz, __dmul_rn((double)nz, Lz));
            if (fabs(dz) >= R) continue;
            const double d2 = __dadd_rn(sxy, __dmul_rn(dz, dz));
            if (d2 > R2) continue;
            const double dis = __dsqrt_rn(d2);
            const double q = dis * inv_dr;
            const int b0 = max(0, (int)(q * (1.0 / 1.01)) - 3);
            const int b1 = min(nb - 1, (int)q + 1);
            for (int bin = b0; bin <= b1; ++bin) {
              if (radii[bin] < dis && dis < upper[bin]) {
                if (hist_shared) atomicAdd(&s_hist[bin], 1u);
                else atomicAdd(&counts[bin], 1ull);
              }
            }
          }
        }
      }
    }
  }
  if (hist_shared) {
    __syncthreads();
    for (int k = threadIdx.x; k < nb; k += blockDim.x)
      if (s_hist[k]) atomicAdd(&counts[k], (unsigned long long)s_hist[k]);
  }
}

void launch_rdf_count(const SysDev* sys, int slot, const int* centers, int nc, const int* targets, int nt,
                      const double* radii, const double* upper, int nb, double dr, int exclude_mol,
                      unsigned long long* counts, cudaStream_t s) {
  if (nc <= 0 || nt <= 0 || nb <= 0) return;
  const int hist_shared = nb <= kRdfSharedBins ? 1 : 0;
  const dim3 grid((unsigned)((nc + kObsThreads - 1) / kObsThreads),
                  (unsigned)((nt + kRdfTargetsPerBlock - 1) / kRdfTargetsPerBlock));
  const size_t smem = hist_shared ? sizeof(unsigned int) * (size_t)nb : 0;
  k_rdf_count<<<grid, kObsThreads, smem, s>>>(sys, slot, centers, nc, targets, nt, radii, upper, nb, 1.0 / dr,
                                              exclude_mol, hist_shared, counts);
  note_launch();
}

}  // namespace rbmd

namespace rbmd {

// ------------------------------------------------------------------------- asynchronous snapshot
// Packs one system's state for a snapshot copied to the host while later steps run: step, box
// (lo xyz, hi xyz), positions and velocities [3n] and image counters [3n], in that order.
__global__ void k_snapshot_pack(const SysDev* __restrict__ sys, int slot, char* __restrict__ out) {
  const SysDev& D = sys[slot];
  const int n = D.n;
  auto* step = (long long*)out;
  auto* box = (double*)(out + 8);
  auto* x = box + 6;
  auto* v = x + 3 * (size_t)n;
  auto* image = (int*)(v + 3 * (size_t)n);
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  if (tid == 0) {
    *step = (long long)D.st->step;
    for (int k = 0; k < 3; ++k) {
      box[k] = D.lo[k];
      box[3 + k] = D.hi[k];
    }
  }
  for (int i = tid; i < n; i += gridDim.x * blockDim.x) {
    const double4 p = D.x[i], u = D.v[i];
    x[3 * i] = p.x;
    x[3 * i + 1] = p.y;
    x[3 * i + 2] = p.z;
    v[3 * i] = u.x;
    v[3 * i + 1] = u.y;
    v[3 * i + 2] = u.z;
    image[3 * i] = D.image[3 * i];
    image[3 * i + 1] = D.image[3 * i + 1];
    image[3 * i + 2] = D.image[3 * i + 2];
  }
}

size_t snapshot_bytes(int n) { return 56 + 60 * (size_t)n; }

void launch_snapshot_pack(const SysDev* sys, int slot, int n, void* out, cudaStream_t s) {
  const int blocks = obs_blocks(n);
  k_snapshot_pack<<<blocks, kObsThreads, 0, s>>>(sys, slot, (char*)out);
  note_launch();
}

}  // namespace rbmd
