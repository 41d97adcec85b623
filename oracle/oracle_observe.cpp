// oracle_observe.cpp -- CPU restatement of the trajectory observables: MSD, VACF and RDF pair
// counts.  TEST INFRASTRUCTURE ONLY (see oracle.hpp): the checker of rbmd_observe and
// rbmd_rdf_counts.
//
// MSD: ComputeMSDWorklet (framework/output/worklet/OutPutWorklet.cpp:326-362), averaged over the
//   atoms as MSDOutput::ExecuteMSD does (framework/output/MSDOutput.cpp:116-134).  The reference
//   zeroes the image counters at the start step; here their start values are subtracted.
// VACF: ComputeVACFWorklet (OutPutWorklet.cpp:406-428), VACFOutput::ExecuteMSD
//   (framework/output/VACFOutput.cpp:108-118).
// RDF: ComputeRDFWorklet (OutPutWorklet.cpp:230-310; the inbuild twin at :578-640) with the radii
//   of RDFOutput::RDFOutput (framework/output/RDFOutput.cpp:42-53).  Every periodic image closer
//   than the last bin's upper edge is enumerated (the reference's cell stencil reaches the same
//   images whenever it spans them).
#include <cmath>
#include <cstdint>
#include <vector>

extern "C" {

int oracle_rdf_bins(double radius, double dr, double* radii, int cap) {
  if (!(radius > 0.0) || !(dr > 0.0)) return -1;
  const double nq = radius / dr;
  if (!(nq >= 1.0) || nq > (double)(1 << 22)) return -1;
  const int nb = (int)nq;
  double r = 0.0;
  for (int b = 0; b < nb; ++b) {
    r += dr;
    if (radii && b < cap) radii[b] = r;
  }
  return nb;
}

// x0, x, v0, v: [3n]; img0, img: [3n]; L: [3]; msd, vacf: [4]
int oracle_msd_vacf(int n, const double* x0, const int32_t* img0, const double* v0, const double* x,
                    const int32_t* img, const double* v, const double* L, double* msd, double* vacf) {
  double m[4] = {0, 0, 0, 0}, c[4] = {0, 0, 0, 0};
  for (int i = 0; i < n; ++i) {
    double d[3], w[3];
    for (int k = 0; k < 3; ++k) {
      const double flag = (double)(img[3 * i + k] - img0[3 * i + k]);
      const double unwrapped = x[3 * i + k] + flag * L[k];
      d[k] = unwrapped - x0[3 * i + k];
      w[k] = v0[3 * i + k] * v[3 * i + k];
    }
    const double sx = d[0] * d[0], sy = d[1] * d[1], sz = d[2] * d[2];
    m[0] += sx;
    m[1] += sy;
    m[2] += sz;
    m[3] += sx + sy + sz;
    c[0] += w[0];
    c[1] += w[1];
    c[2] += w[2];
    c[3] += w[0] + w[1] + w[2];
  }
  for (int k = 0; k < 4; ++k) {
    msd[k] = m[k] / n;
    vacf[k] = c[k] / n;
  }
  return 0;
}

// x: [3n] positions; mol: [n] molecule ids; L: [3]; counts: [nb] (overwritten)
int oracle_rdf_counts(const double* x, const int32_t* mol, const double* L, const int32_t* centers, int nc,
                      const int32_t* targets, int nt, double radius, double dr, int exclude_same_molecule,
                      int64_t* counts) {
  std::vector<double> r;
  const int nb = oracle_rdf_bins(radius, dr, nullptr, 0);
  if (nb < 0) return -1;
  r.resize(nb);
  oracle_rdf_bins(radius, dr, r.data(), nb);
  std::vector<double> u(nb);
  for (int b = 0; b < nb; ++b) u[b] = r[b] + r[b] * 0.01;
  for (int b = 0; b < nb; ++b) counts[b] = 0;
  const double R = u[nb - 1];
  for (int a = 0; a < nc; ++a) {
    const int i = centers[a];
    for (int t = 0; t < nt; ++t) {
      const int j = targets[t];
      if (exclude_same_molecule && mol[i] == mol[j]) continue;
      double base[3];
      int lo[3], hi[3];
      for (int k = 0; k < 3; ++k) {
        base[k] = x[3 * j + k] - x[3 * i + k];
        lo[k] = (int)std::ceil((-R - base[k]) / L[k]) - 1;
        hi[k] = (int)std::floor((R - base[k]) / L[k]) + 1;
      }
      for (int nx = lo[0]; nx <= hi[0]; ++nx)
        for (int ny = lo[1]; ny <= hi[1]; ++ny)
          for (int nz = lo[2]; nz <= hi[2]; ++nz) {
            const double dx = base[0] + nx * L[0];
            const double dy = base[1] + ny * L[1];
            const double dz = base[2] + nz * L[2];
            if (std::fabs(dx) >= R || std::fabs(dy) >= R || std::fabs(dz) >= R) continue;
            const double dis = std::sqrt(dx * dx + dy * dy + dz * dz);
            for (int b = 0; b < nb; ++b)
              if (dis > r[b] && dis < u[b]) ++counts[b];
          }
    }
  }
  return nb;
}

}  // extern "C"
