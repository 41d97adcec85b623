// observe.cpp -- trajectory observables behind the C ABI: the MSD / VACF reference configuration
// and its averages (output/MSDOutput.cpp, output/VACFOutput.cpp), and RDF pair counts of one
// snapshot (output/RDFOutput.cpp).  The kernels are in k_observe.cu; this file validates, stages
// the index lists and reads the results back.  Everything runs on the context stream, after the
// steps already queued.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "engine.h"

namespace rbmd {

int rdf_bins(double radius, double dr, std::vector<double>* radii) {
  if (!(radius > 0.0) || !(dr > 0.0) || !std::isfinite(radius) || !std::isfinite(dr)) return -1;
  const double nq = radius / dr;
  if (!(nq >= 1.0) || nq > (double)(1 << 22)) return -1;
  const int nb = (int)nq;  // the reference sizes its table with the truncated quotient
  if (radii) {
    radii->resize(nb);
    double r = 0.0;
    for (int b = 0; b < nb; ++b) {
      r += dr;
      (*radii)[b] = r;
    }
  }
  return nb;
}

int Context::observe_reset(int id, int which) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  if (which & ~(RBMD_OBS_MSD | RBMD_OBS_VACF) || !which) return fail(RBMD_ERR_ARG, "observe_reset: bad reference mask");
  const int n = s->dev.n;
  if (!s->obs_x0) {
    s->obs_x0 = (double4*)dmalloc(sizeof(double4) * n);
    s->obs_v0 = (double4*)dmalloc(sizeof(double4) * n);
    s->obs_img0 = (int4*)dmalloc(sizeof(int4) * n);
    for (void* p : {(void*)s->obs_x0, (void*)s->obs_v0, (void*)s->obs_img0})
      if (p) s->allocs.push_back(p);
    if (!s->obs_x0 || !s->obs_v0 || !s->obs_img0) {
      s->obs_x0 = nullptr;
      s->obs_v0 = nullptr;
      s->obs_img0 = nullptr;
      return fail(RBMD_ERR_OOM, "observable reference configuration");
    }
  }
  launch_obs_snapshot(d_sys_, s->slot, n, which, s->obs_x0, s->obs_v0, s->obs_img0, stream);
  s->obs_have |= which;
  return check_cuda("observe_reset");
}

int Context::observe(int id, double* msd, double* vacf) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  if ((msd && !(s->obs_have & RBMD_OBS_MSD)) || (vacf && !(s->obs_have & RBMD_OBS_VACF)))
    return fail(RBMD_ERR_STATE, "no reference configuration (rbmd_observe_reset first)");
  const int n = s->dev.n;
  const int nb = obs_blocks(n);
  double* part = (double*)dmalloc(sizeof(double) * (8 * (size_t)nb + 8));
  if (!part) return fail(RBMD_ERR_OOM, "observable scratch");
  launch_obs_msd_vacf(d_sys_, s->slot, n, s->obs_x0, s->obs_v0, s->obs_img0, part, part + 8 * (size_t)nb, stream);
  double h[8];
  cudaMemcpyAsync(h, part + 8 * (size_t)nb, sizeof(h), cudaMemcpyDeviceToHost, stream);
  dfree(part);
  int rc = check_cuda("observe");
  if (rc) return rc;
  rc = sync();
  if (rc) return rc;
  if (msd) std::memcpy(msd, h, 4 * sizeof(double));
  if (vacf) std::memcpy(vacf, h + 4, 4 * sizeof(double));
  return RBMD_OK;
}

int Context::rdf_counts(int id, const int32_t* centers, int nc, const int32_t* targets, int nt, double radius,
                        double dr, int exclude_same_molecule, int64_t* counts, double* volume) {
  std::lock_guard<std::recursive_mutex> lk(mu);
  System* s = find(id);
  if (!s) return fail(RBMD_ERR_STATE, "unknown system id");
  std::vector<double> radii;
  const int nb = rdf_bins(radius, dr, &radii);
  if (nb < 0) return fail(RBMD_ERR_ARG, "rdf: radius and dr must be positive with radius / dr >= 1");
  if (!counts) return fail(RBMD_ERR_ARG, "rdf: null counts");
  if (nc < 0 || nt < 0 || (nc && !centers) || (nt && !targets)) return fail(RBMD_ERR_ARG, "rdf: bad atom lists");
  const int n = s->dev.n;
  for (int k = 0; k < nc; ++k)
    if (centers[k] < 0 || centers[k] >= n) return fail(RBMD_ERR_ARG, "rdf: center atom id out of range");
  for (int k = 0; k < nt; ++k)
    if (targets[k] < 0 || targets[k] >= n) return fail(RBMD_ERR_ARG, "rdf: target atom id out of range");
  int rc = refresh(s);  // the box of an NPT system lives on the device
  if (rc) return rc;
  // one thread walks every target of its center over the images inside the last bin edge: bound
  // the images per pair and the pairs per call so that one launch stays within seconds
  const double lmin = std::min(s->dev.L[0], std::min(s->dev.L[1], s->dev.L[2]));
  if (radius * 1.01 > 8.0 * lmin) return fail(RBMD_ERR_ARG, "rdf: radius beyond 8 box lengths");
  if ((double)nc * (double)nt > 1e12) return fail(RBMD_ERR_UNSUPPORTED, "rdf: more than 1e12 center-target pairs");
  std::vector<double> upper(nb);
  for (int b = 0; b < nb; ++b) {
    const double grow = radii[b] * 0.01;
    upper[b] = radii[b] + grow;  // current_radius + current_radius * 0.01 (OutPutWorklet.cpp:283-284)
  }
  const size_t bytes = sizeof(unsigned long long) * nb + sizeof(double) * 2 * nb + sizeof(int) * ((size_t)nc + nt);
  char* buf = (char*)dmalloc(bytes);
  if (!buf) return fail(RBMD_ERR_OOM, "rdf scratch");
  auto* d_counts = (unsigned long long*)buf;
  auto* d_radii = (double*)(d_counts + nb);
  auto* d_upper = d_radii + nb;
  auto* d_centers = (int*)(d_upper + nb);
  auto* d_targets = d_centers + nc;
  cudaMemsetAsync(d_counts, 0, sizeof(unsigned long long) * nb, stream);
  cudaMemcpyAsync(d_radii, radii.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, stream);
  cudaMemcpyAsync(d_upper, upper.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, stream);
  if (nc) cudaMemcpyAsync(d_centers, centers, sizeof(int) * nc, cudaMemcpyHostToDevice, stream);
  if (nt) cudaMemcpyAsync(d_targets, targets, sizeof(int) * nt, cudaMemcpyHostToDevice, stream);
  launch_rdf_count(d_sys_, s->slot, d_centers, nc, d_targets, nt, d_radii, d_upper, nb, dr, exclude_same_molecule ? 1 : 0,
                   d_counts, stream);
  std::vector<unsigned long long> h(nb);
  cudaMemcpyAsync(h.data(), d_counts, sizeof(unsigned long long) * nb, cudaMemcpyDeviceToHost, stream);
  dfree(buf);
  rc = check_cuda("rdf");
  if (rc) return rc;
  rc = sync();
  if (rc) return rc;
  for (int b = 0; b < nb; ++b) counts[b] = (int64_t)h[b];
  if (volume) *volume = s->dev.volume;
  return RBMD_OK;
}

}  // namespace rbmd
