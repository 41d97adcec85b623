// oracle_capi.cpp -- extern "C" entry points of the FP64 oracle for the Python tests (ctypes) and
// the CPU baseline timing.  TEST INFRASTRUCTURE ONLY (see oracle.hpp).
#include <cstring>
#include <exception>
#include <memory>

#include "oracle.hpp"

using oracle::System;

extern "C" {

void* oracle_create(const rbmd_system_desc* desc, const rbmd_params* params) {
  try {
    return new System(*desc, *params);
  } catch (const std::exception&) {
    return nullptr;
  }
}

void oracle_destroy(void* h) { delete static_cast<System*>(h); }

int oracle_init(void* h) {
  static_cast<System*>(h)->init();
  return 0;
}

int oracle_step(void* h, int nsteps) {
  System* s = static_cast<System*>(h);
  for (int k = 0; k < nsteps; ++k) s->step_once();
  return s->status;
}

// Forces at the current positions with the current step's random draws (cells rebuilt first).
int oracle_compute_forces(void* h) {
  System* s = static_cast<System*>(h);
  s->build_cells();
  if (s->p.coulomb == RBMD_COUL_RBE) s->sample_k();
  s->compute_force();
  return 0;
}

int oracle_set_step(void* h, int64_t step) {
  static_cast<System*>(h)->step = step;
  return 0;
}

int oracle_get_forces(void* h, double* f) {
  System* s = static_cast<System*>(h);
  std::memcpy(f, s->f.data(), sizeof(double) * 3 * s->N);
  return 0;
}

// parts: 0 near, 1 far (qqr2e applied), 2 bonded
int oracle_get_force_part(void* h, int part, double* f) {
  System* s = static_cast<System*>(h);
  const std::vector<double>& src = part == 0 ? s->f_near : part == 1 ? s->f_far : s->f_bonded;
  std::memcpy(f, src.data(), sizeof(double) * 3 * s->N);
  return 0;
}

int oracle_get_state(void* h, double* x, double* v, int32_t* image) {
  System* s = static_cast<System*>(h);
  if (x) std::memcpy(x, s->x.data(), sizeof(double) * 3 * s->N);
  if (v) std::memcpy(v, s->v.data(), sizeof(double) * 3 * s->N);
  if (image)
    for (int i = 0; i < 3 * s->N; ++i) image[i] = s->image[i];
  return 0;
}

int oracle_set_state(void* h, const double* x, const double* v, const int32_t* image) {
  System* s = static_cast<System*>(h);
  if (x) s->x.assign(x, x + 3 * s->N);
  if (v) s->v.assign(v, v + 3 * s->N);
  if (image) s->image.assign(image, image + 3 * s->N);
  return 0;
}

int oracle_get_thermo(void* h, rbmd_thermo* out) {
  static_cast<System*>(h)->thermo(out);
  return 0;
}

int oracle_get_cells(void* h, int32_t* dims, int32_t* cell_of_atom, int32_t* sorted, int32_t* lower,
                     int32_t* upper) {
  System* s = static_cast<System*>(h);
  s->build_cells();
  const oracle::Cells& c = s->cells;
  if (dims)
    for (int k = 0; k < 3; ++k) dims[k] = c.dims[k];
  int nc = c.dims[0] * c.dims[1] * c.dims[2];
  if (cell_of_atom) std::memcpy(cell_of_atom, c.cell_of_atom.data(), sizeof(int) * s->N);
  if (sorted) std::memcpy(sorted, c.sorted.data(), sizeof(int) * s->N);
  if (lower) std::memcpy(lower, c.lower.data(), sizeof(int) * nc);
  if (upper) std::memcpy(upper, c.upper.data(), sizeof(int) * nc);
  return 0;
}

int oracle_get_rbl_lists(void* h, int32_t cap, int32_t* ncore, int32_t* nshell, int32_t* ids) {
  System* s = static_cast<System*>(h);
  s->build_cells();
  std::vector<int> nc, ns;
  std::vector<std::vector<int>> lists;
  s->rbl_lists(nc, ns, lists, nullptr);
  int rc = 0;
  for (int i = 0; i < s->N; ++i) {
    ncore[i] = nc[i];
    nshell[i] = ns[i];
    int n = (int)lists[i].size();
    if (n > cap) {
      rc = 1;
      n = cap;
    }
    for (int k = 0; k < n; ++k) ids[(size_t)i * cap + k] = lists[i][k];
  }
  return rc;
}

int oracle_get_verlet_lists(void* h, int32_t cap, int32_t* n, int32_t* ids) {
  System* s = static_cast<System*>(h);
  s->build_cells();
  std::vector<std::vector<int>> lists;
  std::vector<std::vector<std::array<double, 3>>> offs;
  s->verlet_lists(lists, offs);
  int rc = 0;
  for (int i = 0; i < s->N; ++i) {
    int c = (int)lists[i].size();
    n[i] = c;
    if (c > cap) {
      rc = 1;
      c = cap;
    }
    for (int k = 0; k < c; ++k) ids[(size_t)i * cap + k] = lists[i][k];
  }
  return rc;
}

int oracle_sample_k(void* h, int32_t* m) {
  System* s = static_cast<System*>(h);
  s->sample_k();
  std::memcpy(m, s->kspace_m.data(), sizeof(int) * s->kspace_m.size());
  return 0;
}

int oracle_get_kspace(void* h, int32_t* m, double* rhok) {
  System* s = static_cast<System*>(h);
  if (m) std::memcpy(m, s->kspace_m.data(), sizeof(int) * s->kspace_m.size());
  if (rhok) std::memcpy(rhok, s->rhok.data(), sizeof(double) * s->rhok.size());
  return 0;
}

// Full Ewald k-space force (x qqr2e) at the current positions; the FP64 yardstick for RBE's own error.
int oracle_ewald_kspace_force(void* h, double* f) {
  System* s = static_cast<System*>(h);
  std::vector<double> F;
  double vir[6];
  s->ewald_force(F, vir);
  for (int i = 0; i < 3 * s->N; ++i) f[i] = F[i] * s->u.qqr2e;
  return 0;
}

int oracle_get_derived(void* h, rbmd_derived* out) {
  System* s = static_cast<System*>(h);
  std::memset(out, 0, sizeof(*out));
  out->rs_num = s->dv.rs_num;
  out->rc_num = s->dv.rc_num;
  out->pice_num = s->dv.pice_num;
  out->num_cycles = s->dv.num_cycles;
  for (int k = 0; k < 3; ++k) {
    out->dims[k] = s->dv.dims[k];
    out->cell_width[k] = s->dv.d[k];
  }
  out->n_cells = s->dv.ncell;
  out->rho_system = s->dv.rho;
  out->S_rbe = s->dv.S;
  out->volume = s->dv.volume;
  return 0;
}

int oracle_status(void* h) { return static_cast<System*>(h)->status; }

int oracle_near_key(float r) { return oracle::near_key(r); }

int oracle_near_table(float* out) {
  if (!out) return 1;
  oracle::near_table(out);
  return 0;
}

int oracle_philox(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  oracle::philox4x32_10(ctr, key, out);
  return 0;
}

int oracle_eam_read_funcfl(const char* path, int32_t* nrho, int32_t* nr, double* drho, double* dr,
                           double* cut, double* frho, double* zr, double* rhor) {
  oracle::EamFile f;
  if (!oracle::read_funcfl(path, f)) return 9;
  *nrho = f.nrho;
  *nr = f.nr;
  *drho = f.drho;
  *dr = f.dr;
  *cut = f.cut;
  if (frho) std::memcpy(frho, f.frho.data(), sizeof(double) * f.nrho);
  if (zr) std::memcpy(zr, f.zr.data(), sizeof(double) * f.nr);
  if (rhor) std::memcpy(rhor, f.rhor.data(), sizeof(double) * f.nr);
  return 0;
}

int oracle_eam_build_setfl_splines(int32_t ne, int32_t nrho, double drho, int32_t nr, double dr, const double* frho,
                                   const double* rhor, const double* z2r, const int32_t* type_element,
                                   int32_t n_types, double* frho_s, double* rhor_s, double* z2r_s,
                                   double* rhomax) {
  std::vector<double> a, b, c;
  oracle::build_setfl_splines(ne, nrho, drho, nr, dr, frho, rhor, z2r, type_element, n_types, a, b, c, *rhomax);
  std::memcpy(frho_s, a.data(), sizeof(double) * a.size());
  std::memcpy(rhor_s, b.data(), sizeof(double) * b.size());
  std::memcpy(z2r_s, c.data(), sizeof(double) * c.size());
  return 0;
}

int oracle_eam_build_splines(int32_t nrho_in, int32_t nr_in, double drho_in, double dr_in, double cut,
                             const double* frho, const double* zr, const double* rhor,
                             double* frho_s, double* rhor_s, double* z2r_s, int32_t* nrho,
                             double* drho, int32_t* nr, double* dr, double* rhomax) {
  oracle::EamFile f;
  f.nrho = nrho_in;
  f.nr = nr_in;
  f.drho = drho_in;
  f.dr = dr_in;
  f.cut = cut;
  f.frho.assign(frho, frho + nrho_in);
  f.frho.push_back(0.0);
  f.zr.assign(zr, zr + nr_in);
  f.zr.push_back(0.0);
  f.rhor.assign(rhor, rhor + nr_in);
  f.rhor.push_back(0.0);
  std::vector<double> a, b, c;
  int nrho_o, nr_o;
  double drho_o, dr_o, rhomax_o;
  oracle::build_splines(f, a, b, c, nrho_o, drho_o, nr_o, dr_o, rhomax_o);
  if (frho_s) std::memcpy(frho_s, a.data(), sizeof(double) * a.size());
  if (rhor_s) std::memcpy(rhor_s, b.data(), sizeof(double) * b.size());
  if (z2r_s) std::memcpy(z2r_s, c.data(), sizeof(double) * c.size());
  *nrho = nrho_o;
  *nr = nr_o;
  *drho = drho_o;
  *dr = dr_o;
  *rhomax = rhomax_o;
  return 0;
}

}  // extern "C"
