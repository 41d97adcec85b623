// capi.cpp -- extern "C" entry points declared in include/rbmd_gpu.h.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <new>
#include <sstream>
#include <string>
#include <vector>

#include "engine.h"
#include "serve.h"

using rbmd::Context;

struct rbmd_ctx {
  Context* c = nullptr;
  rbmd::Server* server = nullptr;
};

#define CTX_CHECK(ctx)                                 \
  do {                                                 \
    if (!(ctx) || !(ctx)->c) return RBMD_ERR_ARG;      \
  } while (0)

extern "C" {

int rbmd_abi_version(void) { return RBMD_ABI_VERSION; }

void rbmd_params_default(rbmd_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->force_field = RBMD_FF_LJ_CUT;
  p->neighbor = RBMD_NEIGH_RBL;
  p->coulomb = RBMD_COUL_NONE;
  p->ensemble = RBMD_ENS_NVT;
  p->temp_ctrl = RBMD_TC_NOSE_HOOVER;
  p->units = RBMD_UNITS_LJ;
  p->precision = RBMD_PREC_FP64;
  p->rbl_mode = RBMD_RBL_STRIDE;
  p->random_mode = RBMD_RANDOM_PHILOX;
  p->fix_shake = RBMD_SHAKE_NULL;
  p->neighbor_sample_num = 100;
  p->cut_off = 2.5;
  p->r_core = 1.2;
  p->coulomb_sample_num = 100;
  p->kmax[0] = p->kmax[1] = p->kmax[2] = 3;
  p->alpha = 0.1;
  p->temperature[0] = p->temperature[1] = 1.0;
  p->temperature[2] = 0.5;
  p->pressure[0] = p->pressure[1] = 1.0;
  p->pressure[2] = 1000.0;
  p->timestep = 0.005;
  p->num_steps = 1000;
  p->seed = 1;
  p->bulk_modulus = 10.0;
}

int rbmd_ctx_create(const rbmd_device_cfg* cfg, rbmd_ctx** out) {
  if (!out) return RBMD_ERR_ARG;
  *out = nullptr;
  rbmd_device_cfg c{};
  c.batched = 1;
  c.use_graphs = 1;
  if (cfg) c = *cfg;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return RBMD_ERR_CUDA;
  }
  if (c.device < 0 || c.device >= ndev) return RBMD_ERR_ARG;
  auto* h = new (std::nothrow) rbmd_ctx();
  if (!h) return RBMD_ERR_OOM;
  h->c = new Context(c);
  *out = h;
  return RBMD_OK;
}

int rbmd_ctx_destroy(rbmd_ctx* ctx) {
  if (!ctx) return RBMD_ERR_ARG;
  if (ctx->server) {
    ctx->server->stop();
    delete ctx->server;
  }
  delete ctx->c;
  delete ctx;
  return RBMD_OK;
}

const char* rbmd_last_error(const rbmd_ctx* ctx) {
  if (!ctx || !ctx->c) return "null context";
  return ctx->c->last_error.c_str();
}

int rbmd_system_bytes(const rbmd_system_desc* d, const rbmd_params* p, int64_t* bytes) {
  if (!d || !p || !bytes || d->n_atoms <= 0) return RBMD_ERR_ARG;
  *bytes = Context::estimate_bytes(*d, *p);
  return RBMD_OK;
}

int rbmd_system_add(rbmd_ctx* ctx, const rbmd_system_desc* d, const rbmd_params* p, int32_t* id) {
  CTX_CHECK(ctx);
  if (!d || !p || !id) return ctx->c->fail(RBMD_ERR_ARG, "null argument");
  return ctx->c->add_system(*d, *p, id);
}

int rbmd_system_remove(rbmd_ctx* ctx, int32_t id) {
  CTX_CHECK(ctx);
  return ctx->c->remove_system(id);
}

int rbmd_init(rbmd_ctx* ctx, const int32_t* ids, int32_t n) {
  CTX_CHECK(ctx);
  if (!ids || n <= 0) return ctx->c->fail(RBMD_ERR_ARG, "empty system list");
  return ctx->c->init(ids, n);
}

int rbmd_step(rbmd_ctx* ctx, const int32_t* ids, int32_t n, int32_t nsteps) {
  CTX_CHECK(ctx);
  if (!ids || n <= 0 || nsteps < 0) return ctx->c->fail(RBMD_ERR_ARG, "bad step arguments");
  return ctx->c->step(ids, n, nsteps);
}

int rbmd_sync(rbmd_ctx* ctx) {
  CTX_CHECK(ctx);
  return ctx->c->sync();
}

int rbmd_compute_forces(rbmd_ctx* ctx, const int32_t* ids, int32_t n) {
  CTX_CHECK(ctx);
  if (!ids || n <= 0) return ctx->c->fail(RBMD_ERR_ARG, "empty system list");
  return ctx->c->compute_forces(ids, n);
}

int rbmd_get_forces(rbmd_ctx* ctx, int32_t id, double* f) {
  CTX_CHECK(ctx);
  return ctx->c->get_forces(id, f);
}

int rbmd_get_state(rbmd_ctx* ctx, int32_t id, double* x, double* v, int32_t* image) {
  CTX_CHECK(ctx);
  return ctx->c->get_state(id, x, v, image);
}

int rbmd_set_state(rbmd_ctx* ctx, int32_t id, const double* x, const double* v, const int32_t* image) {
  CTX_CHECK(ctx);
  return ctx->c->set_state(id, x, v, image);
}

int rbmd_set_step(rbmd_ctx* ctx, int32_t id, int64_t step) {
  CTX_CHECK(ctx);
  return ctx->c->set_step(id, step);
}

int rbmd_get_thermo(rbmd_ctx* ctx, int32_t id, rbmd_thermo* out) {
  CTX_CHECK(ctx);
  return ctx->c->get_thermo(id, out);
}

int rbmd_get_cells(rbmd_ctx* ctx, int32_t id, int32_t* dims, int32_t* coa, int32_t* sorted,
                   int32_t* lo, int32_t* up) {
  CTX_CHECK(ctx);
  return ctx->c->get_cells(id, dims, coa, sorted, lo, up);
}

int rbmd_get_rbl_lists(rbmd_ctx* ctx, int32_t id, int32_t cap, int32_t* nc, int32_t* ns, int32_t* ids) {
  CTX_CHECK(ctx);
  return ctx->c->get_rbl_lists(id, cap, nc, ns, ids);
}

int rbmd_get_rbl_lists_static(rbmd_ctx* ctx, int32_t id, int32_t cap, int32_t* nc, int32_t* ns,
                              int32_t* ids) {
  CTX_CHECK(ctx);
  return ctx->c->get_rbl_lists_static(id, cap, nc, ns, ids);
}

int rbmd_get_kspace(rbmd_ctx* ctx, int32_t id, int32_t* m, double* rhok) {
  CTX_CHECK(ctx);
  return ctx->c->get_kspace(id, m, rhok);
}

int rbmd_get_derived(rbmd_ctx* ctx, int32_t id, rbmd_derived* out) {
  CTX_CHECK(ctx);
  if (!out) return RBMD_ERR_ARG;
  return ctx->c->get_derived(id, out);
}

int rbmd_observe_reset(rbmd_ctx* ctx, int32_t id, int32_t which) {
  CTX_CHECK(ctx);
  return ctx->c->observe_reset(id, which);
}

int rbmd_observe(rbmd_ctx* ctx, int32_t id, double* msd, double* vacf) {
  CTX_CHECK(ctx);
  return ctx->c->observe(id, msd, vacf);
}

int rbmd_rdf_bins(double radius, double dr, double* radii, int32_t cap, int32_t* n_bins) {
  std::vector<double> r;
  const int nb = rbmd::rdf_bins(radius, dr, radii ? &r : nullptr);
  if (nb < 0) return RBMD_ERR_ARG;
  if (n_bins) *n_bins = nb;
  if (radii)
    for (int b = 0; b < nb && b < cap; ++b) radii[b] = r[b];
  return RBMD_OK;
}

int32_t rbmd_near_table_key(float r) { return rbmd::near_table_key(r); }

int rbmd_near_table_default(float* out) {
  if (!out) return RBMD_ERR_ARG;
  rbmd::near_table_default(out);
  return RBMD_OK;
}

int rbmd_rdf_counts(rbmd_ctx* ctx, int32_t id, const int32_t* centers, int32_t nc, const int32_t* targets, int32_t nt,
                    double radius, double dr, int32_t exclude_same_molecule, int64_t* counts, double* volume) {
  CTX_CHECK(ctx);
  return ctx->c->rdf_counts(id, centers, nc, targets, nt, radius, dr, exclude_same_molecule, counts, volume);
}

int rbmd_snapshot_begin(rbmd_ctx* ctx, int32_t id, double* x, double* v, int32_t* image, double* box, int64_t* step,
                        int64_t* ticket) {
  CTX_CHECK(ctx);
  return ctx->c->snapshot_begin(id, x, v, image, box, step, ticket);
}

int rbmd_snapshot_poll(rbmd_ctx* ctx, int64_t ticket, int32_t* done) {
  CTX_CHECK(ctx);
  if (!done) return RBMD_ERR_ARG;
  int d = 0;
  const int rc = ctx->c->snapshot_poll(ticket, &d);
  *done = d;
  return rc;
}

int rbmd_snapshot_wait(rbmd_ctx* ctx, int64_t ticket, double timeout_s) {
  CTX_CHECK(ctx);
  return ctx->c->snapshot_wait(ticket, timeout_s);
}

// ------------------------------------------------------------------ EAM input (host)
int rbmd_eam_read_funcfl(const char* path, rbmd_eam_file* out, double* frho, double* zr, double* rhor) {
  // ExecutionNVT::ReadPotentialFile, framework/run/ExecutionNVT.cpp:899-931: two comment lines,
  // then "nrho drho nr dr cutoff", then frho[nrho], zr[nr], rhor[nr].
  if (!path || !out) return RBMD_ERR_ARG;
  std::ifstream in(path);
  if (!in.is_open()) return RBMD_ERR_IO;
  for (int i = 0; i < 2; ++i) in.ignore(std::numeric_limits<std::streamsize>::max(), '\n');
  int nrho = 0, nr = 0;
  double drho = 0, dr = 0, cut = 0;
  in >> nrho >> drho >> nr >> dr >> cut;
  if (!in || nrho < 5 || nr < 5) return RBMD_ERR_IO;
  out->nrho = nrho;
  out->nr = nr;
  out->drho = drho;
  out->dr = dr;
  out->cut_off = cut;
  if (!frho && !zr && !rhor) return RBMD_OK;
  if (!frho || !zr || !rhor) return RBMD_ERR_ARG;
  for (int i = 0; i < nrho; ++i) in >> frho[i];
  for (int i = 0; i < nr; ++i) in >> zr[i];
  for (int i = 0; i < nr; ++i) in >> rhor[i];
  if (!in) return RBMD_ERR_IO;
  out->frho = frho;
  out->zr = zr;
  out->rhor = rhor;
  return RBMD_OK;
}

int rbmd_eam_spline_sizes(const rbmd_eam_file* in, int32_t* nrho_out, int32_t* nr_out) {
  if (!in || !nrho_out || !nr_out || in->nrho < 5 || in->nr < 5) return RBMD_ERR_ARG;
  const double rmax = (in->nr - 1) * in->dr, rhomax = (in->nrho - 1) * in->drho;
  *nr_out = (int)(rmax / in->dr + 0.5);
  *nrho_out = (int)(rhomax / in->drho + 0.5);
  return RBMD_OK;
}

static void eam_interpolate(int n, double delta, const std::vector<double>& f, double* s) {
  // ExecutionNVT::interpolate, framework/run/ExecutionNVT.cpp:1033-1068
  auto S = [&](int m, int c) -> double& { return s[7 * m + c]; };
  for (int m = 1; m <= n; m++) S(m, 6) = f[m];
  S(1, 5) = S(2, 6) - S(1, 6);
  S(2, 5) = 0.5 * (S(3, 6) - S(1, 6));
  S(n - 1, 5) = 0.5 * (S(n, 6) - S(n - 2, 6));
  S(n, 5) = S(n, 6) - S(n - 1, 6);
  for (int m = 3; m <= n - 2; m++)
    S(m, 5) = ((S(m - 2, 6) - S(m + 2, 6)) + 8.0 * (S(m + 1, 6) - S(m - 1, 6))) / 12.0;
  for (int m = 1; m <= n - 1; m++) {
    S(m, 4) = 3.0 * (S(m + 1, 6) - S(m, 6)) - 2.0 * S(m, 5) - S(m + 1, 5);
    S(m, 3) = S(m, 5) + S(m + 1, 5) - 2.0 * (S(m + 1, 6) - S(m, 6));
  }
  S(n, 4) = 0.0;
  S(n, 3) = 0.0;
  for (int m = 1; m <= n; m++) {
    S(m, 2) = S(m, 5) / delta;
    S(m, 1) = 2.0 * S(m, 4) / delta;
    S(m, 0) = 3.0 * S(m, 3) / delta;
  }
}

int rbmd_eam_read_setfl(const char* path, rbmd_eam_setfl* out, char* names, double* mass, double* frho,
                        double* rhor, double* z2r) {
  // LAMMPS pair eam/alloy read_file: 3 comment lines, elements line, grid line, per-element
  // blocks, then the lower triangle of r phi tables.
  if (!path || !out) return RBMD_ERR_ARG;
  std::ifstream in(path);
  if (!in.is_open()) return RBMD_ERR_IO;
  for (int i = 0; i < 3; ++i) in.ignore(std::numeric_limits<std::streamsize>::max(), '\n');
  std::string line;
  if (!std::getline(in, line)) return RBMD_ERR_IO;
  std::istringstream el(line);
  int ne = 0;
  el >> ne;
  if (!el || ne < 1 || ne > 64) return RBMD_ERR_IO;
  std::vector<std::string> nm(ne);
  for (int e = 0; e < ne; ++e)
    if (!(el >> nm[e])) return RBMD_ERR_IO;
  int nrho = 0, nr = 0;
  double drho = 0, dr = 0, cut = 0;
  in >> nrho >> drho >> nr >> dr >> cut;
  if (!in || nrho < 5 || nr < 5 || !(drho > 0) || !(dr > 0) || !(cut > 0)) return RBMD_ERR_IO;
  out->n_elements = ne;
  out->nrho = nrho;
  out->nr = nr;
  out->pad0 = 0;
  out->drho = drho;
  out->dr = dr;
  out->cut_off = cut;
  if (!names && !mass && !frho && !rhor && !z2r) return RBMD_OK;
  if (!frho || !rhor || !z2r) return RBMD_ERR_ARG;
  for (int e = 0; e < ne; ++e) {
    int z = 0;
    double m = 0, a = 0;
    std::string lat;
    in >> z >> m >> a >> lat;
    if (!in) return RBMD_ERR_IO;
    if (mass) mass[e] = m;
    if (names) {
      std::memset(names + 16 * e, 0, 16);
      std::strncpy(names + 16 * e, nm[e].c_str(), 15);
    }
    for (int k = 0; k < nrho; ++k) in >> frho[(size_t)e * nrho + k];
    for (int k = 0; k < nr; ++k) in >> rhor[(size_t)e * nr + k];
    if (!in) return RBMD_ERR_IO;
  }
  const size_t pairs = (size_t)ne * (ne + 1) / 2;
  for (size_t q = 0; q < pairs; ++q)
    for (int k = 0; k < nr; ++k) in >> z2r[q * nr + k];
  if (!in) return RBMD_ERR_IO;
  return RBMD_OK;
}

int rbmd_eam_build_setfl_splines(const rbmd_eam_setfl* in, const double* frho, const double* rhor,
                                 const double* z2r, const int32_t* type_element, int32_t n_types,
                                 double* frho_s, double* rhor_s, double* z2r_s, double* rhomax_out) {
  // LAMMPS PairEAMAlloy::file2array (the file's grid, arrays copied) then array2spline.
  if (!in || !frho || !rhor || !z2r || !type_element || n_types < 1 || !frho_s || !rhor_s || !z2r_s)
    return RBMD_ERR_ARG;
  const int ne = in->n_elements, nrho = in->nrho, nr = in->nr;
  if (ne < 1 || nrho < 5 || nr < 5) return RBMD_ERR_ARG;
  for (int t = 0; t < n_types; ++t)
    if (type_element[t] < 0 || type_element[t] >= ne) return RBMD_ERR_ARG;
  const size_t rf = 7 * (size_t)(nrho + 1), rr = 7 * (size_t)(nr + 1);
  std::vector<double> f(std::max(nrho, nr) + 1, 0.0);
  auto spline = [&](const double* src, int n, double delta, double* dst) {
    std::fill(f.begin(), f.end(), 0.0);
    for (int m = 1; m <= n; ++m) f[m] = src[m - 1];
    std::memset(dst, 0, sizeof(double) * 7 * (n + 1));
    eam_interpolate(n, delta, f, dst);
  };
  for (int t = 0; t < n_types; ++t) {
    const int e = type_element[t];
    spline(frho + (size_t)e * nrho, nrho, in->drho, frho_s + t * rf);
    spline(rhor + (size_t)e * nr, nr, in->dr, rhor_s + t * rr);
  }
  for (int i = 0; i < n_types; ++i)
    for (int j = 0; j <= i; ++j) {
      const int a = std::max(type_element[i], type_element[j]), b = std::min(type_element[i], type_element[j]);
      spline(z2r + (size_t)(a * (a + 1) / 2 + b) * nr, nr, in->dr, z2r_s + (size_t)(i * (i + 1) / 2 + j) * rr);
    }
  if (rhomax_out) *rhomax_out = (nrho - 1) * in->drho;
  return RBMD_OK;
}

int rbmd_eam_build_splines(const rbmd_eam_file* in, double* frho_s, double* rhor_s, double* z2r_s,
                           int32_t* nrho_out, double* drho_out, int32_t* nr_out, double* dr_out,
                           double* rhomax_out) {
  // ExecutionNVT::file2array + array2spline, framework/run/ExecutionNVT.cpp:933-1079: 4-point
  // Lagrange resampling, z2r = 27.2 * 0.529 * Z^2, then the 7-coefficient cubic rows.
  if (!in || !in->frho || !in->zr || !in->rhor || !frho_s || !rhor_s || !z2r_s) return RBMD_ERR_ARG;
  int nrho, nr;
  if (rbmd_eam_spline_sizes(in, &nrho, &nr)) return RBMD_ERR_ARG;
  const double sixth = 1.0 / 6.0;
  const double dr = in->dr, drho = in->drho;
  auto lag = [&](const double* src, int nsrc, double h, double r) {
    double p = r / h + 1.0;
    int k = (int)p;
    k = std::min(k, nsrc - 2);
    k = std::max(k, 2);
    p -= k;
    p = std::min(p, 2.0);
    const double c1 = -sixth * p * (p - 1.0) * (p - 2.0);
    const double c2 = 0.5 * (p * p - 1.0) * (p - 2.0);
    const double c3 = -0.5 * p * (p + 1.0) * (p - 2.0);
    const double c4 = sixth * p * (p * p - 1.0);
    auto at = [&](int idx) { return idx < nsrc ? src[idx] : 0.0; };
    return c1 * at(k - 1) + c2 * at(k) + c3 * at(k + 1) + c4 * at(k + 2);
  };
  std::vector<double> frho(nrho + 1, 0.0), rhor(nr + 1, 0.0), z2r(nr + 1, 0.0);
  for (int m = 1; m <= nrho; m++) frho[m] = lag(in->frho, in->nrho, in->drho, (m - 1) * drho);
  for (int m = 1; m <= nr; m++) rhor[m] = lag(in->rhor, in->nr, in->dr, (m - 1) * dr);
  for (int m = 1; m <= nr; m++) {
    const double zri = lag(in->zr, in->nr, in->dr, (m - 1) * dr);
    z2r[m] = 27.2 * 0.529 * zri * zri;
  }
  std::memset(frho_s, 0, sizeof(double) * 7 * (nrho + 1));
  std::memset(rhor_s, 0, sizeof(double) * 7 * (nr + 1));
  std::memset(z2r_s, 0, sizeof(double) * 7 * (nr + 1));
  eam_interpolate(nrho, drho, frho, frho_s);
  eam_interpolate(nr, dr, rhor, rhor_s);
  eam_interpolate(nr, dr, z2r, z2r_s);
  if (nrho_out) *nrho_out = nrho;
  if (nr_out) *nr_out = nr;
  if (drho_out) *drho_out = drho;
  if (dr_out) *dr_out = dr;
  if (rhomax_out) *rhomax_out = (in->nrho - 1) * in->drho;
  return RBMD_OK;
}

// ------------------------------------------------------------------ serving
int rbmd_serve_start(rbmd_ctx* ctx, const rbmd_serve_cfg* cfg) {
  CTX_CHECK(ctx);
  if (ctx->server) return ctx->c->fail(RBMD_ERR_STATE, "serving loop already running");
  rbmd_serve_cfg c{};
  c.steps_per_round = 10;
  c.use_graphs = 1;
  if (cfg) c = *cfg;
  ctx->server = new rbmd::Server(ctx->c, c);
  return ctx->server->start();
}

int rbmd_serve_submit(rbmd_ctx* ctx, const rbmd_system_desc* d, const rbmd_params* p, int32_t nsteps,
                      int64_t* rid) {
  CTX_CHECK(ctx);
  if (!ctx->server) return ctx->c->fail(RBMD_ERR_STATE, "serving loop not started");
  if (!d || !p || !rid || nsteps < 0) return ctx->c->fail(RBMD_ERR_ARG, "bad submit arguments");
  return ctx->server->submit(*d, *p, nsteps, rid);
}

int rbmd_serve_poll(rbmd_ctx* ctx, int64_t rid, int32_t* state) {
  CTX_CHECK(ctx);
  if (!ctx->server) return ctx->c->fail(RBMD_ERR_STATE, "serving loop not started");
  return ctx->server->poll(rid, state);
}

int rbmd_serve_wait(rbmd_ctx* ctx, int64_t rid, double timeout_s) {
  CTX_CHECK(ctx);
  if (!ctx->server) return ctx->c->fail(RBMD_ERR_STATE, "serving loop not started");
  return ctx->server->wait(rid, timeout_s);
}

int rbmd_serve_result(rbmd_ctx* ctx, int64_t rid, double* x, double* v, rbmd_thermo* th,
                      rbmd_request_stats* stats) {
  CTX_CHECK(ctx);
  if (!ctx->server) return ctx->c->fail(RBMD_ERR_STATE, "serving loop not started");
  return ctx->server->result(rid, x, v, th, stats);
}

int rbmd_serve_stop(rbmd_ctx* ctx) {
  CTX_CHECK(ctx);
  if (!ctx->server) return RBMD_OK;
  int rc = ctx->server->stop();
  delete ctx->server;
  ctx->server = nullptr;
  return rc;
}

// ------------------------------------------------------------------ diagnostics
int rbmd_launch_count(rbmd_ctx* ctx, int64_t* launches) {
  CTX_CHECK(ctx);
  if (!launches) return RBMD_ERR_ARG;
  *launches = rbmd::launches_issued();
  return RBMD_OK;
}

int rbmd_profile_enable(rbmd_ctx* ctx, int32_t on) {
  CTX_CHECK(ctx);
  std::lock_guard<std::recursive_mutex> lk(ctx->c->mu);
  ctx->c->sync();
  for (auto& r : ctx->c->prof.recs)
    for (auto& e : r.second.ev) {
      cudaEventDestroy(e.first);
      cudaEventDestroy(e.second);
    }
  ctx->c->prof.recs.clear();
  ctx->c->prof.on = on != 0;
  return RBMD_OK;
}

int rbmd_profile_get(rbmd_ctx* ctx, const char* kernel, double* avg_ms, int64_t* launches,
                     double* units_per_launch) {
  CTX_CHECK(ctx);
  if (!kernel) return RBMD_ERR_ARG;
  std::lock_guard<std::recursive_mutex> lk(ctx->c->mu);
  int rc = ctx->c->sync();
  if (rc) return rc;
  auto it = ctx->c->prof.recs.find(kernel);
  if (it == ctx->c->prof.recs.end()) {
    if (avg_ms) *avg_ms = 0;
    if (launches) *launches = 0;
    if (units_per_launch) *units_per_launch = 0;
    return RBMD_OK;
  }
  auto& r = it->second;
  for (size_t k = 0; k < r.ev.size(); ++k) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, r.ev[k].first, r.ev[k].second);
    r.ms += ms;
    r.n += 1;
    r.units_sum += r.units[k];
    cudaEventDestroy(r.ev[k].first);
    cudaEventDestroy(r.ev[k].second);
  }
  r.ev.clear();
  r.units.clear();
  if (avg_ms) *avg_ms = r.n ? r.ms / r.n : 0.0;
  if (launches) *launches = r.n;
  if (units_per_launch) *units_per_launch = r.n ? r.units_sum / r.n : 0.0;
  return RBMD_OK;
}

int rbmd_autotune(rbmd_ctx* ctx, const int32_t* ids, int32_t n, rbmd_tune_result* results, int32_t cap,
                  int32_t* n_groups) {
  CTX_CHECK(ctx);
  if (!ids || n <= 0 || cap < 0 || (cap > 0 && !results)) return ctx->c->fail(RBMD_ERR_ARG, "bad autotune arguments");
  int ng = 0;
  rbmd_tune_result dummy;
  const int rc = ctx->c->autotune(ids, n, cap > 0 ? results : &dummy, cap, &ng, true);
  if (n_groups) *n_groups = ng;
  return rc;
}

int rbmd_step_timed(rbmd_ctx* ctx, const int32_t* ids, int32_t n, int32_t nsteps, double* ms) {
  CTX_CHECK(ctx);
  if (!ids || n <= 0 || nsteps < 0 || !ms) return ctx->c->fail(RBMD_ERR_ARG, "bad step arguments");
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  cudaEventRecord(a, ctx->c->stream);
  int rc = ctx->c->step(ids, n, nsteps);
  cudaEventRecord(b, ctx->c->stream);
  cudaEventSynchronize(b);
  float t = 0.f;
  cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = t;
  return rc;
}

int rbmd_fma_peak(rbmd_ctx* ctx, int32_t fp64, double* tflops) {
  CTX_CHECK(ctx);
  if (!tflops) return RBMD_ERR_ARG;
  *tflops = rbmd::fma_peak_tflops(fp64, ctx->c->stream);
  return RBMD_OK;
}

}  // extern "C"
