// app.cpp -- the `rbmd` host (see app.hpp).
#include "app.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <fstream>
#include <random>
#include <stdexcept>

namespace rbmd_host {

namespace {

const double kPi = 3.14159265358979323846;

std::string dir_of(const std::string& path) {
  const size_t k = path.find_last_of('/');
  return k == std::string::npos ? std::string(".") : path.substr(0, k);
}

bool exists(const std::string& p) { return std::ifstream(p).good(); }

// Gaussian velocities as the reference draws them (ModelFileInitCondition::Velocity, :605-655;
// MeshFreeCondition::InitMassAndVelocity): three Box-Muller normals per atom scaled by sigma.
// The stream is a seeded mt19937_64 where the reference takes std::random_device.
void gauss_velocities(Para& p, const std::vector<double>& sigma_of_atom) {
  std::mt19937_64 g(p.params.seed);
  std::uniform_real_distribution<double> u(0.0, 1.0);
  p.velocity.assign(3 * (size_t)p.n, 0.0);
  for (int i = 0; i < p.n; ++i)
    for (int k = 0; k < 3; ++k) {
      double u1 = u(g);
      while (u1 <= 0.0) u1 = u(g);
      const double u2 = u(g);
      p.velocity[3 * (size_t)i + k] = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2) * sigma_of_atom[i];
    }
}

int units_of(const std::string& u) {
  if (u == "LJ") return RBMD_UNITS_LJ;
  if (u == "REAL") return RBMD_UNITS_REAL;
  if (u == "METAL") return RBMD_UNITS_METAL;
  throw std::runtime_error("unit must be LJ, REAL or METAL, not \"" + u + "\"");
}

}  // namespace

rbmd_system_desc Para::desc() const {
  rbmd_system_desc d;
  std::memset(&d, 0, sizeof(d));
  d.n_atoms = n;
  d.n_types = n_types;
  for (int k = 0; k < 3; ++k) {
    d.box_lo[k] = lo[k];
    d.box_hi[k] = hi[k];
  }
  d.position = position.data();
  d.velocity = velocity.empty() ? nullptr : velocity.data();
  d.charge = charge.empty() ? nullptr : charge.data();
  d.mass = mass.data();
  d.type = type.data();
  d.molecule = molecule.empty() ? nullptr : molecule.data();
  d.epsilon = eps.data();
  d.sigma = sigma.data();
  d.n_bonds = (int32_t)bond_type.size();
  d.n_bond_types = (int32_t)bond_k.size();
  d.bond_atoms = bond_atoms.empty() ? nullptr : bond_atoms.data();
  d.bond_type = bond_type.empty() ? nullptr : bond_type.data();
  d.bond_k = bond_k.empty() ? nullptr : bond_k.data();
  d.bond_r0 = bond_r0.empty() ? nullptr : bond_r0.data();
  d.n_angles = (int32_t)angle_type.size();
  d.n_angle_types = (int32_t)angle_k.size();
  d.angle_atoms = angle_atoms.empty() ? nullptr : angle_atoms.data();
  d.angle_type = angle_type.empty() ? nullptr : angle_type.data();
  d.angle_k = angle_k.empty() ? nullptr : angle_k.data();
  d.angle_theta0 = angle_theta0.empty() ? nullptr : angle_theta0.data();
  if (!sp_off.empty()) {
    d.special_offsets = sp_off.data();
    d.special_ids = sp_ids.data();
    d.special_weights = sp_w.data();
  }
  d.eam_nrho = eam_nrho;
  d.eam_nr = eam_nr;
  d.eam_drho = eam_drho;
  d.eam_dr = eam_dr;
  d.eam_rhomax = eam_rhomax;
  d.eam_cut = eam_cut;
  d.eam_frho_spline = frho_spline.empty() ? nullptr : frho_spline.data();
  d.eam_rhor_spline = rhor_spline.empty() ? nullptr : rhor_spline.data();
  d.eam_z2r_spline = z2r_spline.empty() ? nullptr : z2r_spline.data();
  d.eam_per_type = eam_per_type;
  d.near_table_values = near_table.empty() ? nullptr : near_table.data();
  if (!dihedral_type.empty()) {
    d.n_dihedrals = (int32_t)dihedral_type.size();
    d.n_dihedral_types = (int32_t)dihedral_k.size();
    d.dihedral_atoms = dihedral_atoms.data();
    d.dihedral_type = dihedral_type.data();
    d.dihedral_k = dihedral_k.data();
    d.dihedral_sign = dihedral_sign.data();
    d.dihedral_multiplicity = dihedral_multiplicity.data();
  }
  return d;
}

// ------------------------------------------------------------------------------------------ init
ModelFileInitCondition::ModelFileInitCondition(const Json& cfg, const std::string& base_dir) {
  _file = cfg.string("file", "");
  if (_file.empty()) throw std::runtime_error("read_data needs \"file\"");
  if (!exists(_file) && exists(base_dir + "/" + _file)) _file = base_dir + "/" + _file;
  _atom_style = cfg.string("atom_style", "atomic");
  _velocity_type = cfg.string("velocity_type", "GAUSS");
}

void ModelFileInitCondition::Execute(Para& p) {
  const DataFile d = read_data_file(_file, _atom_style, p.unit);
  p.init_way = "read_data";
  p.atom_style = _atom_style;
  p.n = d.n_atoms;
  p.n_types = d.n_types;
  for (int k = 0; k < 3; ++k) {
    p.lo[k] = d.lo[k];
    p.hi[k] = d.hi[k];
  }
  p.position = d.position;
  p.charge = d.charge;
  p.type = d.type;
  p.molecule = d.molecule;
  p.eps = d.type_eps;
  p.sigma = d.type_sigma;
  p.mass.resize(p.n);
  for (int i = 0; i < p.n; ++i) p.mass[i] = d.type_mass[d.type[i]];
  p.bond_atoms = d.bond_atoms;
  p.bond_type = d.bond_type;
  p.bond_k = d.bond_k;
  p.bond_r0 = d.bond_r0;
  p.angle_atoms = d.angle_atoms;
  p.angle_type = d.angle_type;
  p.angle_k = d.angle_k;
  p.angle_theta0 = d.angle_theta0;
  p.file_dihedrals = d.has_dihedrals;
  p.dihedral_atoms = d.dihedral_atoms;
  p.dihedral_type = d.dihedral_type;
  p.dihedral_k = d.dihedral_k;
  p.dihedral_sign = d.dihedral_sign;
  p.dihedral_multiplicity = d.dihedral_multiplicity;
  if (!d.velocity.empty()) {
    p.velocity = d.velocity;
  } else if (_velocity_type == "GAUSS") {
    // REAL: sqrt(kB 298 / m); other units sqrt(1 / m) (ModelFileInitCondition.cpp:622-633)
    std::vector<double> sg(p.n);
    for (int i = 0; i < p.n; ++i)
      sg[i] = std::sqrt((p.unit == "REAL" ? 1.9872067e-3 * 298.0 : 1.0) / p.mass[i]);
    gauss_velocities(p, sg);
  } else {
    p.velocity.assign(3 * (size_t)p.n, 0.0);  // "ZERO", "TEST" and anything else (:641)
  }
}

MeshFreeCondition::MeshFreeCondition(const Json& cfg) {
  const std::vector<double> dims = cfg.numbers("dims");
  if (dims.size() != 3) throw std::runtime_error("inbuild needs \"dims\": [nx, ny, nz]");
  const char* keys[3] = {"x_range", "y_range", "z_range"};
  for (int k = 0; k < 3; ++k) {
    _dims[k] = (int)dims[k];
    if (_dims[k] <= 0) throw std::runtime_error("inbuild dims must be positive");
    const std::vector<double> r = cfg.numbers(keys[k]);
    if (r.size() != 2 || !(r[1] > r[0])) throw std::runtime_error(std::string("inbuild needs \"") + keys[k] + "\": [lo, hi]");
    _range[k][0] = r[0];
    _range[k][1] = r[1];
  }
  _velocity_type = cfg.string("velocity_type", "GAUSS");
}

void MeshFreeCondition::Execute(Para& p) {
  // one atom at the centre of every cell of the dims grid, x fastest (RunWorklet InitPosition)
  p.init_way = "inbuild";
  p.params.init_inbuild = 1;
  p.n = _dims[0] * _dims[1] * _dims[2];
  p.n_types = 1;
  double sp[3];
  for (int k = 0; k < 3; ++k) {
    p.lo[k] = _range[k][0];
    p.hi[k] = _range[k][1];
    sp[k] = (_range[k][1] - _range[k][0]) / _dims[k];
  }
  p.position.resize(3 * (size_t)p.n);
  int a = 0;
  for (int kz = 0; kz < _dims[2]; ++kz)
    for (int ky = 0; ky < _dims[1]; ++ky)
      for (int kx = 0; kx < _dims[0]; ++kx, ++a) {
        p.position[3 * (size_t)a] = p.lo[0] + (kx + 0.5) * sp[0];
        p.position[3 * (size_t)a + 1] = p.lo[1] + (ky + 0.5) * sp[1];
        p.position[3 * (size_t)a + 2] = p.lo[2] + (kz + 0.5) * sp[2];
      }
  p.mass.assign(p.n, 1.0);
  p.type.assign(p.n, 0);
  p.molecule.clear();
  p.charge.assign(p.n, 0.0);
  p.eps.assign(1, 1.0);
  p.sigma.assign(1, 1.0);
  if (_velocity_type == "GAUSS")
    gauss_velocities(p, std::vector<double>(p.n, 1.0));  // unit variance (MeshFreeCondition.cpp:82-98)
  else
    p.velocity.assign(3 * (size_t)p.n, 0.0);
}

// ----------------------------------------------------------------------------------- execution
ExecutionMD::ExecutionMD(Para& para, int device) : _para(para), _device(device) {}

ExecutionMD::~ExecutionMD() {
  if (_ctx) rbmd_ctx_destroy(_ctx);
}

void ExecutionMD::check(int rc, const char* what) {
  if (rc == RBMD_OK) return;
  const char* msg = _ctx ? rbmd_last_error(_ctx) : "";
  throw std::runtime_error(std::string(what) + " failed (status " + std::to_string(rc) + "): " + (msg ? msg : ""));
}

void ExecutionMD::Init() {
  rbmd_device_cfg cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.device = _device;
  cfg.batched = 0;
  cfg.use_graphs = 1;
  cfg.autotune = _para.autotune ? 1 : 0;
  check(rbmd_ctx_create(&cfg, &_ctx), "rbmd_ctx_create");
  const rbmd_system_desc d = _para.desc();
  check(rbmd_system_add(_ctx, &d, &_para.params, &_sys), "rbmd_system_add");
  check(rbmd_init(_ctx, &_sys, 1), "rbmd_init");
}

rbmd_thermo ExecutionMD::Thermo() {
  rbmd_thermo t;
  check(rbmd_get_thermo(_ctx, _sys, &t), "rbmd_get_thermo");
  return t;
}

void ExecutionMD::State(std::vector<double>& x, std::vector<double>& v, std::vector<int>& image) {
  x.resize(3 * (size_t)_para.n);
  v.resize(3 * (size_t)_para.n);
  image.resize(3 * (size_t)_para.n);
  check(rbmd_get_state(_ctx, _sys, x.data(), v.data(), image.data()), "rbmd_get_state");
}

void ExecutionNVT::Execute() { check(rbmd_step(_ctx, &_sys, 1, 1), "rbmd_step"); }

int64_t ExecutionMD::SnapshotBegin(StateSnapshot& s) {
  s.x.resize(3 * (size_t)_para.n);
  s.v.resize(3 * (size_t)_para.n);
  s.image.resize(3 * (size_t)_para.n);
  int64_t t = 0;
  check(rbmd_snapshot_begin(_ctx, _sys, s.x.data(), s.v.data(), s.image.data(), s.box, &s.step, &t),
        "rbmd_snapshot_begin");
  return t;
}

bool ExecutionMD::SnapshotDone(int64_t ticket) {
  int32_t done = 0;
  check(rbmd_snapshot_poll(_ctx, ticket, &done), "rbmd_snapshot_poll");
  return done != 0;
}

void ExecutionMD::SnapshotWait(int64_t ticket) { check(rbmd_snapshot_wait(_ctx, ticket, -1.0), "rbmd_snapshot_wait"); }

void ExecutionMD::ObserveReset(int which) { check(rbmd_observe_reset(_ctx, _sys, which), "rbmd_observe_reset"); }

void ExecutionMD::Observe(double* msd, double* vacf) { check(rbmd_observe(_ctx, _sys, msd, vacf), "rbmd_observe"); }

double ExecutionMD::RdfCounts(const std::vector<int>& centers, const std::vector<int>& targets, double radius,
                              double dr, bool exclude_same_molecule, std::vector<int64_t>& counts) {
  int32_t nb = 0;
  check(rbmd_rdf_bins(radius, dr, nullptr, 0, &nb), "rbmd_rdf_bins");
  counts.assign(nb, 0);
  double volume = 0.0;
  check(rbmd_rdf_counts(_ctx, _sys, centers.data(), (int32_t)centers.size(), targets.data(), (int32_t)targets.size(),
                        radius, dr, exclude_same_molecule ? 1 : 0, counts.data(), &volume),
        "rbmd_rdf_counts");
  return volume;
}

// ------------------------------------------------------------------------------------- outputs
ThermoOutput::ThermoOutput(int interval, const std::string& path, const std::string& temp_path, bool console)
    : _interval(std::max(1, interval)), _console(console) {
  _file = std::fopen(path.c_str(), "w");
  if (!_file) throw std::runtime_error("cannot write " + path);
  _temp = std::fopen(temp_path.c_str(), "w");
  if (!_temp) throw std::runtime_error("cannot write " + temp_path);
}

ThermoOutput::~ThermoOutput() {
  if (_file) std::fclose(_file);
  if (_temp) std::fclose(_temp);
}

void ThermoOutput::Execute(Executioner& ex) {
  const int64_t step = ex.CurrentStep();
  if (step == 0) {
    std::fprintf(_file, "Step Time VanderWaalsEnergy NearCoulombicEnergy FarCoulombicEnergy KinticEnergy "
                        "PotentialEnergy TotalEnergy BondEnergy AngleEnergy DihedralEnergy Temperature Pressure\n");
    std::fprintf(_temp, "Step Temperature Pressure\n");
  }
  if (step % _interval != 0 && step != ex.NumStep()) return;
  const rbmd_thermo t = ex.Run().Thermo();
  std::fprintf(_temp, "%lld %g %g\n", (long long)step, t.temperature, t.pressure);
  std::fflush(_temp);
  const double vdw = t.e_lj + t.e_eam;
  std::fprintf(_file, "%lld %.10g %.10g %.10g %.10g %.10g %.10g %.10g %.10g %.10g %.10g %.10g %.10g\n",
               (long long)step, ex.CurrentTime(), vdw, t.e_coul_near, t.e_coul_far, t.kinetic_energy,
               t.potential_energy, t.total_energy, t.e_bond, t.e_angle, t.e_dihedral, t.temperature, t.pressure);
  std::fflush(_file);
  if (_console)
    std::printf("step %lld  T %.6g  E_pot %.10g  E_tot %.10g  P %.6g%s\n", (long long)step, t.temperature,
                t.potential_energy, t.total_energy, t.pressure, t.status ? "  (device status set)" : "");
  if (t.status) throw std::runtime_error("device status word " + std::to_string(t.status) + " at step " + std::to_string(step));
}

void SnapshotOutput::Execute(Executioner& ex) {
  // write every snapshot that has landed, oldest first; make room when too many are in flight
  while (!_pending.empty() && (ex.Run().SnapshotDone(_pending.front()->ticket) || _pending.size() >= kInFlight)) {
    ex.Run().SnapshotWait(_pending.front()->ticket);
    Write(*_pending.front());
    _pending.erase(_pending.begin());
  }
  if (!ShouldOutput(ex)) return;
  auto s = std::make_unique<StateSnapshot>();
  s->ticket = ex.Run().SnapshotBegin(*s);
  _pending.push_back(std::move(s));
}

void SnapshotOutput::Finish(Executioner& ex) {
  for (auto& s : _pending) {
    ex.Run().SnapshotWait(s->ticket);
    Write(*s);
  }
  _pending.clear();
}

TrajectoryOutput::TrajectoryOutput(const Para& para, int interval, const std::string& path)
    : _para(para), _interval(std::max(1, interval)) {
  _file = std::fopen(path.c_str(), "w");
  if (!_file) throw std::runtime_error("cannot write " + path);
}

TrajectoryOutput::~TrajectoryOutput() {
  if (_file) std::fclose(_file);
}

bool TrajectoryOutput::ShouldOutput(const Executioner& ex) const {
  return ex.CurrentStep() >= 1 && ex.CurrentStep() % _interval == 0;
}

void TrajectoryOutput::Write(const StateSnapshot& s) {
  const size_t n = s.x.size() / 3;
  std::fprintf(_file, "ITEM: TIMESTEP\n%lld\nITEM: NUMBER OF ATOMS\n%zu\nITEM: BOX BOUNDS pp pp pp\n", (long long)s.step, n);
  for (int k = 0; k < 3; ++k) std::fprintf(_file, "%g %g\n", s.box[k], s.box[3 + k]);
  std::fprintf(_file, "ITEM: ATOMS id type x y z\n");
  for (size_t i = 0; i < n; ++i)
    std::fprintf(_file, "%zu %d %g %g %g\n", i + 1, _para.type[i] + 1, s.x[3 * i], s.x[3 * i + 1], s.x[3 * i + 2]);
  std::fflush(_file);
}

CheckpointOutput::CheckpointOutput(const Para& para, int interval, const std::string& path)
    : _para(para), _interval(std::max(1, interval)), _path(path) {}

bool CheckpointOutput::ShouldOutput(const Executioner& ex) const {
  return ex.CurrentStep() >= 1 && (ex.CurrentStep() % _interval == 0 || ex.CurrentStep() == ex.NumStep());
}

void CheckpointOutput::Write(const StateSnapshot& s) {
  // written beside the previous checkpoint and renamed over it, so a crash never leaves half a file
  const Para& p = _para;
  const std::string tmp = _path + ".tmp";
  FILE* f = std::fopen(tmp.c_str(), "w");
  if (!f) throw std::runtime_error("cannot write " + tmp);
  const int nb = (int)p.bond_type.size(), na = (int)p.angle_type.size(), nd = (int)p.dihedral_type.size();
  std::fprintf(f, "LAMMPS data file: rbmd checkpoint at step %lld (atom_style %s)\n\n", (long long)s.step,
               p.atom_style.c_str());
  std::fprintf(f, "%d atoms\n%d atom types\n", p.n, p.n_types);
  if (nb) std::fprintf(f, "%d bonds\n%zu bond types\n", nb, p.bond_k.size());
  if (na) std::fprintf(f, "%d angles\n%zu angle types\n", na, p.angle_k.size());
  if (nd) std::fprintf(f, "%d dihedrals\n%zu dihedral types\n", nd, p.dihedral_k.size());
  const char* ax = "xyz";
  std::fprintf(f, "\n");
  for (int k = 0; k < 3; ++k) std::fprintf(f, "%.17g %.17g %clo %chi\n", s.box[k], s.box[3 + k], ax[k], ax[k]);
  std::vector<double> tmass(p.n_types, 1.0);
  for (int i = p.n - 1; i >= 0; --i) tmass[p.type[i]] = p.mass[i];
  std::fprintf(f, "\nMasses\n\n");
  for (int t = 0; t < p.n_types; ++t) std::fprintf(f, "%d %.17g\n", t + 1, tmass[t]);
  std::fprintf(f, "\nPair Coeffs # lj/cut\n\n");
  for (int t = 0; t < p.n_types; ++t) std::fprintf(f, "%d %.17g %.17g\n", t + 1, p.eps[t], p.sigma[t]);
  if (nb) {
    std::fprintf(f, "\nBond Coeffs # harmonic\n\n");
    for (size_t t = 0; t < p.bond_k.size(); ++t) std::fprintf(f, "%zu %.17g %.17g\n", t + 1, p.bond_k[t], p.bond_r0[t]);
  }
  if (na) {
    std::fprintf(f, "\nAngle Coeffs # harmonic\n\n");
    for (size_t t = 0; t < p.angle_k.size(); ++t)
      std::fprintf(f, "%zu %.17g %.17g\n", t + 1, p.angle_k[t], p.angle_theta0[t]);
  }
  if (nd) {
    std::fprintf(f, "\nDihedral Coeffs # harmonic\n\n");
    for (size_t t = 0; t < p.dihedral_k.size(); ++t)
      std::fprintf(f, "%zu %.17g %d %d\n", t + 1, p.dihedral_k[t], p.dihedral_sign[t], p.dihedral_multiplicity[t]);
  }
  std::fprintf(f, "\nAtoms # %s\n\n", p.atom_style.c_str());
  for (int i = 0; i < p.n; ++i) {
    const double* x = &s.x[3 * (size_t)i];
    const int* im = &s.image[3 * (size_t)i];
    const double q = p.charge.empty() ? 0.0 : p.charge[i];
    if (p.atom_style == "full")
      std::fprintf(f, "%d %d %d %.17g %.17g %.17g %.17g %d %d %d\n", i + 1, (p.molecule.empty() ? i : p.molecule[i]) + 1,
                   p.type[i] + 1, q, x[0], x[1], x[2], im[0], im[1], im[2]);
    else if (p.atom_style == "charge")
      std::fprintf(f, "%d %d %.17g %.17g %.17g %.17g %d %d %d\n", i + 1, p.type[i] + 1, q, x[0], x[1], x[2], im[0], im[1],
                   im[2]);
    else
      std::fprintf(f, "%d %d %.17g %.17g %.17g %d %d %d\n", i + 1, p.type[i] + 1, x[0], x[1], x[2], im[0], im[1], im[2]);
  }
  std::fprintf(f, "\nVelocities\n\n");
  for (int i = 0; i < p.n; ++i)
    std::fprintf(f, "%d %.17g %.17g %.17g\n", i + 1, s.v[3 * (size_t)i], s.v[3 * (size_t)i + 1], s.v[3 * (size_t)i + 2]);
  if (nb) {
    std::fprintf(f, "\nBonds\n\n");
    for (int b = 0; b < nb; ++b)
      std::fprintf(f, "%d %d %d %d\n", b + 1, p.bond_type[b] + 1, p.bond_atoms[2 * b] + 1, p.bond_atoms[2 * b + 1] + 1);
  }
  if (na) {
    std::fprintf(f, "\nAngles\n\n");
    for (int a = 0; a < na; ++a)
      std::fprintf(f, "%d %d %d %d %d\n", a + 1, p.angle_type[a] + 1, p.angle_atoms[3 * a] + 1, p.angle_atoms[3 * a + 1] + 1,
                   p.angle_atoms[3 * a + 2] + 1);
  }
  if (nd) {
    std::fprintf(f, "\nDihedrals\n\n");
    for (int d = 0; d < nd; ++d)
      std::fprintf(f, "%d %d %d %d %d %d\n", d + 1, p.dihedral_type[d] + 1, p.dihedral_atoms[4 * d] + 1,
                   p.dihedral_atoms[4 * d + 1] + 1, p.dihedral_atoms[4 * d + 2] + 1, p.dihedral_atoms[4 * d + 3] + 1);
  }
  const bool ok = std::fflush(f) == 0;
  std::fclose(f);
  if (!ok || std::rename(tmp.c_str(), _path.c_str()) != 0) throw std::runtime_error("cannot write " + _path);
}

CorrelationOutput::CorrelationOutput(bool vacf, int interval, int64_t start_step, int64_t end_step,
                                     const std::string& path)
    : _vacf(vacf), _interval(std::max(1, interval)), _start(start_step), _end(end_step) {
  _file = std::fopen(path.c_str(), "w");
  if (!_file) throw std::runtime_error("cannot write " + path);
}

CorrelationOutput::~CorrelationOutput() {
  if (_file) std::fclose(_file);
}

void CorrelationOutput::Execute(Executioner& ex) {
  // MSDOutput::Execute (MSDOutput.cpp:56-105), VACFOutput::Execute (VACFOutput.cpp:52-96)
  const int64_t step = ex.CurrentStep();
  if (step == _start) {
    ex.Run().ObserveReset(_vacf ? RBMD_OBS_VACF : RBMD_OBS_MSD);
    for (double& a : _ave) a = 0.0;
  }
  if (step >= _start && step <= _end) {
    if (_vacf) ex.Run().Observe(nullptr, _ave);
    else ex.Run().Observe(_ave, nullptr);
  }
  if (step == 0) std::fprintf(_file, _vacf ? "Step Time VACFx VACFy VACFz VACF_total\n"
                                           : "Step Time MSD_x MSD_y MSD_z MSD_total sqrt(MSD_total) \n");
  if (step < 1 || step % _interval != 0) return;
  std::fprintf(_file, "%lld %g %g %g %g %g", (long long)step, ex.CurrentTime(), _ave[0], _ave[1], _ave[2], _ave[3]);
  if (!_vacf) std::fprintf(_file, " %g", std::sqrt(_ave[3]));
  std::fprintf(_file, "\n");
  std::fflush(_file);
}

RDFOutput::RDFOutput(const Para& para, double radius, double dr, int64_t statistics_steps,
                     const std::vector<std::pair<int, int>>& pairs, const std::string& path)
    : _path(path), _radius(radius), _dr(dr), _stat(statistics_steps), _inbuild(para.init_way == "inbuild"),
      _pairs(pairs) {
  int32_t nb = 0;
  if (rbmd_rdf_bins(radius, dr, nullptr, 0, &nb) != RBMD_OK)
    throw std::runtime_error("rdf_out: radius and dr must be positive with radius / dr >= 1");
  _radii.resize(nb);
  rbmd_rdf_bins(radius, dr, _radii.data(), nb, &nb);
  if (_inbuild) {
    // ExecutionNVT::SetCenterTargetPositions (ExecutionNVT.cpp:293-322): first half against second
    const int h = para.n / 2;
    _centers.emplace_back();
    _targets.emplace_back();
    for (int i = 0; i < h; ++i) {
      _centers[0].push_back(i);
      _targets[0].push_back(h + i);
    }
  } else {
    if (pairs.empty()) throw std::runtime_error("rdf_out needs \"atoms_pair\": [[type, type], ...]");
    // atom ids of each type in id order (ModelFileInitCondition.cpp:786-806)
    for (const auto& pr : pairs) {
      for (int t : {pr.first, pr.second})
        if (t < 0 || t >= para.n_types)
          throw std::runtime_error("rdf_out: atoms_pair type " + std::to_string(t) + " out of range (types are 0-based)");
      _centers.emplace_back();
      _targets.emplace_back();
      for (int i = 0; i < para.n; ++i) {
        if (para.type[i] == pr.first) _centers.back().push_back(i);
        if (para.type[i] == pr.second) _targets.back().push_back(i);
      }
    }
  }
  _rdf.assign(_centers.size(), std::vector<double>(nb, 0.0));
}

void RDFOutput::Execute(Executioner& ex) {
  // RDFOutput::Execute / ComputeRDF (RDFOutput.cpp:107-262)
  const int64_t step = ex.CurrentStep();
  const int64_t lower = ex.NumStep() - _stat, upper = ex.NumStep() + 1;
  if (step >= lower && step < upper) {
    const float pif = 3.14159265358979323846f;  // vtkm::Pif() of the normalisation
    for (size_t p = 0; p < _centers.size(); ++p) {
      std::vector<int64_t> counts;
      const double volume = ex.Run().RdfCounts(_centers[p], _targets[p], _radius, _dr, !_inbuild, counts);
      const double nc = (double)_centers[p].size(), rho = (double)_targets[p].size() / volume;
      for (size_t b = 0; b < _radii.size(); ++b) {
        const double r = _radii[b];
        const double dr3 = std::pow(r + r * 0.01, 3), r3 = std::pow(r, 3);
        _rdf[p][b] += (double)counts[b] / (nc * rho * ((4 / 3.0) * pif * dr3 - ((4 / 3.0) * pif * r3)));
      }
    }
  }
  if (step != ex.NumStep() - 1) return;
  FILE* f = std::fopen(_path.c_str(), "w");
  if (!f) throw std::runtime_error("cannot write " + _path);
  std::fprintf(f, "Radius ");
  if (_inbuild) {
    std::fprintf(f, "RDF\n");
  } else {
    for (const auto& pr : _pairs) std::fprintf(f, "RDF:%d-%d ", pr.first, pr.second);
    std::fprintf(f, "\n");
  }
  const double div = (double)(upper - lower - 1);
  for (size_t b = 0; b < _radii.size(); ++b) {
    std::fprintf(f, "%g", _radii[b]);
    for (size_t p = 0; p < _rdf.size(); ++p) {
      const double v = _rdf[p][b] / div;
      if (std::isnan(v)) std::fprintf(f, " ");
      else std::fprintf(f, " %g", v);
    }
    std::fprintf(f, "\n");
  }
  std::fclose(f);
}

// --------------------------------------------------------------------------------- executioner
Executioner::Executioner(ExecutionMD& run, int64_t num_steps, double dt) : _run(run), _num_steps(num_steps), _dt(dt) {}

void Executioner::Init() { _run.Init(); }

void Executioner::PreStep() {
  for (auto& o : _outputs) o->Execute(*this);
}

void Executioner::TakeStep() {
  ++_current_step;
  _current_time += _dt;
  _run.Execute();
}

void Executioner::Execute() {
  // num_steps + 1 iterations with the outputs before each (Executioner.cpp:100-135)
  while (KeepGoing()) {
    PreStep();
    TakeStep();
  }
  for (auto& o : _outputs) o->Finish(*this);
}

// --------------------------------------------------------------------------------- application
Application::Application(int argc, char** argv) : _argv(argv, argv + argc) {}

void Application::HelpMessages() const {
  std::printf(
      "usage: rbmd [cuda] -j <input>.json [--device N] [--dump-system <out>.json]\n"
      "  Runs RBMD's per-step force-and-integrate path on a B200 (sm_100a).\n"
      "  cuda        device word of the reference CLI (the only backend this build carries)\n"
      "  -j FILE     input in RBMD's JSON schema (comments and trailing commas allowed)\n"
      "  --device N  CUDA ordinal (default 0)\n"
      "  --dump-system OUT  write the resolved system and parameters as JSON and stop (no GPU use)\n");
}

void Application::ParseCLI() {
  for (size_t k = 1; k < _argv.size(); ++k) {
    const std::string& a = _argv[k];
    if (a == "-h" || a == "--help") {
      _help = true;
    } else if (a == "-j" && k + 1 < _argv.size()) {
      _json_path = _argv[++k];
    } else if (a == "--device" && k + 1 < _argv.size()) {
      _device = std::atoi(_argv[++k].c_str());
    } else if (a == "--dump-system" && k + 1 < _argv.size()) {
      _dump_path = _argv[++k];
    } else if (a == "cuda" || a == "mpi" || a == "dcu") {
      _device_word = a;
    } else {
      throw std::runtime_error("unknown argument \"" + a + "\" (try --help)");
    }
  }
  if (_help) return;
  if (_json_path.size() < 5 || _json_path.compare(_json_path.size() - 5, 5, ".json") != 0)
    throw std::runtime_error("-j needs a .json input file");  // JsonParser.h:73-77
  if (_device_word == "mpi" || _device_word == "dcu")
    throw std::runtime_error("device \"" + _device_word + "\" is not built here; this library runs the cuda (sm_100a) path");
}

int Application::Run() {
  try {
    ParseCLI();
    if (_help) {
      HelpMessages();
      return 0;
    }
    CreateActions();
  } catch (const std::exception& e) {
    std::fprintf(stderr, "rbmd: %s\n", e.what());
    return 1;
  }
  return 0;
}

// The reference's G tables for the RBL near Coulomb force (res/json_files/Gnear_table_leq2_2.txt and
// Gnear_table_geq2_2.txt, compiled into model/ERFTable.h): rows "key r dr G dG", G stored at its
// key.  A row whose key is not that of its distance is refused; keys the files do not list keep
// the library's values.
static std::vector<float> read_near_tables(const std::vector<std::string>& paths) {
  std::vector<float> tab(RBMD_NEAR_TABLE_KEYS);
  rbmd_near_table_default(tab.data());
  for (const std::string& path : paths) {
    std::ifstream in(path);
    if (!in.is_open()) throw std::runtime_error("cannot open near-Coulomb table file " + path);
    long key;
    double r, dr, g, dg;
    int rows = 0;
    while (in >> key >> r >> dr >> g >> dg) {
      if (key < 0 || key >= RBMD_NEAR_TABLE_KEYS || rbmd_near_table_key((float)r) != key)
        throw std::runtime_error(path + ": the row of key " + std::to_string(key) + " holds r = " + std::to_string(r) +
                                 ", whose key differs");
      tab[key] = (float)g;
      ++rows;
    }
    if (!in.eof() || rows == 0) throw std::runtime_error(path + ": expected rows of five numbers (key r dr G dG)");
  }
  return tab;
}

void MDApplication::ReadHyperParameters(const Json& hp) {
  rbmd_params& P = _para.params;
  if (const Json* ff = hp.find("force_field")) {
    _ff_type = ff->string("type", "LJ/CUT");
    if (_ff_type == "LJ/CUT") P.force_field = RBMD_FF_LJ_CUT;
    else if (_ff_type == "LJ/CUT/COUL/LONG") P.force_field = RBMD_FF_LJ_CUT_COUL_LONG;
    else if (_ff_type == "CVFF") P.force_field = RBMD_FF_CVFF;
    else if (_ff_type == "EAM") P.force_field = RBMD_FF_EAM;
    else throw std::runtime_error("force_field type \"" + _ff_type + "\" is not supported");
    _potential_file = ff->string("potential_file", "");
    _dihedral_type = ff->string("dihedral_type", "");  // ForceField.cpp:49
    // setfl (eam/alloy) potentials: "potential_format": "setfl", or a file named *.alloy / *.setfl;
    // "elements": the file's element of each atom type (default: type t is element t)
    _potential_format = ff->string("potential_format", "");
    _eam_elements.clear();
    if (const Json* el = ff->find("elements")) {
      if (!el->is_array()) throw std::runtime_error("force_field.elements must be an array of element names");
      for (const Json& e : el->arr) {
        if (!e.is_string()) throw std::runtime_error("force_field.elements must be an array of element names");
        _eam_elements.push_back(e.str);
      }
    }
  }
  if (const Json* nb = hp.find("neighbor")) {
    const std::string t = nb->string("type", "RBL");
    if (t == "RBL") P.neighbor = RBMD_NEIGH_RBL;
    else if (t == "VERLETLIST" || t == "VERLET-LIST") P.neighbor = RBMD_NEIGH_VERLET;
    else throw std::runtime_error("neighbor type \"" + t + "\" is not supported");
    P.cut_off = nb->number("cut_off", P.cut_off);
    P.r_core = nb->number("r_core", P.r_core);
    P.neighbor_sample_num = (int32_t)nb->number("neighbor_sample_num", P.neighbor_sample_num);
  }
  P.coulomb = RBMD_COUL_NONE;
  if (const Json* cl = hp.find("coulomb")) {
    const std::string t = cl->string("type", "RBE");
    if (t == "RBE") P.coulomb = RBMD_COUL_RBE;
    else if (t == "EWALD") P.coulomb = RBMD_COUL_EWALD;
    else throw std::runtime_error("coulomb type \"" + t + "\" is not supported");
    P.coulomb_sample_num = (int32_t)cl->number("coulomb_sample_num", P.coulomb_sample_num);
    P.alpha = cl->number("alpha", P.alpha);
    // Coulomb::Execute (hyperparameters/Coulomb.cpp:40) reads kmax with GetVectorValue, which stops
    // the run when the value is not an array (parser/Configuration.h:142-163), and the k loops index
    // it per dimension: a scalar or a list of other than three entries is refused here too.
    if (const Json* km = cl->find("kmax")) {
      if (!km->is_array()) throw std::runtime_error("coulomb.kmax must be an array of three integers, e.g. [2, 2, 2]");
      const std::vector<double> v = cl->numbers("kmax");
      if (v.size() != 3) throw std::runtime_error("coulomb.kmax must hold three integers (one per dimension)");
      for (int k = 0; k < 3; ++k) P.kmax[k] = (int32_t)v[k];
    }
    // "near_table": true takes the reference's alpha = 0.1 lookup for the RBL near Coulomb force
    // (its only form there, RunWorklet.cpp:1046-1047, 1171-1172) with the library's table; a list of
    // the reference's two Gnear_table files takes their values (this key is not the reference's:
    // its RBL runs always use the table, the library defaults to the analytic form)
    if (const Json* nt = cl->find("near_table")) {
      std::vector<std::string> files;
      if (nt->is_bool()) {
        P.near_table = nt->b ? RBMD_NEAR_TABLE : RBMD_NEAR_ANALYTIC;
      } else if (nt->is_array()) {
        P.near_table = RBMD_NEAR_TABLE;
        for (const Json& e : nt->arr) {
          if (!e.is_string()) throw std::runtime_error("coulomb.near_table: file names must be strings");
          files.push_back(e.str);
        }
        if (files.empty()) throw std::runtime_error("coulomb.near_table: an empty list of files");
      } else {
        throw std::runtime_error("coulomb.near_table must be true, false or a list of Gnear_table files");
      }
      _para.near_table = files.empty() ? std::vector<float>() : read_near_tables(files);
    }
  }
  P.fix_shake = RBMD_SHAKE_NULL;
  if (const Json* ex = hp.find("extend")) {
    if (ex->has("fix_shake")) P.fix_shake = ex->boolean("fix_shake", false) ? RBMD_SHAKE_TRUE : RBMD_SHAKE_FALSE;
    const std::vector<double> sb = ex->numbers("special_bonds");
    if (!sb.empty()) {  // MDApplication.cpp:158-163: a non-empty list switches the special lists on
      _special_bonds = true;
      for (int k = 0; k < 3 && k < (int)sb.size(); ++k) _special_w[k] = (double)(int)sb[k];  // read as ints
      for (int k = 0; k < 3; ++k) P.special_bonds[k] = _special_w[k];
    }
  }
}

void MDApplication::ReadExecution(const Json& ex) {
  rbmd_params& P = _para.params;
  const std::string ens = ex.string("ensemble", "NVT");
  if (ens == "NVT") P.ensemble = RBMD_ENS_NVT;
  else if (ens == "NVE") P.ensemble = RBMD_ENS_NVE;
  else if (ens == "NPT") P.ensemble = RBMD_ENS_NPT;
  else throw std::runtime_error("ensemble \"" + ens + "\" is not supported");
  const std::vector<double> t = ex.numbers("temperature");
  for (int k = 0; k < 3 && k < (int)t.size(); ++k) P.temperature[k] = t[k];
  // "pressure": [P_start, P_stop, P_damp, bulk modulus] (ExecutionMD.cpp:152, ExecutionNPT.cpp:953);
  // the reference reads the fourth entry unconditionally, here it is optional (default 10)
  const std::vector<double> pr = ex.numbers("pressure");
  for (int k = 0; k < 3 && k < (int)pr.size(); ++k) P.pressure[k] = pr[k];
  if (pr.size() >= 4) P.bulk_modulus = pr[3];
  const std::string tc = ex.string("temp_ctrl_type", "NOSE_HOOVER");
  if (P.ensemble == RBMD_ENS_NVE) P.temp_ctrl = RBMD_TC_NONE;
  else if (tc == "NOSE_HOOVER") P.temp_ctrl = RBMD_TC_NOSE_HOOVER;
  else if (tc == "BERENDSEN") P.temp_ctrl = RBMD_TC_BERENDSEN;
  else if (tc == "TEMP_RESCALE") P.temp_ctrl = RBMD_TC_RESCALE;
  else throw std::runtime_error("temp_ctrl_type \"" + tc + "\" is not supported");
  if (P.ensemble == RBMD_ENS_NPT) {
    // ExecutionNPT::Solve (ExecutionNPT.cpp:90-141) controls the pressure for temp_ctrl_type /
    // press_ctrl_type BERENDSEN / BERENDSEN and NOSE_HOOVER / NOSE_HOOVER only
    const std::string pc = ex.string("press_ctrl_type", tc);
    if (pc == "BERENDSEN") P.press_ctrl = RBMD_PC_BERENDSEN;
    else if (pc == "NOSE_HOOVER") P.press_ctrl = RBMD_PC_NOSE_HOOVER;
    else throw std::runtime_error("press_ctrl_type \"" + pc + "\" is not supported (BERENDSEN, NOSE_HOOVER)");
    const bool ok = (P.press_ctrl == RBMD_PC_BERENDSEN && P.temp_ctrl == RBMD_TC_BERENDSEN) ||
                    (P.press_ctrl == RBMD_PC_NOSE_HOOVER && P.temp_ctrl == RBMD_TC_NOSE_HOOVER);
    if (!ok)
      throw std::runtime_error("ensemble NPT needs temp_ctrl_type and press_ctrl_type both BERENDSEN or both "
                               "NOSE_HOOVER (the reference controls the pressure in no other pairing)");
  }
  P.timestep = ex.number("timestep", P.timestep);
  P.num_steps = (int64_t)ex.number("num_steps", (double)P.num_steps);
  // keys this library adds (absent from reference files): seed, precision, rbl_mode, autotune
  P.seed = (uint64_t)ex.number("seed", (double)P.seed);
  _para.autotune = ex.boolean("autotune", false);
  const std::string prec = ex.string("precision", "FP64");
  if (prec == "FP64") P.precision = RBMD_PREC_FP64;
  else if (prec == "MIXED") P.precision = RBMD_PREC_MIXED;
  else throw std::runtime_error("precision must be FP64 or MIXED");
  const std::string rm = ex.string("rbl_mode", "STRIDE");
  if (rm == "STRIDE") P.rbl_mode = RBMD_RBL_STRIDE;
  else if (rm == "PHILOX") P.rbl_mode = RBMD_RBL_PHILOX;
  else throw std::runtime_error("rbl_mode must be STRIDE or PHILOX");
}

void MDApplication::CreateActions() {
  _cfg = parse_json_file(_json_path);
  _base_dir = dir_of(_json_path);
  rbmd_params_default(&_para.params);
  if (const Json* hp = _cfg.find("hyper_parameters")) ReadHyperParameters(*hp);
  if (const Json* ex = _cfg.find("execution")) ReadExecution(*ex);
  const Json* ic = _cfg.find("init_configuration");
  if (!ic) throw std::runtime_error("input has no init_configuration");
  std::unique_ptr<InitCondition> init;
  if (const Json* rd = ic->find("read_data")) {
    _para.unit = rd->string("unit", "LJ");
    init.reset(new ModelFileInitCondition(*rd, _base_dir));
  } else if (const Json* ib = ic->find("inbuild")) {
    _para.unit = ib->string("unit", "LJ");
    init.reset(new MeshFreeCondition(*ib));
  } else {
    throw std::runtime_error("init_configuration needs read_data or inbuild");
  }
  _para.params.units = units_of(_para.unit);
  init->Execute(_para);
  if (_para.init_way == "inbuild" && _para.params.coulomb != RBMD_COUL_NONE) {
    // ExecutionMD::InitialCondition (ExecutionMD.cpp:157-168): -1 for the first half, +1 after
    for (int i = 0; i < _para.n; ++i) _para.charge[i] = (i < _para.n / 2) ? -1.0 : 1.0;
  }
  if (_special_bonds) special_lists(_para.n, _para.bond_atoms, _special_w, _para.sp_off, _para.sp_ids, _para.sp_w);
  // dihedral forces: CVFF with special_bonds (PARA_DIHEDRALS_FORCE) and a Dihedrals section
  // (PARA_FILE_DIHEDRALS), style "Harmonic" (ExecutionNVT.cpp:223-228, 585-588); the reference has
  // no other style (its DihedralsForce returns nothing otherwise)
  const bool dihedrals = _para.params.force_field == RBMD_FF_CVFF && _special_bonds && _para.file_dihedrals;
  if (dihedrals && _dihedral_type != "Harmonic")
    throw std::runtime_error("the data file has Dihedrals: force_field.dihedral_type must be \"Harmonic\" (got \"" +
                             _dihedral_type + "\")");
  if (!dihedrals) {
    _para.dihedral_atoms.clear();
    _para.dihedral_type.clear();
    _para.dihedral_k.clear();
    _para.dihedral_sign.clear();
    _para.dihedral_multiplicity.clear();
  }
  if (_para.params.force_field == RBMD_FF_EAM) {
    if (_potential_file.empty()) throw std::runtime_error("EAM needs force_field.potential_file");
    std::string path = _potential_file;
    if (!exists(path) && exists(_base_dir + "/" + path)) path = _base_dir + "/" + path;
    auto ends = [&](const char* suf) {
      const size_t k = std::strlen(suf);
      return _potential_file.size() >= k && _potential_file.compare(_potential_file.size() - k, k, suf) == 0;
    };
    const bool setfl = _potential_format == "setfl" || (_potential_format.empty() && (ends(".alloy") || ends(".setfl")));
    if (!_potential_format.empty() && _potential_format != "setfl" && _potential_format != "funcfl")
      throw std::runtime_error("potential_format must be \"funcfl\" or \"setfl\"");
    if (setfl) {
      ReadSetfl(path);
    } else {
    rbmd_eam_file f;
    std::memset(&f, 0, sizeof(f));
    if (rbmd_eam_read_funcfl(path.c_str(), &f, nullptr, nullptr, nullptr) != RBMD_OK)
      throw std::runtime_error("cannot read EAM potential " + path);
    std::vector<double> frho(f.nrho), zr(f.nr), rhor(f.nr);
    if (rbmd_eam_read_funcfl(path.c_str(), &f, frho.data(), zr.data(), rhor.data()) != RBMD_OK)
      throw std::runtime_error("cannot read EAM potential " + path);
    f.frho = frho.data();
    f.zr = zr.data();
    f.rhor = rhor.data();
    int32_t nrho = 0, nr = 0;
    if (rbmd_eam_spline_sizes(&f, &nrho, &nr) != RBMD_OK) throw std::runtime_error("bad EAM table sizes in " + path);
    _para.frho_spline.assign(7 * ((size_t)nrho + 1), 0.0);  // rows 1..nrho (row 0 unused)
    _para.rhor_spline.assign(7 * ((size_t)nr + 1), 0.0);
    _para.z2r_spline.assign(7 * ((size_t)nr + 1), 0.0);
    if (rbmd_eam_build_splines(&f, _para.frho_spline.data(), _para.rhor_spline.data(), _para.z2r_spline.data(),
                               &_para.eam_nrho, &_para.eam_drho, &_para.eam_nr, &_para.eam_dr, &_para.eam_rhomax) != RBMD_OK)
      throw std::runtime_error("cannot build EAM splines from " + path);
    _para.eam_cut = f.cut_off;
    }
  }
  if (const Json* outs = _cfg.find("outputs")) {
    if (const Json* th = outs->find("thermo_out")) _thermo_interval = (int)th->number("interval", 1);
    if (const Json* tr = outs->find("trajectory_out")) _traj_interval = (int)tr->number("interval", 1);
    if (const Json* cp = outs->find("checkpoint_out")) {
      _checkpoint_interval = (int)cp->number("interval", 1000);
      _checkpoint_file = cp->string("file", _checkpoint_file);
    }
    // msd_out / vacf_out: interval (default 1), start_step and end_step (required);
    // rdf_out: radius, dr, statistics_rdf_steps, atoms_pair (read_data) (MDApplication.cpp:221-235)
    auto need = [](const Json* o, const char* out, const char* key) {
      if (!o->find(key) || !o->find(key)->is_number())
        throw std::runtime_error(std::string(out) + " needs a number \"" + key + "\"");
      return o->find(key)->num;
    };
    for (const char* name : {"msd_out", "vacf_out"}) {
      const Json* o = outs->find(name);
      if (!o) continue;
      Correlation& c = name[0] == 'm' ? _msd : _vacf;
      c.on = true;
      c.interval = (int)o->number("interval", 1);
      c.start = (int64_t)need(o, name, "start_step");
      c.end = (int64_t)need(o, name, "end_step");
    }
    if (const Json* o = outs->find("rdf_out")) {
      _rdf.on = true;
      _rdf.radius = need(o, "rdf_out", "radius");
      _rdf.dr = need(o, "rdf_out", "dr");
      _rdf.statistics_steps = (int64_t)need(o, "rdf_out", "statistics_rdf_steps");
      if (const Json* ap = o->find("atoms_pair")) {
        if (!ap->is_array()) throw std::runtime_error("rdf_out: atoms_pair must be an array of [type, type]");
        for (const Json& e : ap->arr) {
          if (!e.is_array() || e.arr.size() != 2 || !e.arr[0].is_number() || !e.arr[1].is_number())
            throw std::runtime_error("rdf_out: atoms_pair must be an array of [type, type]");
          _rdf.pairs.emplace_back((int)e.arr[0].num, (int)e.arr[1].num);
        }
      }
      if (_para.init_way != "inbuild") {
        if (_rdf.pairs.empty()) throw std::runtime_error("rdf_out needs \"atoms_pair\": [[type, type], ...]");
        for (const auto& pr : _rdf.pairs)
          for (int t : {pr.first, pr.second})
            if (t < 0 || t >= _para.n_types)
              throw std::runtime_error("rdf_out: atoms_pair type " + std::to_string(t) +
                                       " out of range (types are 0-based)");
      }
      if (rbmd_rdf_bins(_rdf.radius, _rdf.dr, nullptr, 0, nullptr) != RBMD_OK)
        throw std::runtime_error("rdf_out: radius and dr must be positive with radius / dr >= 1");
    }
  }
}

void MDApplication::ReadSetfl(const std::string& path) {
  rbmd_eam_setfl f;
  std::memset(&f, 0, sizeof(f));
  if (rbmd_eam_read_setfl(path.c_str(), &f, nullptr, nullptr, nullptr, nullptr, nullptr) != RBMD_OK)
    throw std::runtime_error("cannot read setfl potential " + path);
  const int ne = f.n_elements;
  std::vector<char> names(16 * (size_t)ne);
  std::vector<double> mass(ne), frho((size_t)ne * f.nrho), rhor((size_t)ne * f.nr), z2r((size_t)ne * (ne + 1) / 2 * f.nr);
  if (rbmd_eam_read_setfl(path.c_str(), &f, names.data(), mass.data(), frho.data(), rhor.data(), z2r.data()) != RBMD_OK)
    throw std::runtime_error("cannot read setfl potential " + path);
  std::vector<int32_t> te(_para.n_types);
  for (int t = 0; t < _para.n_types; ++t) {
    if (_eam_elements.empty()) {
      if (t >= ne)
        throw std::runtime_error(path + " has " + std::to_string(ne) + " elements for " + std::to_string(_para.n_types) +
                                 " atom types (map them with force_field.elements)");
      te[t] = t;
    } else {
      if ((int)_eam_elements.size() != _para.n_types)
        throw std::runtime_error("force_field.elements needs one element name per atom type");
      te[t] = -1;
      for (int e = 0; e < ne; ++e)
        if (_eam_elements[t] == std::string(names.data() + 16 * e)) te[t] = e;
      if (te[t] < 0) throw std::runtime_error("element " + _eam_elements[t] + " is not in " + path);
    }
  }
  const size_t nt = _para.n_types;
  _para.frho_spline.assign(7 * ((size_t)f.nrho + 1) * nt, 0.0);
  _para.rhor_spline.assign(7 * ((size_t)f.nr + 1) * nt, 0.0);
  _para.z2r_spline.assign(7 * ((size_t)f.nr + 1) * nt * (nt + 1) / 2, 0.0);
  if (rbmd_eam_build_setfl_splines(&f, frho.data(), rhor.data(), z2r.data(), te.data(), (int32_t)nt,
                                   _para.frho_spline.data(), _para.rhor_spline.data(), _para.z2r_spline.data(),
                                   &_para.eam_rhomax) != RBMD_OK)
    throw std::runtime_error("cannot build EAM splines from " + path);
  _para.eam_nrho = f.nrho;
  _para.eam_nr = f.nr;
  _para.eam_drho = f.drho;
  _para.eam_dr = f.dr;
  _para.eam_cut = f.cut_off;
  _para.eam_per_type = 1;
}

void MDApplication::DumpSystem(const std::string& path) const {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) throw std::runtime_error("cannot write " + path);
  auto darr = [&](const char* name, const std::vector<double>& v) {
    std::fprintf(f, "\"%s\": [", name);
    for (size_t k = 0; k < v.size(); ++k) std::fprintf(f, "%s%.17g", k ? "," : "", v[k]);
    std::fprintf(f, "],\n");
  };
  auto iarr = [&](const char* name, const std::vector<int>& v) {
    std::fprintf(f, "\"%s\": [", name);
    for (size_t k = 0; k < v.size(); ++k) std::fprintf(f, "%s%d", k ? "," : "", v[k]);
    std::fprintf(f, "],\n");
  };
  const rbmd_params& P = _para.params;
  std::fprintf(f, "{\n\"n_atoms\": %d, \"n_types\": %d, \"init_way\": \"%s\",\n", _para.n, _para.n_types,
               _para.init_way.c_str());
  std::fprintf(f, "\"box_lo\": [%.17g,%.17g,%.17g], \"box_hi\": [%.17g,%.17g,%.17g],\n", _para.lo[0], _para.lo[1],
               _para.lo[2], _para.hi[0], _para.hi[1], _para.hi[2]);
  std::fprintf(f,
               "\"params\": {\"force_field\": %d, \"neighbor\": %d, \"coulomb\": %d, \"ensemble\": %d, "
               "\"temp_ctrl\": %d, \"units\": %d, \"precision\": %d, \"rbl_mode\": %d, \"fix_shake\": %d, "
               "\"init_inbuild\": %d, \"neighbor_sample_num\": %d, \"cut_off\": %.17g, \"r_core\": %.17g, "
               "\"coulomb_sample_num\": %d, \"kmax\": [%d,%d,%d], \"alpha\": %.17g, \"temperature\": [%.17g,%.17g,%.17g], "
               "\"timestep\": %.17g, \"num_steps\": %lld, \"special_bonds\": [%.17g,%.17g,%.17g], \"seed\": %llu, "
               "\"pressure\": [%.17g,%.17g,%.17g], \"bulk_modulus\": %.17g, \"press_ctrl\": %d, \"near_table\": %d},\n",
               P.force_field, P.neighbor, P.coulomb, P.ensemble, P.temp_ctrl, P.units, P.precision, P.rbl_mode,
               P.fix_shake, P.init_inbuild, P.neighbor_sample_num, P.cut_off, P.r_core, P.coulomb_sample_num,
               P.kmax[0], P.kmax[1], P.kmax[2], P.alpha, P.temperature[0], P.temperature[1], P.temperature[2],
               P.timestep, (long long)P.num_steps, P.special_bonds[0], P.special_bonds[1], P.special_bonds[2],
               (unsigned long long)P.seed, P.pressure[0], P.pressure[1], P.pressure[2], P.bulk_modulus,
               P.press_ctrl, P.near_table);
  darr("position", _para.position);
  darr("velocity", _para.velocity);
  darr("charge", _para.charge);
  darr("mass", _para.mass);
  darr("epsilon", _para.eps);
  darr("sigma", _para.sigma);
  iarr("type", _para.type);
  iarr("molecule", _para.molecule);
  iarr("bond_atoms", _para.bond_atoms);
  iarr("bond_type", _para.bond_type);
  darr("bond_k", _para.bond_k);
  darr("bond_r0", _para.bond_r0);
  iarr("angle_atoms", _para.angle_atoms);
  iarr("angle_type", _para.angle_type);
  darr("angle_k", _para.angle_k);
  darr("angle_theta0", _para.angle_theta0);
  iarr("dihedral_atoms", _para.dihedral_atoms);
  iarr("dihedral_type", _para.dihedral_type);
  darr("dihedral_k", _para.dihedral_k);
  iarr("dihedral_sign", _para.dihedral_sign);
  iarr("dihedral_multiplicity", _para.dihedral_multiplicity);
  iarr("special_offsets", _para.sp_off);
  iarr("special_ids", _para.sp_ids);
  darr("special_weights", _para.sp_w);
  std::fprintf(f, "\"eam\": {\"nrho\": %d, \"nr\": %d, \"drho\": %.17g, \"dr\": %.17g, \"rhomax\": %.17g, \"cut\": %.17g, "
               "\"per_type\": %d},\n",
               _para.eam_nrho, _para.eam_nr, _para.eam_drho, _para.eam_dr, _para.eam_rhomax, _para.eam_cut,
               _para.eam_per_type);
  darr("eam_frho_spline", _para.frho_spline);
  darr("eam_rhor_spline", _para.rhor_spline);
  darr("eam_z2r_spline", _para.z2r_spline);
  darr("near_table_values", std::vector<double>(_para.near_table.begin(), _para.near_table.end()));
  std::fprintf(f, "\"outputs\": {\"thermo_interval\": %d, \"trajectory_interval\": %d, \"checkpoint_interval\": %d, "
               "\"checkpoint_file\": \"%s\"", _thermo_interval, _traj_interval, _checkpoint_interval,
               _checkpoint_file.c_str());
  for (const Correlation* c : {&_msd, &_vacf})
    if (c->on)
      std::fprintf(f, ", \"%s\": {\"interval\": %d, \"start_step\": %lld, \"end_step\": %lld}",
                   c == &_msd ? "msd" : "vacf", c->interval, (long long)c->start, (long long)c->end);
  if (_rdf.on) {
    std::fprintf(f, ", \"rdf\": {\"radius\": %.17g, \"dr\": %.17g, \"statistics_rdf_steps\": %lld, \"atoms_pair\": [",
                 _rdf.radius, _rdf.dr, (long long)_rdf.statistics_steps);
    for (size_t k = 0; k < _rdf.pairs.size(); ++k)
      std::fprintf(f, "%s[%d,%d]", k ? "," : "", _rdf.pairs[k].first, _rdf.pairs[k].second);
    std::fprintf(f, "]}");
  }
  std::fprintf(f, "}\n}\n");
  std::fclose(f);
}

int MDApplication::Run() {
  try {
    ParseCLI();
    if (_help) {
      HelpMessages();
      return 0;
    }
    CreateActions();
    if (!_dump_path.empty()) {
      DumpSystem(_dump_path);
      return 0;
    }
    ExecutionNVT run(_para, _device);
    Executioner ex(run, _para.params.num_steps, _para.params.timestep);
    if (_thermo_interval > 0)
      ex.AddOutput(std::unique_ptr<Output>(new ThermoOutput(_thermo_interval, "energy.rbmd", "temperature.rbmd", true)));
    if (_traj_interval > 0) ex.AddOutput(std::unique_ptr<Output>(new TrajectoryOutput(_para, _traj_interval, "rbmd.trj")));
    if (_checkpoint_interval > 0)
      ex.AddOutput(std::unique_ptr<Output>(new CheckpointOutput(_para, _checkpoint_interval, _checkpoint_file)));
    if (_rdf.on)
      ex.AddOutput(std::unique_ptr<Output>(
          new RDFOutput(_para, _rdf.radius, _rdf.dr, _rdf.statistics_steps, _rdf.pairs, "rdf.rbmd")));
    if (_msd.on)
      ex.AddOutput(std::unique_ptr<Output>(new CorrelationOutput(false, _msd.interval, _msd.start, _msd.end, "msd.rbmd")));
    if (_vacf.on)
      ex.AddOutput(
          std::unique_ptr<Output>(new CorrelationOutput(true, _vacf.interval, _vacf.start, _vacf.end, "vacf.rbmd")));
    const auto t0 = std::chrono::steady_clock::now();
    ex.Init();
    ex.Execute();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("rbmd: %lld steps of %d atoms in %.3f s (%.4g atom-steps/s)\n", (long long)ex.CurrentStep(), _para.n,
                secs, (double)_para.n * (double)ex.CurrentStep() / secs);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "rbmd: %s\n", e.what());
    return 1;
  }
  return 0;
}

}  // namespace rbmd_host
