// app.hpp -- the `rbmd` host: RBMD's Application -> Executioner -> Execution(MD/NVT) shape driving
// the sm_100a library through its C ABI (include/rbmd_gpu.h).
//
//   reference                                   here
//   Application (application/Application.h:52)  Application: CLI, device set-up, actions, Run
//   MDApplication (MDApplication.cpp)           MDApplication: JSON sections -> Para, outputs
//   InitCondition + ModelFileInitCondition /    InitCondition, ModelFileInitCondition (read_data),
//     MeshFreeCondition (InitCondition/)          MeshFreeCondition (inbuild)
//   Executioner (executioner/Executioner.h:38)  Executioner: num_steps + 1 iterations, outputs
//                                                 before each step
//   Execution / ExecutionMD / ExecutionNVT      Execution, ExecutionMD, ExecutionNVT: rbmd_init
//     (run/)                                      once, rbmd_step per step
//   ThermoOutput, TrajectoryOutput (output/)    ThermoOutput (energy.rbmd), TrajectoryOutput
#pragma once

#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "data_file.hpp"
#include "json.hpp"
#include "rbmd_gpu.h"

namespace rbmd_host {

// Everything the C ABI needs for one system: parameters and the arrays the descriptor points into.
struct Para {
  rbmd_params params{};
  std::string init_way;  // "read_data" or "inbuild"
  std::string atom_style = "charge";  // of the data file read (inbuild: charge)
  std::string unit = "LJ";
  bool autotune = false;  // execution.autotune: time the pair layouts before the first step
  int n = 0, n_types = 0;
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  std::vector<double> position, velocity, charge, mass, eps, sigma;
  std::vector<int> type, molecule;
  std::vector<int> bond_atoms, bond_type, angle_atoms, angle_type;
  std::vector<double> bond_k, bond_r0, angle_k, angle_theta0;
  std::vector<int> sp_off, sp_ids;
  std::vector<double> sp_w;
  // harmonic dihedrals (evaluated when special_bonds, a Dihedrals section and dihedral_type
  // "Harmonic" are all given)
  std::vector<int> dihedral_atoms, dihedral_type, dihedral_sign, dihedral_multiplicity;
  std::vector<double> dihedral_k;
  bool file_dihedrals = false;
  // EAM
  int eam_nrho = 0, eam_nr = 0;
  double eam_drho = 0, eam_dr = 0, eam_rhomax = 0, eam_cut = 0;
  int eam_per_type = 0;  // setfl: tables per atom type
  std::vector<double> frho_spline, rhor_spline, z2r_spline;
  // coulomb.near_table given as the reference's two Gnear_table files: G by key (empty: the library's table)
  std::vector<float> near_table;

  rbmd_system_desc desc() const;  // pointers into this object
};

// One rbmd_snapshot_begin in flight; heap-allocated so its buffers never move before the wait.
struct StateSnapshot {
  std::vector<double> x, v;
  std::vector<int32_t> image;
  double box[6] = {0, 0, 0, 0, 0, 0};
  int64_t step = 0;
  int64_t ticket = 0;
};

class InitCondition {
 public:
  virtual ~InitCondition() = default;
  virtual void Execute(Para& para) = 0;
};

// read_data (InitCondition/ModelFileInitCondition.cpp)
class ModelFileInitCondition : public InitCondition {
 public:
  ModelFileInitCondition(const Json& cfg, const std::string& base_dir);
  void Execute(Para& para) override;

 private:
  std::string _file, _atom_style, _velocity_type;
};

// inbuild (InitCondition/MeshFreeCondition.cpp): one atom per lattice cell centre
class MeshFreeCondition : public InitCondition {
 public:
  explicit MeshFreeCondition(const Json& cfg);
  void Execute(Para& para) override;

 private:
  int _dims[3] = {1, 1, 1};
  double _range[3][2] = {{0, 1}, {0, 1}, {0, 1}};
  std::string _velocity_type;
};

class Execution {
 public:
  virtual ~Execution() = default;
  virtual void Init() = 0;
  virtual void Execute() = 0;
  virtual void SetParameters() {}
};

// Owns the library context and the system (run/ExecutionMD.cpp).
class ExecutionMD : public Execution {
 public:
  ExecutionMD(Para& para, int device);
  ~ExecutionMD() override;
  void Init() override;
  rbmd_thermo Thermo();
  void State(std::vector<double>& x, std::vector<double>& v, std::vector<int>& image);
  // trajectory observables (rbmd_observe_reset / rbmd_observe / rbmd_rdf_counts)
  int64_t SnapshotBegin(StateSnapshot& s);
  bool SnapshotDone(int64_t ticket);
  void SnapshotWait(int64_t ticket);
  void ObserveReset(int which);
  void Observe(double* msd, double* vacf);
  double RdfCounts(const std::vector<int>& centers, const std::vector<int>& targets, double radius, double dr,
                   bool exclude_same_molecule, std::vector<int64_t>& counts);  // returns the box volume

 protected:
  void check(int rc, const char* what);
  Para& _para;
  int _device;
  rbmd_ctx* _ctx = nullptr;
  int32_t _sys = -1;
};

// NVT / NVE velocity Verlet with the configured thermostat (run/ExecutionNVT.cpp)
class ExecutionNVT : public ExecutionMD {
 public:
  using ExecutionMD::ExecutionMD;
  void Execute() override;
};

class Executioner;

class Output {
 public:
  virtual ~Output() = default;
  virtual void Execute(Executioner& ex) = 0;
  virtual void Finish(Executioner&) {}  // after the last step: complete pending work
};

// Outputs written from asynchronous snapshots: the state is queued for copy at the output step
// and the file written once the copy has landed (at a later output call or at Finish), so the
// steps in between are not held up.  At most kInFlight snapshots are pending.
class SnapshotOutput : public Output {
 public:
  void Execute(Executioner& ex) override;
  void Finish(Executioner& ex) override;

 protected:
  virtual bool ShouldOutput(const Executioner& ex) const = 0;
  virtual void Write(const StateSnapshot& s) = 0;

 private:
  static constexpr size_t kInFlight = 4;
  std::vector<std::unique_ptr<StateSnapshot>> _pending;
};

// energy.rbmd columns of output/ThermoOutput.cpp:223-291 plus temperature and pressure
class ThermoOutput : public Output {
 public:
  ThermoOutput(int interval, const std::string& path, const std::string& temp_path, bool console);
  ~ThermoOutput() override;
  void Execute(Executioner& ex) override;

 private:
  int _interval;
  FILE* _file = nullptr;
  FILE* _temp = nullptr;  // temperature.rbmd (output/TempOutput.cpp:85-103): Step Temperature Pressure
  bool _console;
};

// rbmd.trj (output/TrajectoryOutput.cpp:33-85): a LAMMPS dump block ("ITEM: TIMESTEP" ... "ITEM:
// ATOMS id type x y z") every `interval` steps from step 1.
class TrajectoryOutput : public SnapshotOutput {
 public:
  TrajectoryOutput(const Para& para, int interval, const std::string& path);
  ~TrajectoryOutput() override;

 protected:
  bool ShouldOutput(const Executioner& ex) const override;
  void Write(const StateSnapshot& s) override;

 private:
  const Para& _para;
  int _interval;
  FILE* _file = nullptr;
};

// A LAMMPS data file of the current state (positions with image flags, velocities, the topology
// and coefficients the run was read with) every `interval` steps, replacing the previous one: the
// checkpoint a read_data input restarts from.  The reference writes none.
class CheckpointOutput : public SnapshotOutput {
 public:
  CheckpointOutput(const Para& para, int interval, const std::string& path);

 protected:
  bool ShouldOutput(const Executioner& ex) const override;
  void Write(const StateSnapshot& s) override;

 private:
  const Para& _para;
  int _interval;
  std::string _path;
};

// msd.rbmd / vacf.rbmd (output/MSDOutput.cpp, output/VACFOutput.cpp): the reference configuration
// is taken at start_step, the atom average recomputed every step of [start_step, end_step], and a
// line "Step Time x y z total" (MSD: and sqrt(total)) written every `interval` steps from step 1,
// holding the last average computed.
class CorrelationOutput : public Output {
 public:
  CorrelationOutput(bool vacf, int interval, int64_t start_step, int64_t end_step, const std::string& path);
  ~CorrelationOutput() override;
  void Execute(Executioner& ex) override;

 private:
  bool _vacf;
  int _interval;
  int64_t _start, _end;
  double _ave[4] = {0, 0, 0, 0};
  FILE* _file = nullptr;
};

// rdf.rbmd (output/RDFOutput.cpp): pair counts of the last statistics_rdf_steps steps, normalised
// per snapshot and averaged, written once at step num_steps - 1.  Pairs of atom types (0-based)
// with same-molecule pairs skipped (read_data), or the first half of the atoms against the second
// (inbuild).
class RDFOutput : public Output {
 public:
  RDFOutput(const Para& para, double radius, double dr, int64_t statistics_steps,
            const std::vector<std::pair<int, int>>& pairs, const std::string& path);
  void Execute(Executioner& ex) override;

 private:
  std::string _path;
  double _radius, _dr;
  int64_t _stat;
  bool _inbuild;
  std::vector<std::pair<int, int>> _pairs;
  std::vector<std::vector<int>> _centers, _targets;
  std::vector<double> _radii;
  std::vector<std::vector<double>> _rdf;
};

class Executioner {
 public:
  Executioner(ExecutionMD& run, int64_t num_steps, double dt);
  void AddOutput(std::unique_ptr<Output> o) { _outputs.push_back(std::move(o)); }
  void Init();
  void Execute();
  int64_t CurrentStep() const { return _current_step; }
  int64_t NumStep() const { return _num_steps; }
  double CurrentTime() const { return _current_time; }
  ExecutionMD& Run() { return _run; }

 private:
  void PreStep();
  void TakeStep();
  bool KeepGoing() const { return _current_step <= _num_steps; }
  ExecutionMD& _run;
  std::vector<std::unique_ptr<Output>> _outputs;
  int64_t _num_steps;
  int64_t _current_step = 0;
  double _dt, _current_time = 0.0;
};

class Application {
 public:
  Application(int argc, char** argv);
  virtual ~Application() = default;
  // returns the process exit status; errors are reported on stderr, never by exit()
  virtual int Run();

 protected:
  virtual void ParseCLI();
  virtual void CreateActions() = 0;
  void HelpMessages() const;
  std::vector<std::string> _argv;
  std::string _device_word;  // cuda | mpi | dcu | "" (serial)
  std::string _json_path;
  std::string _dump_path;    // --dump-system: write the resolved system and stop (no device use)
  int _device = 0;
  bool _help = false;
};

// JSON-driven molecular dynamics (application/MDApplication.cpp)
class MDApplication : public Application {
 public:
  using Application::Application;
  int Run() override;

 protected:
  void CreateActions() override;

 private:
  void ReadHyperParameters(const Json& hp);
  void ReadExecution(const Json& ex);
  void DumpSystem(const std::string& path) const;
  void ReadSetfl(const std::string& path);
  Json _cfg;
  Para _para;
  int _thermo_interval = 0, _traj_interval = 0, _checkpoint_interval = 0;
  std::string _checkpoint_file = "rbmd_checkpoint.data";
  struct Correlation {
    bool on = false;
    int interval = 1;
    int64_t start = 0, end = 0;
  } _msd, _vacf;
  struct Rdf {
    bool on = false;
    double radius = 0, dr = 0;
    int64_t statistics_steps = 0;
    std::vector<std::pair<int, int>> pairs;
  } _rdf;
  bool _special_bonds = false;
  double _special_w[3] = {0, 0, 0};
  std::string _ff_type, _potential_file, _base_dir, _dihedral_type, _potential_format;
  std::vector<std::string> _eam_elements;
};

}  // namespace rbmd_host
