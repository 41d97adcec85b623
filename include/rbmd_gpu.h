/*
 * rbmd_gpu.h -- C ABI of the B200 (sm_100a) per-step force-and-integrate path of RBMD.
 *
 * This header is the drop-in boundary.  It replaces the VTK-m execution objects and worklet
 * launches that RBMD's NVT execution class drives (framework/run/ExecutionNVT.cpp:76-235), and the
 * four Cont* and Exec* device objects:
 *   - point locator      framework/locator/ContPointLocator.cxx:70-115, ExecPointLocator.h:38-382
 *   - force function     framework/forceFunction/ContForceFunction.cpp:30-45, ExecForceFunction.h
 *   - static erfc table  framework/staticTable/ContStaticTable.cpp:30-44 (analytic erfc by default;
 *                        the table lookup on request, rbmd_params.near_table)
 *   - topology           framework/topology/ContTopology.cpp:31-42, ExecTopology.h:35-97
 * and the worklet library framework/run/worklet/RunWorklet.h:40-502 plus the water constraint and
 * bonded worklets of framework/run/worklet/MolecularWorklet.h.
 *
 * Plain C: pointers, sizes and status codes; no C++ or torch types cross this boundary.  Every
 * function returns an int status (RBMD_OK == 0).  rbmd_last_error() gives the text of the last
 * failure on a context.  The library never calls exit() (the reference's console::Error does,
 * framework/Logging.h:44-51).
 *
 * Threading: one context per host thread, or external locking.  rbmd_step() only enqueues work on
 * the context's CUDA stream; results are valid after rbmd_sync() (or any rbmd_get_* call, which
 * synchronises first).
 */
#ifndef RBMD_GPU_H
#define RBMD_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RBMD_ABI_VERSION 6

/* ---------------------------------------------------------------- status codes */
enum rbmd_status {
  RBMD_OK = 0,
  RBMD_ERR_ARG = 1,          /* bad argument (null pointer, size, unknown enum) */
  RBMD_ERR_OOM = 2,          /* device allocation failed */
  RBMD_ERR_NUMERIC = 3,      /* non-finite force / SHAKE or RATTLE singular / overflow */
  RBMD_ERR_TIMEOUT = 4,      /* bounded device wait or serving wait expired */
  RBMD_ERR_CUDA = 5,         /* CUDA runtime error */
  RBMD_ERR_STATE = 6,        /* call out of order (unknown system id, serving not started ...) */
  RBMD_ERR_BUDGET = 7,       /* request exceeds the HBM budget */
  RBMD_ERR_UNSUPPORTED = 8,  /* configuration not implemented */
  RBMD_ERR_IO = 9            /* file could not be read or parsed */
};

/* ---------------------------------------------------------------- enums (JSON strings in comments) */
enum rbmd_force_field {      /* hyper_parameters.force_field.type */
  RBMD_FF_LJ_CUT = 0,        /* "LJ/CUT" */
  RBMD_FF_LJ_CUT_COUL_LONG = 1, /* "LJ/CUT/COUL/LONG" */
  RBMD_FF_CVFF = 2,          /* "CVFF" (LJ + Coulomb + harmonic bond/angle + special bonds) */
  RBMD_FF_EAM = 3            /* "EAM" (funcfl) */
};
enum rbmd_neighbor {         /* hyper_parameters.neighbor.type */
  RBMD_NEIGH_RBL = 0,        /* "RBL" */
  RBMD_NEIGH_VERLET = 1      /* "VERLETLIST" */
};
enum rbmd_coulomb {          /* hyper_parameters.coulomb.type (absent = NONE) */
  RBMD_COUL_NONE = 0,
  RBMD_COUL_RBE = 1,         /* "RBE" */
  RBMD_COUL_EWALD = 2        /* "EWALD" */
};
enum rbmd_temp_ctrl {        /* execution.temp_ctrl_type */
  RBMD_TC_NOSE_HOOVER = 0,   /* "NOSE_HOOVER" */
  RBMD_TC_BERENDSEN = 1,     /* "BERENDSEN" */
  RBMD_TC_RESCALE = 2,       /* "TEMP_RESCALE" */
  RBMD_TC_NONE = 3           /* plain velocity Verlet (NVE) */
};
enum rbmd_units {            /* init_configuration.*.unit */
  RBMD_UNITS_LJ = 0, RBMD_UNITS_REAL = 1, RBMD_UNITS_METAL = 2
};
enum rbmd_precision {
  RBMD_PREC_FP64 = 0,        /* every kernel in FP64 */
  RBMD_PREC_MIXED = 1        /* pair + RBE arithmetic FP32; positions, rho(k) sums (of FP32
                                partials over 32 atoms), reductions, SHAKE, thermostat and
                                barostat FP64 */
};
enum rbmd_rbl_mode {
  RBMD_RBL_STRIDE = 0,       /* every pice-th shell atom in cell traversal order (reference) */
  RBMD_RBL_PHILOX = 1        /* same stride, start offset drawn per (seed, step, atom) */
};
enum rbmd_random_mode {
  RBMD_RANDOM_PHILOX = 0,    /* counter-based Philox4x32-10 keyed by (seed, step, index) */
  RBMD_RANDOM_TEST = 1       /* every uniform is 0.5 (reference velocity_type "TEST") */
};
enum rbmd_shake_flag {       /* hyper_parameters.extend.fix_shake */
  RBMD_SHAKE_NULL = -1,      /* key absent ("null") */
  RBMD_SHAKE_FALSE = 0,
  RBMD_SHAKE_TRUE = 1
};
enum rbmd_ensemble {
  RBMD_ENS_NVT = 0, RBMD_ENS_NVE = 1, RBMD_ENS_NPT = 2
};
enum rbmd_press_ctrl {
  RBMD_PC_BERENDSEN = 0,     /* "BERENDSEN": isotropic volume rescale at the end of the step
                                (ExecutionNPT::fix_press_berendsen); needs temp_ctrl BERENDSEN */
  RBMD_PC_NOSE_HOOVER = 1    /* "NOSE_HOOVER": isotropic MTK barostat with its own chain
                                (ExecutionNPT::InitialIntegrate / FinalIntegrate); needs temp_ctrl
                                NOSE_HOOVER */
};

/* Real-space Coulomb kernel G(r) of the RBL near forces (ComputeNearEnergyForceERF[_box],
 * ExecForceFunction.h:581-596, 665-680: F = -qi qj G(r) r_ij / r). */
enum rbmd_near_coulomb {
  RBMD_NEAR_ANALYTIC = 0,    /* G(r) = erfc(sqrt(a) r)/r^2 + 2 sqrt(a) exp(-a r^2)/(sqrt(pi) r) at the
                                system's alpha (the form of ExecForceFunction::Gnear, :682-689) */
  RBMD_NEAR_TABLE = 1        /* the reference's lookup (ExecStaticTable::Extract / TableGnearValue,
                                staticTable/ExecStaticTable.h:96-135): G of alpha = 0.1 whatever the
                                system's alpha, read without interpolation at the 11-bit key of
                                the FP32 distance (rbmd_near_table_key); from
                                rbmd_system_desc.near_table_values, else rbmd_near_table_default.
                                RBL near forces only (Verlet forces and every energy stay analytic,
                                as in the reference); needs cut_off <= 12, where the reference's
                                table ends; pairs closer than 0.1 (before its first entry, where
                                the reference reads outside the table) take the entry of r = 0.1 */
};

/* ---------------------------------------------------------------- run parameters */
/* Mirrors the JSON keys that framework/hyperparameters/{ForceField,Neighbor,Coulomb,Extend}.cpp
 * and ExecutionMD::SetParameters (framework/run/ExecutionMD.cpp:144-153) copy into Para. */
typedef struct rbmd_params {
  int32_t force_field;          /* enum rbmd_force_field */
  int32_t neighbor;             /* enum rbmd_neighbor */
  int32_t coulomb;              /* enum rbmd_coulomb */
  int32_t ensemble;             /* enum rbmd_ensemble */
  int32_t temp_ctrl;            /* enum rbmd_temp_ctrl */
  int32_t units;                /* enum rbmd_units */
  int32_t precision;            /* enum rbmd_precision */
  int32_t rbl_mode;             /* enum rbmd_rbl_mode */
  int32_t random_mode;          /* enum rbmd_random_mode */
  int32_t fix_shake;            /* enum rbmd_shake_flag */
  int32_t init_inbuild;         /* 1: system built by the inbuild lattice (temperature without kB) */
  int32_t neighbor_sample_num;  /* RBL shell sample target */
  double cut_off;               /* r_c */
  double r_core;                /* r_s (VERLETLIST: ignored, r_s = r_c) */
  int32_t coulomb_sample_num;   /* RBE P */
  int32_t kmax[3];              /* Ewald k range (energy in RBE mode, force in EWALD mode) */
  double alpha;                 /* Ewald splitting, reference convention: erfc(sqrt(alpha) r) */
  double temperature[3];        /* T_start, T_stop, T_damp */
  double pressure[3];           /* P_start, P_stop, P_damp (NPT; ExecutionNPT.cpp:90-141 controls the
                                   pressure for temp_ctrl / press_ctrl BERENDSEN / BERENDSEN and
                                   NOSE_HOOVER / NOSE_HOOVER, the two pairs accepted here) */
  int32_t press_ctrl;           /* enum rbmd_press_ctrl */
  int32_t near_table;           /* enum rbmd_near_coulomb (default RBMD_NEAR_ANALYTIC) */
  double timestep;
  int64_t num_steps;            /* length of the run, used for temperature ramps */
  double special_bonds[3];      /* 1-2, 1-3, 1-4 LJ weights */
  uint64_t seed;                /* Philox key */
  double bulk_modulus;          /* NPT Berendsen: pressure[3] of the reference's 4-entry "pressure" */
} rbmd_params;

/* Fill *p with the reference defaults (LJ units, RBL, NH, FP64, stride picks, seed 1). */
void rbmd_params_default(rbmd_params* p);

/* ---------------------------------------------------------------- system description */
/* Host arrays; the library copies them at rbmd_system_add and the caller keeps ownership.
 * Layout follows the Para fields of framework/FieldName.h:30-153: position Vec3[N], velocity
 * Vec3[N], mass/charge Real[N], pts_type/molecule_id Id[N], epsilon/sigma Real[ntypes],
 * position_flag Id3[N], special_ids/weights/offsets CSR, bond_atom_id Id[2nb], angle_atom_id
 * Id[3na], {frho,rhor,z2r}_spline Vec7[n+1]. */
typedef struct rbmd_system_desc {
  int32_t n_atoms;
  int32_t n_types;
  double box_lo[3];
  double box_hi[3];
  const double* position;       /* [3*n_atoms] x0 y0 z0 x1 ... */
  const double* velocity;       /* [3*n_atoms] or NULL (zero) */
  const double* charge;         /* [n_atoms] or NULL (zero) */
  const double* mass;           /* [n_atoms] per-atom mass */
  const int32_t* type;          /* [n_atoms] 0-based type index */
  const int32_t* molecule;      /* [n_atoms] or NULL (atom i is molecule i) */
  const int32_t* image;         /* [3*n_atoms] or NULL (zero image flags) */
  const double* epsilon;        /* [n_types] LJ epsilon per type */
  const double* sigma;          /* [n_types] LJ sigma per type */
  /* harmonic bonds (CVFF): E = k (r - r0)^2 */
  int32_t n_bonds;
  int32_t n_bond_types;
  const int32_t* bond_atoms;    /* [2*n_bonds] */
  const int32_t* bond_type;     /* [n_bonds] 0-based */
  const double* bond_k;         /* [n_bond_types] */
  const double* bond_r0;        /* [n_bond_types] */
  /* harmonic angles (CVFF): E = k (theta - theta0)^2; also the SHAKE triples (H, O, H) */
  int32_t n_angles;
  int32_t n_angle_types;
  const int32_t* angle_atoms;   /* [3*n_angles] */
  const int32_t* angle_type;    /* [n_angles] */
  const double* angle_k;        /* [n_angle_types] */
  const double* angle_theta0;   /* [n_angle_types] degrees */
  /* special-bond LJ weights, CSR over atoms (ModelFileInitCondition.cpp:843-923) */
  const int32_t* special_offsets; /* [n_atoms+1] or NULL */
  const int32_t* special_ids;
  const double* special_weights;
  /* EAM splines (ExecutionNVT.cpp:899-1104): Vec7 coefficient rows, index 0 unused */
  int32_t eam_nrho;
  int32_t eam_nr;
  double eam_drho;
  double eam_dr;
  double eam_rhomax;
  double eam_cut;
  const double* eam_frho_spline; /* [(eam_nrho+1)*7] */
  const double* eam_rhor_spline; /* [(eam_nr+1)*7] */
  const double* eam_z2r_spline;  /* [(eam_nr+1)*7] */
  /* harmonic dihedrals (CVFF, ComputeDihedralHarmonicWorklet, MolecularWorklet.h:669-973):
   * E = K [1 + d cos(n phi)]; the reference evaluates them when special_bonds are given, the data
   * file has a Dihedrals section and force_field.dihedral_type is "Harmonic" (ExecutionNVT.cpp:
   * 223-228, 585-658); leave n_dihedrals 0 otherwise */
  int32_t n_dihedrals;
  int32_t n_dihedral_types;
  const int32_t* dihedral_atoms;        /* [4*n_dihedrals] i j k l */
  const int32_t* dihedral_type;         /* [n_dihedrals] 0-based */
  const double* dihedral_k;             /* [n_dihedral_types] K */
  const int32_t* dihedral_sign;         /* [n_dihedral_types] d: 1 (cos shift +1), else -1 */
  const int32_t* dihedral_multiplicity; /* [n_dihedral_types] n >= 0 */
  /* EAM tables per atom type (setfl, LAMMPS eam/alloy; the reference reads funcfl only).  0: one
   * table of each kind for every type (funcfl).  1: eam_frho_spline holds n_types embedding tables
   * of (eam_nrho+1)*7 and eam_rhor_spline n_types density tables of (eam_nr+1)*7 (the density an
   * atom of that type contributes to its neighbours), one after the other in type order, and
   * eam_z2r_spline n_types (n_types+1)/2 pair tables of (eam_nr+1)*7 (r phi), the pair of types
   * i >= j at index i (i+1)/2 + j. */
  int32_t eam_per_type;
  int32_t pad_eam;
  /* RBMD_NEAR_TABLE: G by key, [RBMD_NEAR_TABLE_KEYS] (the reference's tables
   * res/json_files/Gnear_table_{leq,geq}2_2.txt, column 4 at the key of column 1, fill keys
   * 921-2047 and 0-639); NULL: rbmd_near_table_default.  Keys the reference's table does not
   * cover should hold G at the key's lower edge, as the default table does. */
  const float* near_table_values;
} rbmd_system_desc;

/* ---------------------------------------------------------------- results */
typedef struct rbmd_thermo {
  int64_t step;                 /* Executioner current step of the system */
  double temperature;           /* PARA_TEMPT after the last ComputeTempe */
  double tempT_sum;             /* sum m v^2 mvv2e */
  double kinetic_energy;        /* tempT_sum / N / 2 (ThermoOutput.cpp:180) */
  double e_lj;                  /* per-atom averages, as ThermoOutput reports them */
  double e_coul_near;
  double e_coul_far;            /* Ewald k-space (kmax) + self energy */
  double e_bond;
  double e_angle;
  double e_eam;
  double potential_energy;
  double total_energy;
  double pressure;
  double virial[6];             /* xx yy zz xy xz yz */
  double nhc_eta[3];
  double nhc_eta_dot[4];
  double volume;
  double box_lo[3];
  double box_hi[3];
  int32_t status;               /* device-side error word of the system (0 = ok), bits below */
  int32_t pad0;
  double e_dihedral;            /* per-dihedral average (PARA_DIHEDRAL_ENERGY), in potential_energy */
} rbmd_thermo;

/* Bits of rbmd_thermo.status, sticky until the system is removed. */
enum rbmd_status_bit {
  RBMD_STATUS_SHAKE_OVERFLOW = 1,    /* SHAKE multipliers became NaN or exceeded 1e20 */
  RBMD_STATUS_SHAKE_SINGULAR = 2,    /* SHAKE 3x3 system with |det| < 1e-4 */
  RBMD_STATUS_SHAKE_NO_CONVERGE = 4, /* SHAKE iteration hit its 5000-step limit */
  RBMD_STATUS_RATTLE_SINGULAR = 8,   /* RATTLE 3x3 system with |det| < 1e-4 */
  RBMD_STATUS_NON_FINITE = 16,       /* a force component was Inf or NaN */
  RBMD_STATUS_RBE_SLOTS = 32,        /* Metropolis chain ran out of proposal slots */
  RBMD_STATUS_BOX_RANGE = 64         /* NPT: the box left the range its cell tables were sized for
                                        (0.8 to 1.25 of the initial edge); the box stays put */
};

typedef struct rbmd_device_cfg {
  int32_t device;               /* CUDA ordinal */
  int32_t batched;              /* 1: one segment-indexed launch per kernel over all systems of a
                                   rbmd_step call; 0: one launch per system (the plain path) */
  int32_t use_graphs;           /* 1: capture the step of a fixed system set as a CUDA graph */
  int32_t autotune;             /* 1: rbmd_init / rbmd_step run rbmd_autotune on systems that have not
                                   been tuned yet (before their first force evaluation or graph) */
  int64_t hbm_budget_bytes;     /* admission budget for the serving loop (0 = free memory) */
} rbmd_device_cfg;

typedef struct rbmd_ctx rbmd_ctx;

/* ---------------------------------------------------------------- context and systems */
int rbmd_abi_version(void);
int rbmd_ctx_create(const rbmd_device_cfg* cfg, rbmd_ctx** out);
int rbmd_ctx_destroy(rbmd_ctx* ctx);
const char* rbmd_last_error(const rbmd_ctx* ctx);

/* Bytes of device memory a system with this description needs (admission by HBM budget). */
int rbmd_system_bytes(const rbmd_system_desc* desc, const rbmd_params* params, int64_t* bytes);

/* Upload a system (Para fields + JSON parameters; the InitCondition + SetForceFunction/SetTopology
 * of ExecutionMD::Init, framework/run/ExecutionMD.cpp:117-134). */
int rbmd_system_add(rbmd_ctx* ctx, const rbmd_system_desc* desc, const rbmd_params* params,
                    int32_t* sys_id);
int rbmd_system_remove(rbmd_ctx* ctx, int32_t sys_id);

/* ExecutionNVT::Init's tail (framework/run/ExecutionNVT.cpp:60-74,139-187): thermostat set-up
 * (ComputeTempe, ComputeTempTarget, NH chain masses) and the first ComputeForce. */
int rbmd_init(rbmd_ctx* ctx, const int32_t* sys_ids, int32_t n);

/* nsteps x Executioner::TakeStep -> ExecutionMD::Execute (PreSolve, Solve, PostSolve;
 * framework/executioner/Executioner.cpp:112-117, framework/run/ExecutionNVT.cpp:76-135) for every
 * listed system.  Enqueue only. */
int rbmd_step(rbmd_ctx* ctx, const int32_t* sys_ids, int32_t n, int32_t nsteps);
int rbmd_sync(rbmd_ctx* ctx);

/* ComputeForce at the current positions without integrating (ExecutionNVT::ComputeForce,
 * framework/run/ExecutionNVT.cpp:189-235); uses the system's current step for random draws. */
int rbmd_compute_forces(rbmd_ctx* ctx, const int32_t* sys_ids, int32_t n);

int rbmd_get_forces(rbmd_ctx* ctx, int32_t sys_id, double* force /* [3N] */);
int rbmd_get_state(rbmd_ctx* ctx, int32_t sys_id, double* position, double* velocity,
                   int32_t* image);
int rbmd_set_state(rbmd_ctx* ctx, int32_t sys_id, const double* position, const double* velocity,
                   const int32_t* image);
/* Sets the step counter (Executioner::_current_step) that keys the system's random draws and
 * temperature / pressure ramps: a restart from a checkpoint written at that step, or a second
 * system evaluated at the same draws (no reference counterpart). */
int rbmd_set_step(rbmd_ctx* ctx, int32_t sys_id, int64_t step);
/* Thermo quantities; energies are evaluated at the current positions on request (the reference
 * recomputes them every step for ThermoOutput, framework/output/ThermoOutput.cpp:144-186). */
int rbmd_get_thermo(rbmd_ctx* ctx, int32_t sys_id, rbmd_thermo* out);

/* Cell list of the last binning (ContPointLocator::Build, framework/locator/ContPointLocator.cxx:70-92):
 * dims[3]; per atom the reference flat cell id; atom ids sorted by cell (ascending id within a
 * cell); per cell [lower, upper).  Any output pointer may be NULL. */
int rbmd_get_cells(rbmd_ctx* ctx, int32_t sys_id, int32_t* dims, int32_t* cell_of_atom,
                   int32_t* sorted_ids, int32_t* cell_lower, int32_t* cell_upper);

/* Materialise the RBL lists of the current positions and step (ComputeRBLNeighboursOnceWorklet,
 * framework/run/worklet/RunWorklet.cpp:906-980): per atom n_core, n_shell and the picked ids in
 * traversal order, core first, in rows of `cap` ids.  Returns RBMD_ERR_ARG if a row exceeds cap. */
int rbmd_get_rbl_lists(rbmd_ctx* ctx, int32_t sys_id, int32_t cap, int32_t* n_core,
                       int32_t* n_shell, int32_t* ids);

/* The same lists as rbmd_get_rbl_lists, for callers that must not allocate device memory while
 * systems run.  No counterpart in the reference (it keeps its lists in VTK-m arrays).  Who cannot
 * allocate: an observer or monitoring thread beside running steps (cudaFree waits for the whole
 * device, so it would stall every stream on the GPU), and a serving host whose HBM budget has
 * already been handed to admitted systems (an allocation there can fail mid-run).
 * Calls no cudaMalloc, cudaFree or allocating library routine.  Every temporary lives in one
 * file-scope device array of 2^21 ints (8 MiB) that each GPU loading the library holds until the
 * process exits.  The first call on a device looks up that array's address; make it before any
 * stream capture on the device.  Limit: n_atoms * (2 cap + 2) plus small work tables must fit in
 * the 2^21 ints, else RBMD_ERR_ARG is returned and nothing runs.  Rows: core ids, shell ids, then
 * -1 up to cap.  The array keeps the last call's contents, and calls that overlap on the GPU (two
 * host threads, on one context or on different contexts of one device) race on it: serialise
 * them. */
int rbmd_get_rbl_lists_static(rbmd_ctx* ctx, int32_t sys_id, int32_t cap, int32_t* n_core,
                              int32_t* n_shell, int32_t* ids);

/* RBE k samples of the last force evaluation (integer m vectors, [3P]) and rho(k) ([2P]: Re, Im). */
int rbmd_get_kspace(rbmd_ctx* ctx, int32_t sys_id, int32_t* m, double* rhok);

/* Per-system parameters derived at upload: rs_num, rc_num, pice_num, num_cycles, dims[3],
 * S (RBE normalisation), volume. */
typedef struct rbmd_derived {
  int32_t rs_num, rc_num, pice_num, num_cycles;
  int32_t dims[3];
  int32_t n_cells;
  double rho_system;
  double S_rbe;
  double volume;
  double cell_width[3];
} rbmd_derived;
int rbmd_get_derived(rbmd_ctx* ctx, int32_t sys_id, rbmd_derived* out);

/* ---------------------------------------------------------------- trajectory observables */
enum rbmd_observable { RBMD_OBS_MSD = 1, RBMD_OBS_VACF = 2 };
/* Take the current positions and image counters (which & RBMD_OBS_MSD) and / or velocities
 * (which & RBMD_OBS_VACF) as the reference configuration of rbmd_observe (MSDOutput::Execute at
 * start_step, framework/output/MSDOutput.cpp:58-66; VACFOutput::Execute,
 * framework/output/VACFOutput.cpp:54-57).  The reference zeroes the image counters at that point;
 * here they are left alone and their values at the reset subtracted. */
int rbmd_observe_reset(rbmd_ctx* ctx, int32_t sys_id, int32_t which);
/* Atom averages against the reference configuration (MSDOutput::ExecuteMSD,
 * framework/output/MSDOutput.cpp:116-134; VACFOutput::ExecuteMSD,
 * framework/output/VACFOutput.cpp:108-118): msd[4] = (dx^2, dy^2, dz^2, |d|^2) of the unwrapped
 * displacement x + (image - image0) L - x0 (L the current box), vacf[4] = (v0x vx, v0y vy, v0z vz,
 * v0.v).  Either pointer may be NULL; RBMD_ERR_STATE when a requested average has no reference
 * configuration yet. */
int rbmd_observe(rbmd_ctx* ctx, int32_t sys_id, double* msd, double* vacf);
/* RDF radii (RDFOutput::RDFOutput, framework/output/RDFOutput.cpp:42-53): n = (int)(radius / dr)
 * bins at dr, 2 dr, ... accumulated by repeated addition.  radii may be NULL (count only); at most
 * cap values are written.  RBMD_ERR_ARG unless radius > 0, dr > 0 and radius / dr >= 1. */
int rbmd_rdf_bins(double radius, double dr, double* radii, int32_t cap, int32_t* n_bins);

/* ---------------------------------------------------------------- near-Coulomb table */
#define RBMD_NEAR_TABLE_KEYS 2048
/* The key of a distance: bits 15-25 of its FP32 pattern (the exponent's low three bits and the
 * mantissa's top eight; ExecStaticTable::Extract, MASK 2^26 - 2^15 and MANTISSA_BITS 8,
 * ExecStaticTable.h:38-39, 125-133).  Distances in [0.1, 2) give keys 921-2047, [2, 12) 0-639. */
int32_t rbmd_near_table_key(float r);
/* The library's table, [RBMD_NEAR_TABLE_KEYS] floats: G of alpha = 0.1 in FP64, rounded to FP32,
 * at the points the reference tabulates -- for each key the first r of the walks
 * r = 0.1 + 0.0001 m (r < 2) and r = 2 + 0.001 m (r < 12) that has that key (column 2 of its
 * table files) -- and at the key's lower edge for the keys those walks do not reach.  The
 * reference's files print G to six digits; below r = 8 they equal these values to that
 * precision, above it they drift from the FP64 G, to about 1% at r = 12 (as 1 - erf taken in
 * single precision would). */
int rbmd_near_table_default(float* out);
/* RDF pair counts of the current configuration (RDFOutput::ComputeRDF,
 * framework/output/RDFOutput.cpp:181-262; ComputeRDFWorklet,
 * framework/output/worklet/OutPutWorklet.cpp:230-310 and :578-640): counts[b] (n_bins of
 * rbmd_rdf_bins) = number of (center, target, periodic image) triples with
 * r_b < distance < r_b + 0.01 r_b, skipping pairs of one molecule when exclude_same_molecule.
 * centers / targets are atom ids.  *volume (may be NULL) receives the box volume the counts were
 * taken in; the reference's RDF value of one snapshot is
 * counts[b] / (n_centers * (n_targets / volume) * 4/3 pi ((1.01 r_b)^3 - r_b^3)). */
int rbmd_rdf_counts(rbmd_ctx* ctx, int32_t sys_id, const int32_t* centers, int32_t n_centers,
                    const int32_t* targets, int32_t n_targets, double radius, double dr,
                    int32_t exclude_same_molecule, int64_t* counts, double* volume);

/* ---------------------------------------------------------------- asynchronous state snapshots */
/* Outputs that must not stall the step pipeline (trajectory, checkpoints, progress of a served
 * system).  rbmd_snapshot_begin packs the state of one system as of the work queued so far on the
 * device and copies it to pinned host staging on a second stream while later steps run; it
 * returns at once with a ticket.  rbmd_snapshot_wait blocks until that copy has landed, then fills
 * the destinations given at begin (each may be NULL): x, v [3 n_atoms], image [3 n_atoms],
 * box [6] (lo x y z, hi x y z: the current box, NPT included) and step.  The destinations must
 * stay valid until the wait returns RBMD_OK.  timeout_s < 0 waits without limit; on
 * RBMD_ERR_TIMEOUT the ticket stays pending.  rbmd_snapshot_poll sets *done (1: a wait will not
 * block) without blocking.  One waiter per ticket.  No counterpart in the reference (its outputs
 * read the fields synchronously, framework/output/TrajectoryOutput.cpp:45-85). */
int rbmd_snapshot_begin(rbmd_ctx* ctx, int32_t sys_id, double* x, double* v, int32_t* image,
                        double* box, int64_t* step, int64_t* ticket);
int rbmd_snapshot_poll(rbmd_ctx* ctx, int64_t ticket, int32_t* done);
int rbmd_snapshot_wait(rbmd_ctx* ctx, int64_t ticket, double timeout_s);

/* ---------------------------------------------------------------- EAM input helpers (host only) */
/* funcfl file contents after the header lines (ExecutionNVT::ReadPotentialFile,
 * framework/run/ExecutionNVT.cpp:899-931). */
typedef struct rbmd_eam_file {
  int32_t nrho, nr;
  double drho, dr, cut_off;
  const double* frho;   /* [nrho] */
  const double* zr;     /* [nr] */
  const double* rhor;   /* [nr] */
} rbmd_eam_file;
/* nrho and nr of the resampled tables; the spline arrays of rbmd_eam_build_splines then need
 * (nrho + 1) * 7 and (nr + 1) * 7 doubles (row 0 unused). */
int rbmd_eam_spline_sizes(const rbmd_eam_file* in, int32_t* nrho_out, int32_t* nr_out);
/* file2array + array2spline (framework/run/ExecutionNVT.cpp:933-1079): fills the three Vec7
 * tables (caller allocates (nrho+1)*7, (nr+1)*7, (nr+1)*7 doubles) and rhomax. */
int rbmd_eam_build_splines(const rbmd_eam_file* in, double* frho_spline, double* rhor_spline,
                           double* z2r_spline, int32_t* nrho_out, double* drho_out,
                           int32_t* nr_out, double* dr_out, double* rhomax_out);
/* setfl file (LAMMPS eam/alloy format; the reference ships potentials/CuNi.eam.alloy but reads
 * funcfl only): three comment lines; "n_elements name1 name2 ..."; "nrho drho nr dr cutoff"; per
 * element a line "Z mass a lattice", F(rho) [nrho] and rho(r) [nr]; then r phi(r) [nr] for every
 * element pair i >= j in the order (0,0), (1,0), (1,1), (2,0) ... */
typedef struct rbmd_eam_setfl {
  int32_t n_elements, nrho, nr, pad0;
  double drho, dr, cut_off;
} rbmd_eam_setfl;
/* First call with every array NULL fills *out (sizes); the second fills names [n_elements * 16]
 * chars (NUL-padded), mass [n_elements], frho [n_elements * nrho], rhor [n_elements * nr] and
 * z2r [n_elements (n_elements + 1) / 2 * nr]. */
int rbmd_eam_read_setfl(const char* path, rbmd_eam_setfl* out, char* names, double* mass, double* frho,
                        double* rhor, double* z2r);
/* Per-type spline tables of a setfl potential (eam_per_type = 1): type t takes element
 * type_element[t].  The tables are splined on the file's own grid (nrho, drho, nr, dr; rhomax =
 * (nrho - 1) drho) with the 7-coefficient rows of rbmd_eam_build_splines, as LAMMPS eam/alloy
 * builds them (no resampling).  frho_spline needs n_types (nrho + 1) 7 doubles, rhor_spline
 * n_types (nr + 1) 7, z2r_spline n_types (n_types + 1) / 2 (nr + 1) 7. */
int rbmd_eam_build_setfl_splines(const rbmd_eam_setfl* in, const double* frho, const double* rhor,
                                 const double* z2r, const int32_t* type_element, int32_t n_types,
                                 double* frho_spline, double* rhor_spline, double* z2r_spline,
                                 double* rhomax_out);

/* Read a funcfl file: first call with arrays NULL to get nrho/nr, second call to fill. */
int rbmd_eam_read_funcfl(const char* path, rbmd_eam_file* out_sizes, double* frho, double* zr,
                         double* rhor);

/* ---------------------------------------------------------------- serving (continuous batching) */
typedef struct rbmd_serve_cfg {
  int64_t hbm_budget_bytes;     /* 0: use the context's budget */
  int32_t max_systems;          /* slots (0 = unlimited) */
  int32_t steps_per_round;      /* MD steps run per batched launch sequence between admissions */
  int32_t use_graphs;
  int32_t round_atoms;          /* atoms stepped per round: 0 = every active request each round;
                                   > 0 = the requests with the least remaining work (remaining
                                   steps x atoms, then arrival order) until their atoms reach this
                                   (at least one request), so small requests finish in few rounds */
} rbmd_serve_cfg;

typedef struct rbmd_request_stats {
  double t_submit;              /* seconds, host monotonic clock */
  double t_admit;
  double t_done;
  int64_t atom_steps;
  int32_t n_atoms;
  int32_t status;
} rbmd_request_stats;

enum rbmd_request_state {
  RBMD_REQ_QUEUED = 0, RBMD_REQ_RUNNING = 1, RBMD_REQ_DONE = 2, RBMD_REQ_FAILED = 3
};

int rbmd_serve_start(rbmd_ctx* ctx, const rbmd_serve_cfg* cfg);
/* Submit an independent MD system that should run nsteps; returns immediately. */
int rbmd_serve_submit(rbmd_ctx* ctx, const rbmd_system_desc* desc, const rbmd_params* params,
                      int32_t nsteps, int64_t* request_id);
int rbmd_serve_poll(rbmd_ctx* ctx, int64_t request_id, int32_t* state);
int rbmd_serve_wait(rbmd_ctx* ctx, int64_t request_id, double timeout_s);
/* Final state and statistics; position/velocity [3N] may be NULL. Frees the request. */
int rbmd_serve_result(rbmd_ctx* ctx, int64_t request_id, double* position, double* velocity,
                      rbmd_thermo* thermo, rbmd_request_stats* stats);
int rbmd_serve_stop(rbmd_ctx* ctx);

/* ---------------------------------------------------------------- diagnostics */
/* Number of kernel launches this context enqueued (graph replays count their nodes). */
int rbmd_launch_count(rbmd_ctx* ctx, int64_t* launches);
/* Average device time per launch of the named kernel family since the last reset, measured with
 * CUDA events on the context stream when profiling is on ("pair", "rho", "final", ...). */
int rbmd_profile_enable(rbmd_ctx* ctx, int32_t on);
int rbmd_profile_get(rbmd_ctx* ctx, const char* kernel, double* avg_ms, int64_t* launches,
                     double* units_per_launch);
/* rbmd_step bracketed by CUDA events recorded on the context stream; *ms is the device time of
 * the nsteps steps (the call synchronises). */
int rbmd_step_timed(rbmd_ctx* ctx, const int32_t* sys_ids, int32_t n, int32_t nsteps, double* ms);

/* ---------------------------------------------------------------- autotuner (no reference counterpart) */
/* Pair traversal layouts of the force kernels. */
enum rbmd_pair_layout {
  RBMD_LAYOUT_TILE = 0,     /* warp per home cell, candidate batches shared by the cell's atoms */
  RBMD_LAYOUT_LEAN = 1,     /* warp per atom over per-row segment tables (dims >= 2 nc + 1) */
  RBMD_LAYOUT_GENERAL = 2,  /* warp per atom, any box */
  RBMD_LAYOUT_COLUMN = 3    /* warp per column of home cells, lane per atom walking its own candidate
                               window of a shared staged row (mixed-precision RBL forces of LJ/CUT,
                               LJ/CUT/COUL/LONG and CVFF; the tile layout's boxes) */
};
typedef struct rbmd_tune_result {
  int32_t n_systems;        /* systems of the group (grouped as rbmd_step batches them) */
  int32_t layout;           /* chosen enum rbmd_pair_layout */
  int64_t atoms;            /* atoms of the group */
  double ms[4];             /* measured pair-kernel time per layout (index = layout); -1: unusable or
                               not timed */
  int32_t from_cache;       /* 1: taken from an earlier decision for the same signature */
  int32_t pad0;
} rbmd_tune_result;
/* Times every pair layout the systems can use, one group at a time (cell list built once, one
 * warm-up, best of three launches on the library stream), and keeps the fastest for the group.  A
 * decision is cached per signature (force field, neighbour, Coulomb, precision, special bonds,
 * bonded terms, SHAKE, barostat, atoms per cell and group size, both binned by factors of 2), so
 * later groups with the same signature take it without timing.  Positions, velocities and forces
 * are left as they were.  NPT systems always use RBMD_LAYOUT_GENERAL (their cell dims change).
 * Up to cap results are written; *n_groups gets the number of groups.  Layouts differ only in
 * summation order, so results after tuning agree with untuned ones to rounding, not bit for bit. */
int rbmd_autotune(rbmd_ctx* ctx, const int32_t* sys_ids, int32_t n, rbmd_tune_result* results, int32_t cap,
                  int32_t* n_groups);
/* Non-tensor pipe peak of the device from a dependent FMA chain microbenchmark (fp64 = 0: FFMA,
 * 1: DFMA); *tflops counts an FMA as 2 flops. */
int rbmd_fma_peak(rbmd_ctx* ctx, int32_t fp64, double* tflops);

#ifdef __cplusplus
}
#endif

#endif /* RBMD_GPU_H */
