"""ctypes mirror of include/rbmd_gpu.h (structs, enums, prototypes).

The C header is the source of truth; tests/test_abi.py checks field offsets against it by compiling
a probe with the host compiler.
"""
import ctypes as C

RBMD_ABI_VERSION = 6

# status
OK, ERR_ARG, ERR_OOM, ERR_NUMERIC, ERR_TIMEOUT, ERR_CUDA, ERR_STATE, ERR_BUDGET, ERR_UNSUPPORTED, ERR_IO = range(10)
STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_OOM", 3: "ERR_NUMERIC", 4: "ERR_TIMEOUT",
                5: "ERR_CUDA", 6: "ERR_STATE", 7: "ERR_BUDGET", 8: "ERR_UNSUPPORTED", 9: "ERR_IO"}

# bits of the device status word (rbmd_thermo.status), enum rbmd_status_bit
(STATUS_SHAKE_OVERFLOW, STATUS_SHAKE_SINGULAR, STATUS_SHAKE_NO_CONVERGE, STATUS_RATTLE_SINGULAR,
 STATUS_NON_FINITE, STATUS_RBE_SLOTS, STATUS_BOX_RANGE) = (1, 2, 4, 8, 16, 32, 64)

FF_LJ_CUT, FF_LJ_CUT_COUL_LONG, FF_CVFF, FF_EAM = 0, 1, 2, 3
NEIGH_RBL, NEIGH_VERLET = 0, 1
COUL_NONE, COUL_RBE, COUL_EWALD = 0, 1, 2
NEAR_ANALYTIC, NEAR_TABLE = 0, 1
TC_NOSE_HOOVER, TC_BERENDSEN, TC_RESCALE, TC_NONE = 0, 1, 2, 3
UNITS_LJ, UNITS_REAL, UNITS_METAL = 0, 1, 2
PREC_FP64, PREC_MIXED = 0, 1
RBL_STRIDE, RBL_PHILOX = 0, 1
RANDOM_PHILOX, RANDOM_TEST = 0, 1
SHAKE_NULL, SHAKE_FALSE, SHAKE_TRUE = -1, 0, 1
ENS_NVT, ENS_NVE, ENS_NPT = 0, 1, 2
PC_BERENDSEN, PC_NOSE_HOOVER = 0, 1
OBS_MSD, OBS_VACF = 1, 2
PRESS_CTRLS = {"BERENDSEN": PC_BERENDSEN, "NOSE_HOOVER": PC_NOSE_HOOVER}
REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED = 0, 1, 2, 3

FORCE_FIELDS = {"LJ/CUT": FF_LJ_CUT, "LJ/CUT/COUL/LONG": FF_LJ_CUT_COUL_LONG, "CVFF": FF_CVFF, "EAM": FF_EAM}
NEIGHBORS = {"RBL": NEIGH_RBL, "VERLETLIST": NEIGH_VERLET}
COULOMBS = {"RBE": COUL_RBE, "EWALD": COUL_EWALD}
TEMP_CTRLS = {"NOSE_HOOVER": TC_NOSE_HOOVER, "BERENDSEN": TC_BERENDSEN, "TEMP_RESCALE": TC_RESCALE}
UNITS = {"LJ": UNITS_LJ, "REAL": UNITS_REAL, "METAL": UNITS_METAL}

dptr = C.POINTER(C.c_double)
iptr = C.POINTER(C.c_int32)
lptr = C.POINTER(C.c_int64)


class Params(C.Structure):
    _fields_ = [
        ("force_field", C.c_int32), ("neighbor", C.c_int32), ("coulomb", C.c_int32),
        ("ensemble", C.c_int32), ("temp_ctrl", C.c_int32), ("units", C.c_int32),
        ("precision", C.c_int32), ("rbl_mode", C.c_int32), ("random_mode", C.c_int32),
        ("fix_shake", C.c_int32), ("init_inbuild", C.c_int32), ("neighbor_sample_num", C.c_int32),
        ("cut_off", C.c_double), ("r_core", C.c_double),
        ("coulomb_sample_num", C.c_int32), ("kmax", C.c_int32 * 3),
        ("alpha", C.c_double), ("temperature", C.c_double * 3), ("pressure", C.c_double * 3),
        ("press_ctrl", C.c_int32), ("near_table", C.c_int32),
        ("timestep", C.c_double), ("num_steps", C.c_int64),
        ("special_bonds", C.c_double * 3), ("seed", C.c_uint64), ("bulk_modulus", C.c_double),
    ]


class SystemDesc(C.Structure):
    _fields_ = [
        ("n_atoms", C.c_int32), ("n_types", C.c_int32),
        ("box_lo", C.c_double * 3), ("box_hi", C.c_double * 3),
        ("position", dptr), ("velocity", dptr), ("charge", dptr), ("mass", dptr),
        ("type", iptr), ("molecule", iptr), ("image", iptr),
        ("epsilon", dptr), ("sigma", dptr),
        ("n_bonds", C.c_int32), ("n_bond_types", C.c_int32),
        ("bond_atoms", iptr), ("bond_type", iptr), ("bond_k", dptr), ("bond_r0", dptr),
        ("n_angles", C.c_int32), ("n_angle_types", C.c_int32),
        ("angle_atoms", iptr), ("angle_type", iptr), ("angle_k", dptr), ("angle_theta0", dptr),
        ("special_offsets", iptr), ("special_ids", iptr), ("special_weights", dptr),
        ("eam_nrho", C.c_int32), ("eam_nr", C.c_int32),
        ("eam_drho", C.c_double), ("eam_dr", C.c_double), ("eam_rhomax", C.c_double),
        ("eam_cut", C.c_double),
        ("eam_frho_spline", dptr), ("eam_rhor_spline", dptr), ("eam_z2r_spline", dptr),
        ("n_dihedrals", C.c_int32), ("n_dihedral_types", C.c_int32),
        ("dihedral_atoms", iptr), ("dihedral_type", iptr), ("dihedral_k", dptr), ("dihedral_sign", iptr),
        ("dihedral_multiplicity", iptr),
        ("eam_per_type", C.c_int32), ("pad_eam", C.c_int32),
        ("near_table_values", C.POINTER(C.c_float)),
    ]


class Thermo(C.Structure):
    _fields_ = [
        ("step", C.c_int64), ("temperature", C.c_double), ("tempT_sum", C.c_double),
        ("kinetic_energy", C.c_double), ("e_lj", C.c_double), ("e_coul_near", C.c_double),
        ("e_coul_far", C.c_double), ("e_bond", C.c_double), ("e_angle", C.c_double),
        ("e_eam", C.c_double), ("potential_energy", C.c_double), ("total_energy", C.c_double),
        ("pressure", C.c_double), ("virial", C.c_double * 6), ("nhc_eta", C.c_double * 3),
        ("nhc_eta_dot", C.c_double * 4), ("volume", C.c_double), ("box_lo", C.c_double * 3),
        ("box_hi", C.c_double * 3), ("status", C.c_int32), ("pad0", C.c_int32), ("e_dihedral", C.c_double),
    ]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            val = getattr(self, name)
            if hasattr(val, "__len__"):
                val = list(val)
            out[name] = val
        out.pop("pad0", None)
        return out


class Derived(C.Structure):
    _fields_ = [
        ("rs_num", C.c_int32), ("rc_num", C.c_int32), ("pice_num", C.c_int32),
        ("num_cycles", C.c_int32), ("dims", C.c_int32 * 3), ("n_cells", C.c_int32),
        ("rho_system", C.c_double), ("S_rbe", C.c_double), ("volume", C.c_double),
        ("cell_width", C.c_double * 3),
    ]


class DeviceCfg(C.Structure):
    _fields_ = [("device", C.c_int32), ("batched", C.c_int32), ("use_graphs", C.c_int32),
                ("autotune", C.c_int32), ("hbm_budget_bytes", C.c_int64)]


LAYOUT_TILE, LAYOUT_LEAN, LAYOUT_GENERAL, LAYOUT_COLUMN = 0, 1, 2, 3
LAYOUT_NAMES = {LAYOUT_TILE: "tile", LAYOUT_LEAN: "lean", LAYOUT_GENERAL: "general", LAYOUT_COLUMN: "column"}


class TuneResult(C.Structure):
    _fields_ = [("n_systems", C.c_int32), ("layout", C.c_int32), ("atoms", C.c_int64), ("ms", C.c_double * 4),
                ("from_cache", C.c_int32), ("pad0", C.c_int32)]

    def as_dict(self):
        return dict(n_systems=self.n_systems, layout=LAYOUT_NAMES[self.layout], atoms=self.atoms,
                    ms={LAYOUT_NAMES[k]: self.ms[k] for k in range(4)}, from_cache=bool(self.from_cache))


class EamSetfl(C.Structure):
    _fields_ = [("n_elements", C.c_int32), ("nrho", C.c_int32), ("nr", C.c_int32), ("pad0", C.c_int32),
                ("drho", C.c_double), ("dr", C.c_double), ("cut_off", C.c_double)]


class ServeCfg(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_int64), ("max_systems", C.c_int32),
                ("steps_per_round", C.c_int32), ("use_graphs", C.c_int32), ("round_atoms", C.c_int32)]


class RequestStats(C.Structure):
    _fields_ = [("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double),
                ("atom_steps", C.c_int64), ("n_atoms", C.c_int32), ("status", C.c_int32)]


class EamFile(C.Structure):
    _fields_ = [("nrho", C.c_int32), ("nr", C.c_int32), ("drho", C.c_double), ("dr", C.c_double),
                ("cut_off", C.c_double), ("frho", dptr), ("zr", dptr), ("rhor", dptr)]


def default_params(**kw):
    """Python twin of rbmd_params_default (the reference defaults), with keyword overrides."""
    p = Params()
    p.force_field = FF_LJ_CUT
    p.neighbor = NEIGH_RBL
    p.coulomb = COUL_NONE
    p.ensemble = ENS_NVT
    p.temp_ctrl = TC_NOSE_HOOVER
    p.units = UNITS_LJ
    p.precision = PREC_FP64
    p.rbl_mode = RBL_STRIDE
    p.random_mode = RANDOM_PHILOX
    p.fix_shake = SHAKE_NULL
    p.init_inbuild = 0
    p.neighbor_sample_num = 100
    p.cut_off = 2.5
    p.r_core = 1.2
    p.coulomb_sample_num = 100
    p.kmax[:] = (3, 3, 3)
    p.alpha = 0.1
    p.temperature[:] = (1.0, 1.0, 0.5)
    p.pressure[:] = (1.0, 1.0, 1000.0)
    p.bulk_modulus = 10.0
    p.press_ctrl = 0
    p.timestep = 0.005
    p.num_steps = 1000
    p.special_bonds[:] = (0.0, 0.0, 0.0)
    p.seed = 1
    for k, v in kw.items():
        cur = getattr(p, k)
        if hasattr(cur, "__len__"):
            cur[:] = v
        else:
            setattr(p, k, v)
    return p


def declare(lib, prefix="rbmd"):
    """Attach argtypes/restype for every exported entry point of include/rbmd_gpu.h."""
    P, V = C.POINTER, C.c_void_p
    ctx = V
    sig = {
        "abi_version": ([], C.c_int),
        "params_default": ([P(Params)], None),
        "ctx_create": ([P(DeviceCfg), P(V)], C.c_int),
        "ctx_destroy": ([ctx], C.c_int),
        "last_error": ([ctx], C.c_char_p),
        "system_bytes": ([P(SystemDesc), P(Params), P(C.c_int64)], C.c_int),
        "system_add": ([ctx, P(SystemDesc), P(Params), P(C.c_int32)], C.c_int),
        "system_remove": ([ctx, C.c_int32], C.c_int),
        "init": ([ctx, iptr, C.c_int32], C.c_int),
        "step": ([ctx, iptr, C.c_int32, C.c_int32], C.c_int),
        "sync": ([ctx], C.c_int),
        "compute_forces": ([ctx, iptr, C.c_int32], C.c_int),
        "get_forces": ([ctx, C.c_int32, dptr], C.c_int),
        "get_state": ([ctx, C.c_int32, dptr, dptr, iptr], C.c_int),
        "set_state": ([ctx, C.c_int32, dptr, dptr, iptr], C.c_int),
        "set_step": ([ctx, C.c_int32, C.c_int64], C.c_int),
        "get_thermo": ([ctx, C.c_int32, P(Thermo)], C.c_int),
        "get_cells": ([ctx, C.c_int32, iptr, iptr, iptr, iptr, iptr], C.c_int),
        "get_rbl_lists": ([ctx, C.c_int32, C.c_int32, iptr, iptr, iptr], C.c_int),
        "get_rbl_lists_static": ([ctx, C.c_int32, C.c_int32, iptr, iptr, iptr], C.c_int),
        "get_kspace": ([ctx, C.c_int32, iptr, dptr], C.c_int),
        "get_derived": ([ctx, C.c_int32, P(Derived)], C.c_int),
        "eam_spline_sizes": ([P(EamFile), iptr, iptr], C.c_int),
        "eam_build_splines": ([P(EamFile), dptr, dptr, dptr, iptr, dptr, iptr, dptr, dptr], C.c_int),
        "eam_read_funcfl": ([C.c_char_p, P(EamFile), dptr, dptr, dptr], C.c_int),
        "eam_read_setfl": ([C.c_char_p, P(EamSetfl), C.c_char_p, dptr, dptr, dptr, dptr], C.c_int),
        "eam_build_setfl_splines": ([P(EamSetfl), dptr, dptr, dptr, iptr, C.c_int32, dptr, dptr, dptr, dptr],
                                    C.c_int),
        "serve_start": ([ctx, P(ServeCfg)], C.c_int),
        "serve_submit": ([ctx, P(SystemDesc), P(Params), C.c_int32, P(C.c_int64)], C.c_int),
        "serve_poll": ([ctx, C.c_int64, iptr], C.c_int),
        "serve_wait": ([ctx, C.c_int64, C.c_double], C.c_int),
        "serve_result": ([ctx, C.c_int64, dptr, dptr, P(Thermo), P(RequestStats)], C.c_int),
        "serve_stop": ([ctx], C.c_int),
        "launch_count": ([ctx, P(C.c_int64)], C.c_int),
        "profile_enable": ([ctx, C.c_int32], C.c_int),
        "profile_get": ([ctx, C.c_char_p, dptr, P(C.c_int64), dptr], C.c_int),
        "step_timed": ([ctx, iptr, C.c_int32, C.c_int32, dptr], C.c_int),
        "fma_peak": ([ctx, C.c_int32, dptr], C.c_int),
        "autotune": ([ctx, iptr, C.c_int32, P(TuneResult), C.c_int32, iptr], C.c_int),
        "observe_reset": ([ctx, C.c_int32, C.c_int32], C.c_int),
        "observe": ([ctx, C.c_int32, dptr, dptr], C.c_int),
        "rdf_bins": ([C.c_double, C.c_double, dptr, C.c_int32, iptr], C.c_int),
        "near_table_key": ([C.c_float], C.c_int32),
        "near_table_default": ([C.POINTER(C.c_float)], C.c_int),
        "snapshot_begin": ([ctx, C.c_int32, dptr, dptr, iptr, dptr, lptr, lptr], C.c_int),
        "snapshot_poll": ([ctx, C.c_int64, iptr], C.c_int),
        "snapshot_wait": ([ctx, C.c_int64, C.c_double], C.c_int),
        "rdf_counts": ([ctx, C.c_int32, iptr, C.c_int32, iptr, C.c_int32, C.c_double, C.c_double, C.c_int32,
                        lptr, dptr], C.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, f"{prefix}_{name}")
        fn.argtypes = args
        fn.restype = res
    return lib


HEADER_FUNCTIONS = [
    "rbmd_abi_version", "rbmd_params_default", "rbmd_ctx_create", "rbmd_ctx_destroy",
    "rbmd_last_error", "rbmd_system_bytes", "rbmd_system_add", "rbmd_system_remove", "rbmd_init",
    "rbmd_step", "rbmd_sync", "rbmd_compute_forces", "rbmd_get_forces", "rbmd_get_state",
    "rbmd_set_state", "rbmd_set_step", "rbmd_get_thermo", "rbmd_get_cells", "rbmd_get_rbl_lists", "rbmd_get_rbl_lists_static",
    "rbmd_get_kspace",
    "rbmd_get_derived", "rbmd_eam_spline_sizes", "rbmd_eam_build_splines", "rbmd_eam_read_funcfl",
    "rbmd_serve_start", "rbmd_serve_submit", "rbmd_serve_poll", "rbmd_serve_wait",
    "rbmd_serve_result", "rbmd_serve_stop", "rbmd_launch_count", "rbmd_profile_enable",
    "rbmd_profile_get", "rbmd_step_timed", "rbmd_fma_peak", "rbmd_autotune",
    "rbmd_observe_reset", "rbmd_observe", "rbmd_rdf_bins", "rbmd_rdf_counts",
    "rbmd_snapshot_begin", "rbmd_snapshot_poll", "rbmd_snapshot_wait",
    "rbmd_eam_read_setfl", "rbmd_eam_build_setfl_splines", "rbmd_near_table_key", "rbmd_near_table_default",
]
