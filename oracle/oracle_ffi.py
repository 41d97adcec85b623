"""ctypes wrapper of the FP64 oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
and reference legs, as the checker and the CPU baseline; never by the rbmd_b200 package.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


def build():
    """Compile the oracle with its Makefile (g++)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        from rbmd_b200 import _abi as A
        L = C.CDLL(LIB_PATH)
        V, P = C.c_void_p, C.POINTER
        L.oracle_create.argtypes = [P(A.SystemDesc), P(A.Params)]
        L.oracle_create.restype = V
        L.oracle_destroy.argtypes = [V]
        L.oracle_destroy.restype = None
        for name, args in {
            "oracle_init": [V], "oracle_step": [V, C.c_int], "oracle_compute_forces": [V],
            "oracle_set_step": [V, C.c_int64], "oracle_get_forces": [V, A.dptr],
            "oracle_get_force_part": [V, C.c_int, A.dptr],
            "oracle_get_state": [V, A.dptr, A.dptr, A.iptr],
            "oracle_set_state": [V, A.dptr, A.dptr, A.iptr],
            "oracle_get_thermo": [V, P(A.Thermo)],
            "oracle_get_cells": [V, A.iptr, A.iptr, A.iptr, A.iptr, A.iptr],
            "oracle_get_rbl_lists": [V, C.c_int32, A.iptr, A.iptr, A.iptr],
            "oracle_get_verlet_lists": [V, C.c_int32, A.iptr, A.iptr],
            "oracle_sample_k": [V, A.iptr], "oracle_get_kspace": [V, A.iptr, A.dptr],
            "oracle_ewald_kspace_force": [V, A.dptr], "oracle_get_derived": [V, P(A.Derived)],
            "oracle_status": [V],
            "oracle_eam_read_funcfl": [C.c_char_p, A.iptr, A.iptr, A.dptr, A.dptr, A.dptr, A.dptr,
                                       A.dptr, A.dptr],
            "oracle_eam_build_splines": [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                         A.dptr, A.dptr, A.dptr, A.dptr, A.dptr, A.dptr, A.iptr,
                                         A.dptr, A.iptr, A.dptr, A.dptr],
        }.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int
        _lib = L
    return _lib


def philox_kat(ctr, key):
    """Philox4x32-10 of the oracle on one counter/key (known-answer checks)."""
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    L = lib()
    L.oracle_philox.argtypes = [C.POINTER(C.c_uint32)] * 3
    L.oracle_philox.restype = C.c_int
    L.oracle_philox(c, k, o)
    return list(o)


def near_table():
    """The oracle's near-Coulomb table (2048 float32 G values by key, alpha = 0.1)."""
    import numpy as np
    out = np.zeros(2048, np.float32)
    L = lib()
    L.oracle_near_table.argtypes = [C.POINTER(C.c_float)]
    L.oracle_near_table.restype = C.c_int
    assert L.oracle_near_table(out.ctypes.data_as(C.POINTER(C.c_float))) == 0
    return out


def near_key(r):
    """Key of a distance (bits 15-25 of its float32 pattern)."""
    L = lib()
    L.oracle_near_key.argtypes = [C.c_float]
    L.oracle_near_key.restype = C.c_int
    return L.oracle_near_key(float(r))


def _dp(a):
    from rbmd_b200 import _abi as A
    return a.ctypes.data_as(A.dptr)


def _ip(a):
    from rbmd_b200 import _abi as A
    return a.ctypes.data_as(A.iptr)


class Oracle:
    """One system in the FP64 oracle."""

    def __init__(self, sd, params=None):
        self.sd = sd
        self.n = sd.n
        desc = sd.desc()
        prm = params if params is not None else sd.params
        self.params = prm
        self.h = lib().oracle_create(C.byref(desc), C.byref(prm))
        if not self.h:
            raise ValueError("oracle_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    def init(self):
        lib().oracle_init(self.h)

    def step(self, n=1):
        return lib().oracle_step(self.h, n)

    def set_step(self, s):
        lib().oracle_set_step(self.h, s)

    def compute_forces(self):
        lib().oracle_compute_forces(self.h)

    def forces(self):
        f = np.zeros((self.n, 3))
        lib().oracle_get_forces(self.h, _dp(f))
        return f

    def force_part(self, part):
        f = np.zeros((self.n, 3))
        lib().oracle_get_force_part(self.h, part, _dp(f))
        return f

    def state(self):
        x = np.zeros((self.n, 3))
        v = np.zeros((self.n, 3))
        img = np.zeros((self.n, 3), np.int32)
        lib().oracle_get_state(self.h, _dp(x), _dp(v), _ip(img))
        return x, v, img

    def set_state(self, x=None, v=None, image=None):
        x = None if x is None else np.ascontiguousarray(x, np.float64)
        v = None if v is None else np.ascontiguousarray(v, np.float64)
        image = None if image is None else np.ascontiguousarray(image, np.int32)
        lib().oracle_set_state(self.h, None if x is None else _dp(x), None if v is None else _dp(v),
                               None if image is None else _ip(image))

    def thermo(self):
        from rbmd_b200 import _abi as A
        t = A.Thermo()
        lib().oracle_get_thermo(self.h, C.byref(t))
        return t.as_dict()

    def cells(self):
        d = self.derived()
        nc = d["n_cells"]
        dims = np.zeros(3, np.int32)
        coa = np.zeros(self.n, np.int32)
        srt = np.zeros(self.n, np.int32)
        lo = np.zeros(nc, np.int32)
        up = np.zeros(nc, np.int32)
        lib().oracle_get_cells(self.h, _ip(dims), _ip(coa), _ip(srt), _ip(lo), _ip(up))
        return dims, coa, srt, lo, up

    def rbl_lists(self, cap=1024):
        nc = np.zeros(self.n, np.int32)
        ns = np.zeros(self.n, np.int32)
        ids = np.full((self.n, cap), -1, np.int32)
        rc = lib().oracle_get_rbl_lists(self.h, cap, _ip(nc), _ip(ns), _ip(ids))
        if rc:
            raise ValueError("list row exceeds cap")
        return nc, ns, ids

    def verlet_lists(self, cap=2048):
        n = np.zeros(self.n, np.int32)
        ids = np.full((self.n, cap), -1, np.int32)
        rc = lib().oracle_get_verlet_lists(self.h, cap, _ip(n), _ip(ids))
        if rc:
            raise ValueError("list row exceeds cap")
        return n, ids

    def sample_k(self):
        P = self.params.coulomb_sample_num
        m = np.zeros((P, 3), np.int32)
        lib().oracle_sample_k(self.h, _ip(m))
        return m

    def kspace(self):
        P = self.params.coulomb_sample_num
        m = np.zeros((P, 3), np.int32)
        rk = np.zeros((P, 2))
        lib().oracle_get_kspace(self.h, _ip(m), _dp(rk))
        return m, rk

    def ewald_kspace_force(self):
        f = np.zeros((self.n, 3))
        lib().oracle_ewald_kspace_force(self.h, _dp(f))
        return f

    def derived(self):
        from rbmd_b200 import _abi as A
        d = A.Derived()
        lib().oracle_get_derived(self.h, C.byref(d))
        return {k: (list(getattr(d, k)) if hasattr(getattr(d, k), "__len__") else getattr(d, k))
                for k, _ in d._fields_}

    def status(self):
        return lib().oracle_status(self.h)


def eam_splines(file_dict):
    """Oracle restatement of file2array + array2spline for a funcfl body (dict of numpy arrays)."""
    nrho_in, nr_in = int(file_dict["nrho"]), int(file_dict["nr"])
    # rows after resampling
    rmax = (nr_in - 1) * file_dict["dr"]
    rhomax = (nrho_in - 1) * file_dict["drho"]
    nr = int(rmax / file_dict["dr"] + 0.5)
    nrho = int(rhomax / file_dict["drho"] + 0.5)
    fs = np.zeros(7 * (nrho + 1))
    rs = np.zeros(7 * (nr + 1))
    zs = np.zeros(7 * (nr + 1))
    o_nrho, o_nr = np.zeros(1, np.int32), np.zeros(1, np.int32)
    o_drho, o_dr, o_rhomax = np.zeros(1), np.zeros(1), np.zeros(1)
    frho = np.ascontiguousarray(file_dict["frho"], np.float64)
    zr = np.ascontiguousarray(file_dict["zr"], np.float64)
    rhor = np.ascontiguousarray(file_dict["rhor"], np.float64)
    lib().oracle_eam_build_splines(nrho_in, nr_in, file_dict["drho"], file_dict["dr"], file_dict["cut"],
                                   _dp(frho), _dp(zr), _dp(rhor), _dp(fs), _dp(rs), _dp(zs),
                                   _ip(o_nrho), _dp(o_drho), _ip(o_nr), _dp(o_dr), _dp(o_rhomax))
    return dict(nrho=int(o_nrho[0]), nr=int(o_nr[0]), drho=float(o_drho[0]), dr=float(o_dr[0]),
                rhomax=float(o_rhomax[0]), cut=float(file_dict["cut"]), frho_spline=fs,
                rhor_spline=rs, z2r_spline=zs)


def read_funcfl(path):
    nrho, nr = np.zeros(1, np.int32), np.zeros(1, np.int32)
    drho, dr, cut = np.zeros(1), np.zeros(1), np.zeros(1)
    rc = lib().oracle_eam_read_funcfl(path.encode(), _ip(nrho), _ip(nr), _dp(drho), _dp(dr), _dp(cut),
                                      None, None, None)
    if rc:
        raise IOError(path)
    frho, zr, rhor = np.zeros(int(nrho[0])), np.zeros(int(nr[0])), np.zeros(int(nr[0]))
    lib().oracle_eam_read_funcfl(path.encode(), _ip(nrho), _ip(nr), _dp(drho), _dp(dr), _dp(cut),
                                 _dp(frho), _dp(zr), _dp(rhor))
    return dict(nrho=int(nrho[0]), nr=int(nr[0]), drho=float(drho[0]), dr=float(dr[0]),
                cut=float(cut[0]), frho=frho, zr=zr, rhor=rhor)


# ---------------------------------------------------------------- trajectory observables
def _observe_sigs():
    L = lib()
    i32, d, P = C.c_int32, C.c_double, C.POINTER
    dp, ip, lp = P(C.c_double), P(C.c_int32), P(C.c_int64)
    L.oracle_rdf_bins.argtypes = [d, d, dp, C.c_int]
    L.oracle_msd_vacf.argtypes = [C.c_int, dp, ip, dp, dp, ip, dp, dp, dp, dp]
    L.oracle_rdf_counts.argtypes = [dp, ip, dp, ip, C.c_int, ip, C.c_int, d, d, C.c_int, lp]
    for f in (L.oracle_rdf_bins, L.oracle_msd_vacf, L.oracle_rdf_counts):
        f.restype = C.c_int
    return L


def rdf_bins(radius, dr):
    """RDF radii (RDFOutput.cpp:42-53): (int)(radius / dr) values, dr accumulated."""
    L = _observe_sigs()
    nb = L.oracle_rdf_bins(float(radius), float(dr), None, 0)
    if nb < 0:
        raise ValueError("bad radius / dr")
    r = np.zeros(nb)
    L.oracle_rdf_bins(float(radius), float(dr), _dp(r), nb)
    return r


def msd_vacf(x0, img0, v0, x, img, v, box_len):
    """(msd[4], vacf[4]) atom averages of the unwrapped displacement and v0 . v."""
    L = _observe_sigs()
    a = [np.ascontiguousarray(t, np.float64) for t in (x0, v0, x, v, box_len)]
    ii = [np.ascontiguousarray(t, np.int32) for t in (img0, img)]
    msd, vacf = np.zeros(4), np.zeros(4)
    L.oracle_msd_vacf(a[0].shape[0], _dp(a[0]), _ip(ii[0]), _dp(a[1]), _dp(a[2]), _ip(ii[1]), _dp(a[3]),
                      _dp(a[4]), _dp(msd), _dp(vacf))
    return msd, vacf


def rdf_counts(x, molecule, box_len, centers, targets, radius, dr, exclude_same_molecule=True):
    """Pair counts per RDF bin of one configuration (every periodic image inside the last edge)."""
    L = _observe_sigs()
    x = np.ascontiguousarray(x, np.float64)
    mol = np.ascontiguousarray(molecule, np.int32)
    bl = np.ascontiguousarray(box_len, np.float64)
    c = np.ascontiguousarray(centers, np.int32)
    t = np.ascontiguousarray(targets, np.int32)
    counts = np.zeros(rdf_bins(radius, dr).size, np.int64)
    L.oracle_rdf_counts(_dp(x), _ip(mol), _dp(bl), _ip(c), c.size, _ip(t), t.size, float(radius), float(dr),
                        int(bool(exclude_same_molecule)), counts.ctypes.data_as(C.POINTER(C.c_int64)))
    return counts


def setfl_splines(body, type_element):
    """Per-type EAM tables of a setfl body, restated (checks rbmd_eam_build_setfl_splines)."""
    L = lib()
    P = C.POINTER
    L.oracle_eam_build_setfl_splines.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_int32, C.c_double,
                                                 P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_int32),
                                                 C.c_int32, P(C.c_double), P(C.c_double), P(C.c_double),
                                                 P(C.c_double)]
    L.oracle_eam_build_setfl_splines.restype = C.c_int
    te = np.ascontiguousarray(type_element, np.int32)
    nt, nrho, nr = te.size, int(body["nrho"]), int(body["nr"])
    fs, rs = np.zeros(7 * (nrho + 1) * nt), np.zeros(7 * (nr + 1) * nt)
    zs = np.zeros(7 * (nr + 1) * nt * (nt + 1) // 2)
    rhomax = np.zeros(1)
    frho = np.ascontiguousarray(body["frho"], np.float64)
    rhor = np.ascontiguousarray(body["rhor"], np.float64)
    z2r = np.ascontiguousarray(body["z2r"], np.float64)
    L.oracle_eam_build_setfl_splines(int(body["n_elements"]), nrho, float(body["drho"]), nr, float(body["dr"]),
                                     _dp(frho), _dp(rhor), _dp(z2r), _ip(te), nt, _dp(fs), _dp(rs), _dp(zs),
                                     _dp(rhomax))
    return dict(nrho=nrho, nr=nr, drho=float(body["drho"]), dr=float(body["dr"]), rhomax=float(rhomax[0]),
                cut=float(body["cut"]), frho_spline=fs, rhor_spline=rs, z2r_spline=zs, per_type=1)
