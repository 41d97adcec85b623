"""rbmd_b200 -- B200-native (sm_100a) force-and-integrate path of RBMD behind a C ABI.

The product is `rbmd_b200/_lib/librbmd_b200.so` (include/rbmd_gpu.h) and the `rbmd` host binary.
This module is a thin ctypes binding of that ABI for Python callers (tests, bench, serving
clients).  There is no CPU fallback: loading fails loudly when the library is missing.
"""
import ctypes as C
import os

import numpy as np

from . import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "librbmd_b200.so")

_lib = None


class RbmdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{A.STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Load the sm_100a library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m rbmd_b200.build` (there is no CPU path)")
        _lib = A.declare(C.CDLL(LIB_PATH))
        if _lib.rbmd_abi_version() != A.RBMD_ABI_VERSION:
            raise ImportError("ABI version mismatch between rbmd_b200/_abi.py and the library")
    return _lib


def _dp(a):
    return a.ctypes.data_as(A.dptr)


def _ip(a):
    return a.ctypes.data_as(A.iptr)


class Context:
    """One CUDA device context: systems, batched steps, serving loop."""

    def __init__(self, device=0, batched=True, graphs=True, hbm_budget_bytes=0, autotune=False):
        L = lib()
        cfg = A.DeviceCfg(device=device, batched=int(batched), use_graphs=int(graphs), autotune=int(autotune),
                          hbm_budget_bytes=int(hbm_budget_bytes))
        h = C.c_void_p()
        rc = L.rbmd_ctx_create(C.byref(cfg), C.byref(h))
        if rc:
            raise RbmdError(rc, "rbmd_ctx_create failed (no CUDA device?)")
        self.h = h
        self._sizes = {}

    def close(self):
        if getattr(self, "h", None):
            lib().rbmd_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc):
        if rc:
            msg = lib().rbmd_last_error(self.h)
            raise RbmdError(rc, msg.decode() if msg else "")
        return rc

    @staticmethod
    def _ids(ids):
        if isinstance(ids, int):
            ids = [ids]
        a = np.ascontiguousarray(ids, np.int32)
        return a, len(a)

    # ---- systems
    def add_system(self, sd, params=None):
        desc = sd.desc()
        prm = params if params is not None else sd.params
        sid = C.c_int32()
        self._check(lib().rbmd_system_add(self.h, C.byref(desc), C.byref(prm), C.byref(sid)))
        self._sizes[sid.value] = (sd.n, prm.coulomb_sample_num if prm.coulomb == A.COUL_RBE else 0)
        return sid.value

    def remove_system(self, sid):
        self._check(lib().rbmd_system_remove(self.h, sid))
        self._sizes.pop(sid, None)

    def init(self, ids):
        a, n = self._ids(ids)
        self._check(lib().rbmd_init(self.h, _ip(a), n))

    def step(self, ids, nsteps=1):
        a, n = self._ids(ids)
        self._check(lib().rbmd_step(self.h, _ip(a), n, nsteps))

    def sync(self):
        self._check(lib().rbmd_sync(self.h))

    def compute_forces(self, ids):
        a, n = self._ids(ids)
        self._check(lib().rbmd_compute_forces(self.h, _ip(a), n))

    def forces(self, sid):
        n = self._sizes[sid][0]
        f = np.zeros((n, 3))
        self._check(lib().rbmd_get_forces(self.h, sid, _dp(f)))
        return f

    def state(self, sid):
        n = self._sizes[sid][0]
        x, v = np.zeros((n, 3)), np.zeros((n, 3))
        img = np.zeros((n, 3), np.int32)
        self._check(lib().rbmd_get_state(self.h, sid, _dp(x), _dp(v), _ip(img)))
        return x, v, img

    def set_step(self, sid, step):
        self._check(lib().rbmd_set_step(self.h, sid, int(step)))

    def set_state(self, sid, x=None, v=None, image=None):
        x = None if x is None else np.ascontiguousarray(x, np.float64)
        v = None if v is None else np.ascontiguousarray(v, np.float64)
        image = None if image is None else np.ascontiguousarray(image, np.int32)
        self._check(lib().rbmd_set_state(self.h, sid, None if x is None else _dp(x),
                                         None if v is None else _dp(v), None if image is None else _ip(image)))

    def thermo(self, sid):
        t = A.Thermo()
        self._check(lib().rbmd_get_thermo(self.h, sid, C.byref(t)))
        return t.as_dict()

    def derived(self, sid):
        d = A.Derived()
        self._check(lib().rbmd_get_derived(self.h, sid, C.byref(d)))
        return {k: (list(getattr(d, k)) if hasattr(getattr(d, k), "__len__") else getattr(d, k))
                for k, _ in d._fields_}

    def cells(self, sid):
        n = self._sizes[sid][0]
        d = self.derived(sid)
        nc = d["n_cells"]
        dims = np.zeros(3, np.int32)
        coa, srt = np.zeros(n, np.int32), np.zeros(n, np.int32)
        lo, up = np.zeros(nc, np.int32), np.zeros(nc, np.int32)
        self._check(lib().rbmd_get_cells(self.h, sid, _ip(dims), _ip(coa), _ip(srt), _ip(lo), _ip(up)))
        return dims, coa, srt, lo, up

    def rbl_lists(self, sid, cap=1024):
        n = self._sizes[sid][0]
        nc, ns = np.zeros(n, np.int32), np.zeros(n, np.int32)
        ids = np.full((n, cap), -1, np.int32)
        self._check(lib().rbmd_get_rbl_lists(self.h, sid, cap, _ip(nc), _ip(ns), _ip(ids)))
        return nc, ns, ids

    def rbl_lists_static(self, sid, cap=1024):
        """rbl_lists without any device allocation, for callers that must not allocate while
        systems run; one 8 MiB file-scope scratch per device, rows core ids, shell ids, then -1."""
        n = self._sizes[sid][0]
        nc, ns = np.zeros(n, np.int32), np.zeros(n, np.int32)
        ids = np.empty((n, cap), np.int32)
        self._check(lib().rbmd_get_rbl_lists_static(self.h, sid, cap, _ip(nc), _ip(ns), _ip(ids)))
        return nc, ns, ids

    def kspace(self, sid):
        P = self._sizes[sid][1]
        m = np.zeros((P, 3), np.int32)
        rk = np.zeros((P, 2))
        self._check(lib().rbmd_get_kspace(self.h, sid, _ip(m), _dp(rk)))
        return m, rk

    # ---- trajectory observables (output/MSDOutput.cpp, VACFOutput.cpp, RDFOutput.cpp)
    def observe_reset(self, sid, msd=True, vacf=True):
        """Take the current positions and image counters (msd) and / or velocities (vacf) as the
        reference configuration of observe()."""
        which = (A.OBS_MSD if msd else 0) | (A.OBS_VACF if vacf else 0)
        self._check(lib().rbmd_observe_reset(self.h, sid, which))

    def observe(self, sid, msd=True, vacf=True):
        """(msd, vacf): atom averages (x, y, z, total) against the reference configuration; None
        for an average not asked for."""
        m = np.zeros(4) if msd else None
        v = np.zeros(4) if vacf else None
        self._check(lib().rbmd_observe(self.h, sid, None if m is None else _dp(m), None if v is None else _dp(v)))
        return m, v

    def rdf_counts(self, sid, centers, targets, radius, dr, exclude_same_molecule=True):
        """Pair counts per RDF bin (rdf_bins(radius, dr)) of the current configuration, and the
        box volume they were taken in."""
        c = np.ascontiguousarray(centers, np.int32)
        t = np.ascontiguousarray(targets, np.int32)
        counts = np.zeros(rdf_bins(radius, dr).size, np.int64)
        vol = C.c_double()
        self._check(lib().rbmd_rdf_counts(self.h, sid, _ip(c), c.size, _ip(t), t.size, float(radius), float(dr),
                                          int(bool(exclude_same_molecule)), counts.ctypes.data_as(A.lptr),
                                          C.byref(vol)))
        return counts, vol.value

    # ---- asynchronous snapshots
    def snapshot_begin(self, sid):
        """Queue a snapshot of the system's state as of the work queued so far; returns a Snapshot
        whose wait() gives (x, v, image, box, step) once the copy has landed (later steps keep
        running meanwhile)."""
        n = self._sizes[sid][0]
        snap = Snapshot(self, n)
        t = C.c_int64()
        self._check(lib().rbmd_snapshot_begin(self.h, sid, _dp(snap.x), _dp(snap.v), _ip(snap.image),
                                              _dp(snap.box), snap.step.ctypes.data_as(A.lptr), C.byref(t)))
        snap.ticket = t.value
        return snap

    # ---- diagnostics
    def launch_count(self):
        v = C.c_int64()
        self._check(lib().rbmd_launch_count(self.h, C.byref(v)))
        return v.value

    def step_timed(self, ids, nsteps):
        """Run nsteps and return their device time in ms (CUDA events on the library stream)."""
        a, n = self._ids(ids)
        ms = C.c_double()
        self._check(lib().rbmd_step_timed(self.h, _ip(a), n, nsteps, C.byref(ms)))
        return ms.value

    def autotune(self, ids, cap=256):
        """Time the pair layouts of these systems (grouped as rbmd_step groups them) and keep the
        fastest per group; returns one dict per group (layout chosen, ms per layout, from_cache)."""
        a, n = self._ids(ids)
        res = (A.TuneResult * cap)()
        ng = C.c_int32()
        self._check(lib().rbmd_autotune(self.h, _ip(a), n, res, cap, C.byref(ng)))
        return [res[k].as_dict() for k in range(min(ng.value, cap))]

    def fma_peak(self, fp64=False):
        v = C.c_double()
        self._check(lib().rbmd_fma_peak(self.h, int(fp64), C.byref(v)))
        return v.value

    def profile(self, on=True):
        self._check(lib().rbmd_profile_enable(self.h, int(on)))

    def profile_get(self, name):
        ms, n, u = C.c_double(), C.c_int64(), C.c_double()
        self._check(lib().rbmd_profile_get(self.h, name.encode(), C.byref(ms), C.byref(n), C.byref(u)))
        return ms.value, n.value, u.value

    # ---- serving
    def serve_start(self, hbm_budget_bytes=0, max_systems=0, steps_per_round=10, graphs=True, round_atoms=0):
        cfg = A.ServeCfg(hbm_budget_bytes=int(hbm_budget_bytes), max_systems=max_systems,
                         steps_per_round=steps_per_round, use_graphs=int(graphs), round_atoms=int(round_atoms))
        self._check(lib().rbmd_serve_start(self.h, C.byref(cfg)))

    def serve_submit(self, sd, nsteps, params=None):
        desc = sd.desc()
        prm = params if params is not None else sd.params
        rid = C.c_int64()
        self._check(lib().rbmd_serve_submit(self.h, C.byref(desc), C.byref(prm), nsteps, C.byref(rid)))
        self._sizes[("req", rid.value)] = sd.n
        return rid.value

    def serve_poll(self, rid):
        st = C.c_int32()
        self._check(lib().rbmd_serve_poll(self.h, rid, C.byref(st)))
        return st.value

    def serve_wait(self, rid, timeout=-1.0):
        return lib().rbmd_serve_wait(self.h, rid, timeout)

    def serve_result(self, rid, want_state=True):
        n = self._sizes.pop(("req", rid))
        x = np.zeros((n, 3)) if want_state else None
        v = np.zeros((n, 3)) if want_state else None
        th, st = A.Thermo(), A.RequestStats()
        rc = lib().rbmd_serve_result(self.h, rid, None if x is None else _dp(x), None if v is None else _dp(v),
                                     C.byref(th), C.byref(st))
        self._check(rc)
        stats = {k: getattr(st, k) for k, _ in st._fields_}
        return x, v, th.as_dict(), stats

    def serve_stop(self):
        self._check(lib().rbmd_serve_stop(self.h))


class Snapshot:
    """Pending rbmd_snapshot_begin: the destination arrays live here until the wait returns."""

    def __init__(self, ctx, n):
        self.ctx = ctx
        self.x, self.v = np.zeros((n, 3)), np.zeros((n, 3))
        self.image = np.zeros((n, 3), np.int32)
        self.box = np.zeros(6)
        self.step = np.zeros(1, np.int64)
        self.ticket = None

    def done(self):
        d = C.c_int32()
        self.ctx._check(lib().rbmd_snapshot_poll(self.ctx.h, self.ticket, C.byref(d)))
        return bool(d.value)

    def wait(self, timeout=-1.0):
        self.ctx._check(lib().rbmd_snapshot_wait(self.ctx.h, self.ticket, float(timeout)))
        return self.x, self.v, self.image, self.box.reshape(2, 3), int(self.step[0])


def read_setfl(path):
    """Reads a setfl (LAMMPS eam/alloy) file into a dict: n_elements, names, mass, nrho, drho, nr,
    dr, cut, frho [n_elements, nrho], rhor [n_elements, nr], z2r [pairs, nr]."""
    f = A.EamSetfl()
    rc = lib().rbmd_eam_read_setfl(str(path).encode(), C.byref(f), None, None, None, None, None)
    if rc:
        raise RbmdError(rc, f"cannot read setfl file {path}")
    ne, nrho, nr = f.n_elements, f.nrho, f.nr
    names = C.create_string_buffer(16 * ne)
    mass, frho, rhor = np.zeros(ne), np.zeros((ne, nrho)), np.zeros((ne, nr))
    z2r = np.zeros((ne * (ne + 1) // 2, nr))
    rc = lib().rbmd_eam_read_setfl(str(path).encode(), C.byref(f), names, _dp(mass), _dp(frho), _dp(rhor), _dp(z2r))
    if rc:
        raise RbmdError(rc, f"cannot read setfl file {path}")
    nm = [names.raw[16 * e:16 * (e + 1)].split(b"\0")[0].decode() for e in range(ne)]
    return dict(n_elements=ne, names=nm, mass=mass, nrho=nrho, drho=f.drho, nr=nr, dr=f.dr, cut=f.cut_off,
                frho=frho, rhor=rhor, z2r=z2r)


def setfl_splines(body, type_element):
    """Per-type EAM spline tables (eam_per_type = 1) of a setfl body: type t takes element
    type_element[t] (rbmd_eam_build_setfl_splines)."""
    f = A.EamSetfl(n_elements=body["n_elements"], nrho=body["nrho"], nr=body["nr"], drho=body["drho"],
                   dr=body["dr"], cut_off=body["cut"])
    te = np.ascontiguousarray(type_element, np.int32)
    nt, nrho, nr = te.size, body["nrho"], body["nr"]
    fs = np.zeros(7 * (nrho + 1) * nt)
    rs = np.zeros(7 * (nr + 1) * nt)
    zs = np.zeros(7 * (nr + 1) * nt * (nt + 1) // 2)
    rhomax = C.c_double()
    frho = np.ascontiguousarray(body["frho"], np.float64)
    rhor = np.ascontiguousarray(body["rhor"], np.float64)
    z2r = np.ascontiguousarray(body["z2r"], np.float64)
    rc = lib().rbmd_eam_build_setfl_splines(C.byref(f), _dp(frho), _dp(rhor), _dp(z2r), _ip(te), nt, _dp(fs),
                                            _dp(rs), _dp(zs), C.byref(rhomax))
    if rc:
        raise RbmdError(rc, "rbmd_eam_build_setfl_splines failed")
    return dict(nrho=nrho, nr=nr, drho=float(body["drho"]), dr=float(body["dr"]), rhomax=rhomax.value,
                cut=float(body["cut"]), frho_spline=fs, rhor_spline=rs, z2r_spline=zs, per_type=1)


def rdf_bins(radius, dr):
    """RDF radii: (int)(radius / dr) bins at dr, 2 dr, ... accumulated (RDFOutput.cpp:42-53)."""
    n = C.c_int32()
    rc = lib().rbmd_rdf_bins(float(radius), float(dr), None, 0, C.byref(n))
    if rc:
        raise RbmdError(rc, "rdf_bins: radius and dr must be positive with radius / dr >= 1")
    r = np.zeros(n.value)
    lib().rbmd_rdf_bins(float(radius), float(dr), _dp(r), n.value, C.byref(n))
    return r


# single-precision pi of the reference's normalisation (vtkm::Pif, OutPutWorklet.cpp:303-306)
PI_F32 = float(np.float32(np.pi))


def rdf_snapshot(counts, radii, n_centers, n_targets, volume):
    """One snapshot's RDF from its pair counts (ComputeRDFWorklet, OutPutWorklet.cpp:303-306):
    counts / (n_centers * rho * (4/3 pi (1.01 r)^3 - 4/3 pi r^3)), rho = n_targets / volume.
    NaN where the denominator is zero (no centers or targets), as in the reference."""
    r = np.asarray(radii, np.float64)
    rho = n_targets / volume
    shell = (4 / 3.0) * PI_F32 * (r + r * 0.01) ** 3 - ((4 / 3.0) * PI_F32 * r ** 3)
    den = n_centers * rho * shell
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.asarray(counts, np.float64) / den


def system_bytes(sd, params=None):
    """Device bytes a system takes (rbmd_system_bytes): the figure serving admission charges."""
    desc = sd.desc()
    out = C.c_int64()
    rc = lib().rbmd_system_bytes(C.byref(desc), C.byref(params if params is not None else sd.params), C.byref(out))
    if rc:
        raise RbmdError(rc, "rbmd_system_bytes")
    return out.value


def eam_splines(file_dict):
    """rbmd_eam_build_splines on a funcfl body given as a dict of numpy arrays."""
    L = lib()
    frho = np.ascontiguousarray(file_dict["frho"], np.float64)
    zr = np.ascontiguousarray(file_dict["zr"], np.float64)
    rhor = np.ascontiguousarray(file_dict["rhor"], np.float64)
    f = A.EamFile(nrho=int(file_dict["nrho"]), nr=int(file_dict["nr"]), drho=float(file_dict["drho"]),
                  dr=float(file_dict["dr"]), cut_off=float(file_dict["cut"]), frho=_dp(frho), zr=_dp(zr),
                  rhor=_dp(rhor))
    nrho, nr = C.c_int32(), C.c_int32()
    if L.rbmd_eam_spline_sizes(C.byref(f), C.byref(nrho), C.byref(nr)):
        raise RbmdError(A.ERR_ARG, "bad EAM table")
    fs = np.zeros(7 * (nrho.value + 1))
    rs = np.zeros(7 * (nr.value + 1))
    zs = np.zeros(7 * (nr.value + 1))
    o_nrho, o_nr = C.c_int32(), C.c_int32()
    drho, dr, rhomax = C.c_double(), C.c_double(), C.c_double()
    rc = L.rbmd_eam_build_splines(C.byref(f), _dp(fs), _dp(rs), _dp(zs), C.byref(o_nrho), C.byref(drho),
                                  C.byref(o_nr), C.byref(dr), C.byref(rhomax))
    if rc:
        raise RbmdError(rc, "rbmd_eam_build_splines failed")
    return dict(nrho=o_nrho.value, nr=o_nr.value, drho=drho.value, dr=dr.value, rhomax=rhomax.value,
                cut=float(file_dict["cut"]), frho_spline=fs, rhor_spline=rs, z2r_spline=zs)


def read_funcfl(path):
    """rbmd_eam_read_funcfl: the body of a funcfl EAM file as a dict of numpy arrays."""
    L = lib()
    f = A.EamFile()
    rc = L.rbmd_eam_read_funcfl(path.encode(), C.byref(f), None, None, None)
    if rc:
        raise RbmdError(rc, path)
    frho, zr, rhor = np.zeros(f.nrho), np.zeros(f.nr), np.zeros(f.nr)
    rc = L.rbmd_eam_read_funcfl(path.encode(), C.byref(f), _dp(frho), _dp(zr), _dp(rhor))
    if rc:
        raise RbmdError(rc, path)
    return dict(nrho=f.nrho, nr=f.nr, drho=f.drho, dr=f.dr, cut=f.cut_off, frho=frho, zr=zr, rhor=rhor)
