"""The reference's own bundled inputs (rbmd.json + LAMMPS data / funcfl files), read at test time
from the reference tree when it is present (RBMD_REFERENCE_ROOT, default the reference checkout
this project is built against); nothing of it is copied into the repository.

`resolve(rel)` copies the input's directory into a scratch directory (the host opens data files
relative to its working directory, and writes outputs there), runs `rbmd -j ... --dump-system`
(which resolves the input without touching a GPU) and returns the dump; `load(dump)` turns it into
a SystemData for the library and the oracle.
"""
import json
import os
import re
import shutil
import subprocess

import numpy as np

from rbmd_b200 import _abi as A
from rbmd_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RBMD = os.path.join(ROOT, "rbmd_b200", "_lib", "rbmd")
REF_ROOT = os.environ.get("RBMD_REFERENCE_ROOT", "/root/reference")

# bundled inputs whose files are all in the tree (res/json_files/EAM/Cu/box_72108144 names a data
# file that is not there, res/json_files/EAM/{Ag,Au,Ni} name potentials by absolute Windows paths)
INPUTS = {
    "h2o_box_305038": "res/json_files/H2O/box_305038/rbmd.json",   # SPC/E water, RBL + RBE, SHAKE
    "h2o_small": "res/json_files/H2O/rbmd.json",                   # 100 waters, RBL + RBE, SHAKE
    "eam_cu": "res/json_files/EAM/Cu/rbmd.json",                   # funcfl Cu_u3.eam, RBL
    "lj_inbuild": "res/json_files/LJ/rbmd.json",                   # BOM, comments, trailing comma
    "lj_coul_inbuild": "res/json_files/LJ/rbmd_lj.json",           # CVFF-typed LJ + RBE, inbuild
    "lj_salt_box": "res/json_files/LJ_salt/box_102030/rbmd.json",  # charged LJ data file, RBE
    "examples_h2o": "examples/H2O/rbmd.json",                      # water, EWALD
    "examples_ch4": "examples/CH4/rbmd.json",                      # methane, CVFF bonds + angles
    "examples_eam_cu": "examples/EAM/Cu/rbmd_new_Cu.json",         # funcfl Cu, Verlet list
}


def available():
    return os.path.isdir(os.path.join(REF_ROOT, "res", "json_files"))


# The older inputs under res/json_files give coulomb.kmax as a scalar; the reference's current
# Coulomb::Execute refuses that (hyperparameters/Coulomb.cpp:40, GetVectorValue), and so does the
# host.  stage(..., array_kmax=True) rewrites such a scalar as the three-entry array it stands for.
SCALAR_KMAX = re.compile(r'("kmax"\s*:\s*)(\d+)')


def has_scalar_kmax(rel):
    text = open(os.path.join(REF_ROOT, rel), encoding="utf-8-sig").read()
    return any(not ln.lstrip().startswith("//") and SCALAR_KMAX.search(ln) for ln in text.split("\n"))


def stage(rel, tmp_path, num_steps=None, array_kmax=False):
    """Copies the input's directory to tmp_path/in and returns the copied JSON path.  num_steps
    rewrites the step count of the copy, array_kmax a scalar kmax (text substitutions; the
    reference tree stays untouched)."""
    src = os.path.join(REF_ROOT, rel)
    dst_dir = os.path.join(str(tmp_path), "in")
    shutil.copytree(os.path.dirname(src), dst_dir)
    dst = os.path.join(dst_dir, os.path.basename(src))
    text = open(dst, encoding="utf-8-sig").read()
    if num_steps is not None:
        text, n = re.subn(r'("num_steps"\s*:\s*)\d+', r"\g<1>%d" % num_steps, text)
        assert n == 1
    if array_kmax:
        lines = text.split("\n")
        for k, ln in enumerate(lines):
            if not ln.lstrip().startswith("//"):
                lines[k] = SCALAR_KMAX.sub(lambda m: f"{m.group(1)}[{m.group(2)}, {m.group(2)}, {m.group(2)}]", ln)
        text = "\n".join(lines)
    with open(dst, "w", encoding="utf-8") as f:
        f.write(text)
    return dst


def dump(json_path):
    out = json_path + ".dump.json"
    r = subprocess.run([RBMD, "-j", os.path.basename(json_path), "--dump-system", out],
                       cwd=os.path.dirname(json_path), capture_output=True, text=True, timeout=300)
    return r, (json.load(open(out)) if r.returncode == 0 else None)


def resolve(rel, tmp_path, num_steps=None):
    path = stage(rel, tmp_path, num_steps, array_kmax=True)
    r, j = dump(path)
    assert r.returncode == 0, r.stdout + r.stderr
    return path, j


def data_header(json_dump_path_dir, data_name):
    """(atoms, types, box lo, box hi) from a LAMMPS data file header."""
    atoms = types = None
    lo, hi = [0.0] * 3, [0.0] * 3
    with open(os.path.join(json_dump_path_dir, data_name)) as f:
        for _ in range(60):
            ln = f.readline()
            if not ln:
                break
            w = ln.split()
            if len(w) >= 2 and w[1] == "atoms":
                atoms = int(w[0])
            elif len(w) >= 3 and w[1:3] == ["atom", "types"]:
                types = int(w[0])
            elif len(w) >= 4 and w[2:4] in (["xlo", "xhi"], ["ylo", "yhi"], ["zlo", "zhi"]):
                k = "xyz".index(w[2][0])
                lo[k], hi[k] = float(w[0]), float(w[1])
    return atoms, types, lo, hi


def _arr(j, key, dtype, shape=None):
    v = j.get(key)
    if v is None or len(v) == 0:
        return None
    a = np.ascontiguousarray(np.asarray(v, dtype=dtype))
    return a.reshape(shape) if shape else a


def load(j):
    """A resolved dump as SystemData (same arrays and parameters the host hands the library)."""
    P = j["params"]
    p = A.Params()
    for name, _ in A.Params._fields_:
        if name in P:
            v = P[name]
            cur = getattr(p, name)
            if hasattr(cur, "__len__"):
                cur[:] = v
            else:
                setattr(p, name, v)
    sd = synth.SystemData(_arr(j, "position", np.float64, (-1, 3)), _arr(j, "mass", np.float64),
                          _arr(j, "type", np.int32), _arr(j, "epsilon", np.float64), _arr(j, "sigma", np.float64),
                          j["box_lo"], j["box_hi"], vel=_arr(j, "velocity", np.float64, (-1, 3)),
                          charge=_arr(j, "charge", np.float64), molecule=_arr(j, "molecule", np.int32), params=p,
                          name=j.get("name", "reference_input"))
    if j.get("bond_atoms"):
        sd.bond_atoms = _arr(j, "bond_atoms", np.int32)
        sd.bond_type = _arr(j, "bond_type", np.int32)
        sd.bond_k = _arr(j, "bond_k", np.float64)
        sd.bond_r0 = _arr(j, "bond_r0", np.float64)
    if j.get("angle_atoms"):
        sd.angle_atoms = _arr(j, "angle_atoms", np.int32)
        sd.angle_type = _arr(j, "angle_type", np.int32)
        sd.angle_k = _arr(j, "angle_k", np.float64)
        sd.angle_theta0 = _arr(j, "angle_theta0", np.float64)
    if j.get("dihedral_atoms"):
        for k in ("dihedral_atoms", "dihedral_type", "dihedral_sign", "dihedral_multiplicity"):
            setattr(sd, k, _arr(j, k, np.int32))
        sd.dihedral_k = _arr(j, "dihedral_k", np.float64)
    if j.get("special_offsets"):
        sd.special_offsets = _arr(j, "special_offsets", np.int32)
        sd.special_ids = _arr(j, "special_ids", np.int32)
        sd.special_weights = _arr(j, "special_weights", np.float64)
    if j.get("near_table_values"):
        sd.near_table_values = _arr(j, "near_table_values", np.float32)
    e = j.get("eam") or {}
    if e.get("nrho"):
        sd.eam = dict(nrho=e["nrho"], nr=e["nr"], drho=e["drho"], dr=e["dr"], rhomax=e["rhomax"], cut=e["cut"],
                      per_type=e.get("per_type", 0), frho_spline=_arr(j, "eam_frho_spline", np.float64),
                      rhor_spline=_arr(j, "eam_rhor_spline", np.float64),
                      z2r_spline=_arr(j, "eam_z2r_spline", np.float64))
    return sd
