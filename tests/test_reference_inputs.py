"""The reference's bundled inputs through the `rbmd -j` host on the CPU.

Every rbmd.json the reference ships with all its files in the tree is resolved by the host
(`--dump-system`: JSON dialect with BOM, comments and trailing commas, LAMMPS data files,
funcfl potentials, inbuild lattices) and checked against what the input says -- atom and type
counts and box from the data file header, the numbers of the JSON itself -- and then stepped by the
FP64 oracle.  The older inputs under res/json_files give kmax as a scalar, which the reference
refuses (hyperparameters/Coulomb.cpp:40 reads it with GetVectorValue); so does the host, and they
are read here with the scalar written as the array it stands for.
Skipped where the reference tree is absent.
"""
import json
import os
import re
import subprocess

import numpy as np
import pytest

import refinputs as R
from rbmd_b200 import _abi as A

pytestmark = pytest.mark.skipif(not R.available(), reason="reference tree not present")


def _json_text(path):
    """The input's JSON as Python data: comments and trailing commas removed (the reference's
    jsoncpp accepts both)."""
    text = open(path, encoding="utf-8-sig").read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    text = re.sub(r",(\s*[}\]])", r"\1", text)
    return json.loads(text)


@pytest.mark.parametrize("name", sorted(R.INPUTS))
def test_reference_input_resolves(name, tmp_path, oracle_mod):
    path, j = R.resolve(R.INPUTS[name], tmp_path)
    cfg = _json_text(path)
    ic = cfg["init_configuration"]
    if "read_data" in ic:
        atoms, types, lo, hi = R.data_header(os.path.dirname(path), ic["read_data"]["file"])
        assert j["n_atoms"] == atoms and j["n_types"] == types
        assert np.allclose(j["box_lo"], lo) and np.allclose(j["box_hi"], hi)
    else:
        dims = ic["inbuild"]["dims"]
        assert j["n_atoms"] == dims[0] * dims[1] * dims[2]
        assert np.allclose(j["box_lo"], [ic["inbuild"][k][0] for k in ("x_range", "y_range", "z_range")])
    P = j["params"]
    hp = cfg["hyper_parameters"]
    nb = hp.get("neighbor", {})
    assert P["cut_off"] == pytest.approx(nb["cut_off"])
    if nb.get("type") == "RBL":
        assert P["neighbor"] == A.NEIGH_RBL
        assert P["r_core"] == pytest.approx(nb["r_core"]) and P["neighbor_sample_num"] == nb["neighbor_sample_num"]
    if "coulomb" in hp:
        cl = hp["coulomb"]
        assert P["coulomb"] == A.COULOMBS[cl["type"]]
        assert P["alpha"] == pytest.approx(cl["alpha"]) and P["kmax"] == list(cl["kmax"])
        if cl["type"] == "RBE":
            assert P["coulomb_sample_num"] == cl["coulomb_sample_num"]
    ex = cfg["execution"]
    assert P["timestep"] == pytest.approx(ex["timestep"]) and P["num_steps"] == ex["num_steps"]
    assert P["temperature"] == pytest.approx(ex["temperature"])
    assert P["temp_ctrl"] == A.TEMP_CTRLS[ex["temp_ctrl_type"]]
    sd = R.load(j)
    o = oracle_mod.Oracle(sd)
    o.init()
    o.step(3)
    x, v, _ = o.state()
    th = o.thermo()
    assert th["status"] == 0 and np.isfinite(x).all() and np.isfinite(v).all()
    assert np.isfinite(th["total_energy"])


@pytest.mark.parametrize("name", sorted(k for k, v in R.INPUTS.items() if R.available() and R.has_scalar_kmax(v)) +
                         ["lj_salt_inbuild"])
def test_scalar_kmax_is_refused(name, tmp_path):
    """The inputs that give kmax as a scalar stop with a message, unmodified, as in the reference;
    the other tests read them with the scalar written as [k, k, k]."""
    rel = R.INPUTS.get(name, "res/json_files/LJ_salt/rbmd.json")
    path = R.stage(rel, tmp_path)
    r, j = R.dump(path)
    assert r.returncode == 1 and j is None
    assert "kmax" in r.stderr
