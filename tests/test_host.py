"""The `rbmd -j` host on the CPU: JSON dialect, LAMMPS data reading, special lists, inbuild lattice,
EAM potential files and error reporting, through `--dump-system` (which resolves the input and
writes it out without touching a GPU)."""
import json
import os
import subprocess

import numpy as np
import pytest

from rbmd_b200 import _abi as A
from rbmd_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RBMD = os.path.join(ROOT, "rbmd_b200", "_lib", "rbmd")


@pytest.fixture(scope="module")
def rbmd_bin():
    if not os.path.exists(RBMD):
        pytest.fail(f"{RBMD} is not built (python -m rbmd_b200.build)")
    return RBMD


def dump(rbmd_bin, json_path, tmp_path):
    out = tmp_path / "dump.json"
    r = subprocess.run([rbmd_bin, "-j", str(json_path), "--dump-system", str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return json.load(open(out))


def test_help_and_bad_arguments(rbmd_bin):
    r = subprocess.run([rbmd_bin, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "-j" in r.stdout
    r = subprocess.run([rbmd_bin, "-j", "input.txt"], capture_output=True, text=True)
    assert r.returncode == 1 and ".json" in r.stderr  # JsonParser.h: -j must name a .json file
    r = subprocess.run([rbmd_bin, "mpi", "-j", "x.json"], capture_output=True, text=True)
    assert r.returncode == 1 and "not built" in r.stderr


def test_json_dialect_and_inbuild(rbmd_bin, tmp_path):
    """BOM, // and /* */ comments and trailing commas as in the reference's bundled inputs; the
    inbuild lattice puts one atom at every cell centre, x fastest, charges -1 then +1."""
    text = "﻿" + """{
  // inbuild lattice
  "init_configuration": {
    "inbuild": { "dims": [ 4, 3, 2 ], "x_range": [ 0.0, 8.0 ], "y_range": [ 0.0, 6.0 ],
                 "z_range": [ 0.0, 4.0 ], "velocity_type": "ZERO", "unit": "LJ", },
  },
  /* block comment */
  "hyper_parameters": {
    "force_field": { "type": "LJ/CUT/COUL/LONG" },
    "neighbor": { "type": "RBL", "cut_off": 1.9, "r_core": 1.0, "neighbor_sample_num": 20, },
    "coulomb": { "type": "RBE", "coulomb_sample_num": 50, "alpha": 0.7, "kmax": [ 2, 2, 2 ] },
    "extend": { },
  },
  "execution": { "ensemble": "NVT", "temperature": [ 1.5, 1.5, 0.2 ], "temp_ctrl_type": "BERENDSEN",
                 "timestep": 0.002, "num_steps": 7, "seed": 11, },
  "outputs": { "thermo_out": { "interval": 2 } }
}
"""
    p = tmp_path / "in.json"
    p.write_text(text, encoding="utf-8")
    j = dump(rbmd_bin, p, tmp_path)
    assert j["n_atoms"] == 24 and j["init_way"] == "inbuild"
    P = j["params"]
    assert P["force_field"] == A.FF_LJ_CUT_COUL_LONG and P["coulomb"] == A.COUL_RBE
    assert P["kmax"] == [2, 2, 2] and P["coulomb_sample_num"] == 50 and P["alpha"] == 0.7
    assert P["temp_ctrl"] == A.TC_BERENDSEN and P["init_inbuild"] == 1 and P["num_steps"] == 7
    assert P["seed"] == 11 and P["fix_shake"] == A.SHAKE_NULL
    pos = np.array(j["position"]).reshape(-1, 3)
    assert np.allclose(pos[0], [1.0, 1.0, 1.0]) and np.allclose(pos[1], [3.0, 1.0, 1.0])
    assert np.allclose(pos[4], [1.0, 3.0, 1.0]) and np.allclose(pos[12], [1.0, 1.0, 3.0])
    q = np.array(j["charge"])
    assert (q[:12] == -1).all() and (q[12:] == 1).all()
    assert np.array(j["velocity"]).max() == 0.0
    assert j["outputs"]["thermo_interval"] == 2


@pytest.mark.parametrize("special", [True, False])
def test_read_data_water_full(rbmd_bin, tmp_path, special):
    sd = synth.spce_water(n_mol=64)
    if not special:
        sd.special_offsets = sd.special_ids = sd.special_weights = None
    path = synth.write_rbmd_input(sd, str(tmp_path))
    j = dump(rbmd_bin, path, tmp_path)
    assert j["n_atoms"] == sd.n and j["n_types"] == len(sd.eps)
    assert np.array_equal(np.array(j["position"]).reshape(-1, 3), sd.pos)
    assert np.array_equal(np.array(j["velocity"]).reshape(-1, 3), sd.vel)
    assert np.array_equal(j["charge"], sd.charge) and np.array_equal(j["mass"], sd.mass)
    assert np.array_equal(j["type"], sd.types) and np.array_equal(j["molecule"], sd.molecule)
    assert np.array_equal(j["bond_atoms"], sd.bond_atoms) and np.array_equal(j["bond_type"], sd.bond_type)
    assert np.array_equal(j["angle_atoms"], sd.angle_atoms) and np.array_equal(j["angle_type"], sd.angle_type)
    assert np.array_equal(j["bond_k"], sd.bond_k) and np.array_equal(j["angle_theta0"], sd.angle_theta0)
    assert np.array_equal(j["epsilon"], sd.eps) and np.array_equal(j["sigma"], sd.sig)
    assert j["box_lo"] == list(sd.box_lo) and j["box_hi"] == list(sd.box_hi)
    P = j["params"]
    assert P["force_field"] == A.FF_CVFF and P["fix_shake"] == A.SHAKE_TRUE and P["units"] == A.UNITS_REAL
    if special:  # the bond-graph lists, built in C++ from the Bonds section
        assert np.array_equal(j["special_offsets"], sd.special_offsets)
        assert np.array_equal(j["special_ids"], sd.special_ids)
        assert np.array_equal(j["special_weights"], sd.special_weights)
    else:
        assert j["special_offsets"] == []


def test_special_lists_match_reference_rule(rbmd_bin, tmp_path):
    """A chain and a branched molecule: 1-2, 1-3 and 1-4 partners in the multimap order of the
    bond list, an unbonded atom listing itself with weight 1 (SetSpecialBonds)."""
    pos = np.array([[1.0 + k, 2.0, 2.0] for k in range(7)])
    sd = synth.SystemData(pos, np.ones(7), np.zeros(7), [1.0], [1.0], [0, 0, 0], [12, 12, 12],
                          vel=np.zeros((7, 3)), charge=np.zeros(7), molecule=np.array([0, 0, 0, 0, 1, 1, 2]))
    sd.bond_atoms = np.array([0, 1, 1, 2, 2, 3, 4, 5], np.int32)
    sd.bond_type = np.zeros(4, np.int32)
    sd.bond_k, sd.bond_r0 = np.array([100.0]), np.array([1.0])
    w = (1.0, 0.0, 0.5)
    sd.special_offsets, sd.special_ids, sd.special_weights = synth.special_lists(
        7, [(0, 1), (1, 2), (2, 3), (4, 5)], w)
    sd.params.special_bonds[:] = [1, 0, 0]  # the reference reads the weights as integers
    path = synth.write_rbmd_input(sd, str(tmp_path), atom_style="full")
    j = dump(rbmd_bin, path, tmp_path)
    ref_off, ref_ids, ref_w = synth.special_lists(7, [(0, 1), (1, 2), (2, 3), (4, 5)], (1.0, 0.0, 0.0))
    assert np.array_equal(j["special_offsets"], ref_off)
    assert np.array_equal(j["special_ids"], ref_ids)
    assert np.array_equal(j["special_weights"], ref_w)
    off = j["special_offsets"]
    assert j["special_ids"][off[6]:off[7]] == [6] and j["special_weights"][off[6]] == 1.0


def test_eam_potential_file(rbmd_bin, tmp_path, oracle_mod):
    body = synth.johnson_funcfl(n=2000)
    pot = synth.write_funcfl(body, str(tmp_path / "cu.eam"))
    sd = synth.eam_cu(cells=3)
    path = synth.write_rbmd_input(sd, str(tmp_path), atom_style="atomic", potential_file="cu.eam")
    j = dump(rbmd_bin, path, tmp_path)
    ref = oracle_mod.eam_splines(oracle_mod.read_funcfl(pot))
    e = j["eam"]
    assert (e["nrho"], e["nr"]) == (ref["nrho"], ref["nr"])
    assert e["drho"] == ref["drho"] and e["dr"] == ref["dr"] and e["rhomax"] == ref["rhomax"]
    assert e["cut"] == ref["cut"]
    assert j["params"]["force_field"] == A.FF_EAM and j["params"]["units"] == A.UNITS_METAL


@pytest.mark.parametrize("mutate,message", [
    (lambda cfg: cfg["execution"].update(ensemble="NPT", temp_ctrl_type="NOSE_HOOVER", press_ctrl_type="BERENDSEN"),
     "both"),
    (lambda cfg: cfg["execution"].update(ensemble="NPT", temp_ctrl_type="TEMP_RESCALE"), "TEMP_RESCALE"),
    (lambda cfg: cfg["execution"].update(ensemble="NPT", temp_ctrl_type="BERENDSEN", press_ctrl_type="MTK"), "MTK"),
    (lambda cfg: cfg["init_configuration"]["read_data"].update(atom_style="molecular"), "atom_style"),
    (lambda cfg: cfg["init_configuration"]["read_data"].update(file="missing.data"), "missing.data"),
    (lambda cfg: cfg["hyper_parameters"]["force_field"].update(type="OPLS-AA"), "OPLS-AA"),
    # Coulomb::Execute reads kmax as an array (hyperparameters/Coulomb.cpp:40) and stops otherwise
    (lambda cfg: cfg["hyper_parameters"]["coulomb"].update(kmax=2), "kmax"),
    (lambda cfg: cfg["hyper_parameters"]["coulomb"].update(kmax=[2, 2]), "kmax"),
])
def test_errors_are_reported(rbmd_bin, tmp_path, mutate, message):
    sd = synth.spce_water(n_mol=8)
    path = synth.write_rbmd_input(sd, str(tmp_path))
    cfg = json.load(open(path))
    mutate(cfg)
    json.dump(cfg, open(path, "w"))
    r = subprocess.run([rbmd_bin, "-j", path, "--dump-system", str(tmp_path / "d.json")], capture_output=True,
                       text=True)
    assert r.returncode == 1 and message in r.stderr


@pytest.mark.parametrize("ctrl,pressure,bulk", [("BERENDSEN", [1.0, 2.0, 100.0], 10.0),
                                                ("BERENDSEN", [1.0, 2.0, 100.0, 25000.0], 25000.0),
                                                ("NOSE_HOOVER", [1.0, 1.0, 1000.0], 10.0)])
def test_npt_input(rbmd_bin, tmp_path, ctrl, pressure, bulk):
    """ensemble NPT with BERENDSEN or NOSE_HOOVER temperature and pressure control; the optional
    fourth pressure entry is the Berendsen bulk modulus (ExecutionNPT.cpp:953)."""
    sd = synth.spce_water(n_mol=8)
    path = synth.write_rbmd_input(sd, str(tmp_path))
    cfg = json.load(open(path))
    cfg["execution"].update(ensemble="NPT", temp_ctrl_type=ctrl, press_ctrl_type=ctrl, pressure=pressure)
    json.dump(cfg, open(path, "w"))
    P = dump(rbmd_bin, path, tmp_path)["params"]
    assert P["ensemble"] == A.ENS_NPT
    assert P["temp_ctrl"] == A.TEMP_CTRLS[ctrl] and P["press_ctrl"] == A.PRESS_CTRLS[ctrl]
    assert P["pressure"] == pressure[:3] and P["bulk_modulus"] == bulk


def test_truncated_data_file(rbmd_bin, tmp_path):
    sd = synth.spce_water(n_mol=8)
    path = synth.write_rbmd_input(sd, str(tmp_path))
    data = tmp_path / "rbmd.data"
    lines = data.read_text().splitlines()
    data.write_text("\n".join(lines[:lines.index("Velocities") - 3]) + "\n")
    r = subprocess.run([rbmd_bin, "-j", path, "--dump-system", str(tmp_path / "d.json")], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "Atoms" in r.stderr


def test_dihedrals_read_when_the_reference_uses_them(rbmd_bin, tmp_path):
    """Dihedral Coeffs / Dihedrals sections (ModelFileInitCondition.cpp:359-376, 551-585) reach the
    library only with special_bonds and dihedral_type "Harmonic" (ExecutionNVT.cpp:223-228)."""
    sd = synth.alkane_chains(n_side=2, length=6)
    path = synth.write_rbmd_input(sd, str(tmp_path), atom_style="full")
    j = dump(rbmd_bin, path, tmp_path)
    assert np.array_equal(j["dihedral_atoms"], sd.dihedral_atoms)
    assert np.array_equal(j["dihedral_type"], sd.dihedral_type)
    assert j["dihedral_k"] == list(sd.dihedral_k) and j["dihedral_multiplicity"] == list(sd.dihedral_multiplicity)
    assert j["dihedral_sign"] == list(sd.dihedral_sign)
    cfg = json.load(open(path))
    del cfg["hyper_parameters"]["extend"]["special_bonds"]  # no special bonds: no dihedral forces
    json.dump(cfg, open(path, "w"))
    assert dump(rbmd_bin, path, tmp_path)["dihedral_atoms"] == []
    cfg["hyper_parameters"]["extend"]["special_bonds"] = [0, 0, 0]
    cfg["hyper_parameters"]["force_field"]["dihedral_type"] = "Charmm"
    json.dump(cfg, open(path, "w"))
    r = subprocess.run([rbmd_bin, "-j", path, "--dump-system", str(tmp_path / "d.json")], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "Harmonic" in r.stderr


def test_observable_outputs_input(rbmd_bin, tmp_path):
    """msd_out / vacf_out / rdf_out keys of the reference's bundled inputs (MDApplication.cpp:221-235)."""
    sd = synth.spce_water(n_mol=8)
    path = synth.write_rbmd_input(sd, str(tmp_path))
    cfg = json.load(open(path))
    cfg["outputs"].update(
        msd_out={"interval": 10, "start_step": 0, "end_step": 10000},
        vacf_out={"start_step": 5, "end_step": 50},
        rdf_out={"interval": 10, "radius": 10, "dr": 0.1, "statistics_rdf_steps": 1000, "atoms_pair": [[0, 0], [0, 1]]})
    json.dump(cfg, open(path, "w"))
    o = dump(rbmd_bin, path, tmp_path)["outputs"]
    assert o["msd"] == {"interval": 10, "start_step": 0, "end_step": 10000}
    assert o["vacf"] == {"interval": 1, "start_step": 5, "end_step": 50}
    assert o["rdf"] == {"radius": 10, "dr": 0.1, "statistics_rdf_steps": 1000, "atoms_pair": [[0, 0], [0, 1]]}


@pytest.mark.parametrize("outputs,message", [
    ({"msd_out": {"interval": 10, "end_step": 100}}, "start_step"),
    ({"rdf_out": {"radius": 10, "dr": 0.1, "statistics_rdf_steps": 10}}, "atoms_pair"),
    ({"rdf_out": {"radius": 10, "dr": 0.1, "statistics_rdf_steps": 10, "atoms_pair": [[0, 2]]}}, "out of range"),
    ({"rdf_out": {"radius": 10, "dr": 0.1, "statistics_rdf_steps": 10, "atoms_pair": [0, 1]}}, "atoms_pair"),
    ({"rdf_out": {"radius": 0.05, "dr": 0.1, "statistics_rdf_steps": 10, "atoms_pair": [[0, 1]]}}, "radius"),
])
def test_observable_output_errors(rbmd_bin, tmp_path, outputs, message):
    sd = synth.spce_water(n_mol=8)
    path = synth.write_rbmd_input(sd, str(tmp_path))
    cfg = json.load(open(path))
    cfg["outputs"].update(outputs)
    json.dump(cfg, open(path, "w"))
    r = subprocess.run([rbmd_bin, "-j", path, "--dump-system", str(tmp_path / "d.json")], capture_output=True,
                       text=True)
    assert r.returncode == 1 and message in r.stderr, r.stderr


def test_checkpoint_and_trajectory_input(rbmd_bin, tmp_path):
    """trajectory_out defaults to every step (TrajectoryOutput.cpp:36); checkpoint_out (no reference
    counterpart) takes an interval and a file name."""
    sd = synth.spce_water(n_mol=8)
    path = synth.write_rbmd_input(sd, str(tmp_path))
    cfg = json.load(open(path))
    cfg["outputs"].update(trajectory_out={}, checkpoint_out={"interval": 50, "file": "x.data"})
    json.dump(cfg, open(path, "w"))
    o = dump(rbmd_bin, path, tmp_path)["outputs"]
    assert o["trajectory_interval"] == 1 and o["checkpoint_interval"] == 50 and o["checkpoint_file"] == "x.data"


@pytest.mark.parametrize("how", ["extension", "format_key", "elements"])
def test_setfl_potential_file(rbmd_bin, tmp_path, oracle_mod, how):
    """setfl (eam/alloy) potentials: per-type tables equal to the oracle's restatement; atom types
    map to the file's elements in order, or by force_field.elements."""
    body = synth.johnson_setfl(n=600)
    name = {"extension": "ab.eam.alloy", "format_key": "ab.pot", "elements": "ab.eam.alloy"}[how]
    synth.write_setfl(body, str(tmp_path / name))
    sd = synth.eam_alloy(cells=2)
    path = synth.write_rbmd_input(sd, str(tmp_path), atom_style="atomic", potential_file=name)
    cfg = json.load(open(path))
    te = [0, 1]
    if how == "format_key":
        cfg["hyper_parameters"]["force_field"]["potential_format"] = "setfl"
    if how == "elements":
        cfg["hyper_parameters"]["force_field"]["elements"] = ["B", "Cu"]
        te = [1, 0]
    json.dump(cfg, open(path, "w"))
    j = dump(rbmd_bin, path, tmp_path)
    ref = oracle_mod.setfl_splines(body, te)
    e = j["eam"]
    assert e["per_type"] == 1 and (e["nrho"], e["nr"]) == (ref["nrho"], ref["nr"])
    assert e["rhomax"] == ref["rhomax"] and e["cut"] == ref["cut"]
    for k in ("frho_spline", "rhor_spline", "z2r_spline"):
        assert np.array_equal(np.array(j["eam_" + k]), ref[k]), k


def test_setfl_errors(rbmd_bin, tmp_path):
    body = synth.johnson_setfl(n=600)
    synth.write_setfl(body, str(tmp_path / "ab.eam.alloy"))
    sd = synth.eam_alloy(cells=2)
    path = synth.write_rbmd_input(sd, str(tmp_path), atom_style="atomic", potential_file="ab.eam.alloy")
    cfg = json.load(open(path))
    for ff, msg in (({"elements": ["Cu", "Zr"]}, "Zr"), ({"elements": ["Cu"]}, "one element name per atom type"),
                    ({"potential_format": "tabulated"}, "potential_format")):
        c = json.loads(json.dumps(cfg))
        c["hyper_parameters"]["force_field"].update(ff)
        json.dump(c, open(path, "w"))
        r = subprocess.run([rbmd_bin, "-j", path, "--dump-system", str(tmp_path / "d.json")], capture_output=True,
                           text=True)
        assert r.returncode == 1 and msg in r.stderr, r.stderr
