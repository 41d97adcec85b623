"""`rbmd cuda -j input.json` end to end: the host reads the reference-style inputs, drives the
library through the C ABI and writes energy.rbmd; every row must match the Python API's thermo of
the same system after the same number of steps (energy.rbmd prints 10 significant digits)."""
import os
import subprocess

import numpy as np
import pytest

import rbmd_b200
from rbmd_b200 import _abi as A
from rbmd_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RBMD = os.path.join(ROOT, "rbmd_b200", "_lib", "rbmd")
COLS = ["Step", "Time", "VanderWaalsEnergy", "NearCoulombicEnergy", "FarCoulombicEnergy", "KinticEnergy",
        "PotentialEnergy", "TotalEnergy", "BondEnergy", "AngleEnergy", "DihedralEnergy", "Temperature", "Pressure"]


def _run_host(json_path, cwd):
    r = subprocess.run([RBMD, "cuda", "-j", json_path], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = open(os.path.join(cwd, "energy.rbmd")).read().split("\n")
    assert lines[0].split() == COLS
    return [dict(zip(COLS, map(float, ln.split()))) for ln in lines[1:] if ln.strip()]


def _api_thermo(sd, nsteps):
    ctx = rbmd_b200.Context()
    sid = ctx.add_system(sd)
    ctx.init(sid)
    out = [ctx.thermo(sid)]
    for _ in range(nsteps):
        ctx.step(sid, 1)
        out.append(ctx.thermo(sid))
    ctx.close()
    return out


def _compare(rows, api):
    assert [int(r["Step"]) for r in rows] == list(range(len(api)))
    for r, t in zip(rows, api):
        assert r["TotalEnergy"] == pytest.approx(t["total_energy"], rel=1e-8, abs=1e-9)
        assert r["PotentialEnergy"] == pytest.approx(t["potential_energy"], rel=1e-8, abs=1e-9)
        assert r["Temperature"] == pytest.approx(t["temperature"], rel=1e-8, abs=1e-9)
        assert r["BondEnergy"] == pytest.approx(t["e_bond"], rel=1e-8, abs=1e-9)


def test_host_water_cvff_rbe_matches_api(tmp_path):
    sd = synth.spce_water(n_mol=300, seed=8)
    sd.params.precision = A.PREC_FP64
    sd.params.num_steps = 4
    path = synth.write_rbmd_input(sd, str(tmp_path))
    rows = _run_host(path, str(tmp_path))
    # the executioner runs num_steps + 1 steps with the thermo output before each (Executioner.cpp)
    assert len(rows) == 5
    _compare(rows, _api_thermo(sd, 4))


def test_host_eam_funcfl_matches_api(tmp_path):
    body = synth.johnson_funcfl(n=2000)
    synth.write_funcfl(body, str(tmp_path / "cu.eam"))
    sd = synth.eam_cu(cells=5, build_splines=rbmd_b200.eam_splines)
    sd.params.precision = A.PREC_FP64
    sd.params.num_steps = 3
    sd.eam = rbmd_b200.eam_splines(body)
    path = synth.write_rbmd_input(sd, str(tmp_path), atom_style="atomic", potential_file="cu.eam")
    rows = _run_host(path, str(tmp_path))
    api = _api_thermo(sd, 3)
    assert [int(r["Step"]) for r in rows] == [0, 1, 2, 3]
    for r, t in zip(rows, api):
        assert r["VanderWaalsEnergy"] == pytest.approx(t["e_eam"], rel=1e-8, abs=1e-9)
        assert r["TotalEnergy"] == pytest.approx(t["total_energy"], rel=1e-8, abs=1e-9)


def test_host_reports_device_errors(tmp_path):
    """A system the library refuses (r_core above cut_off) ends the run with status 1 and the
    library's message, not a crash."""
    sd = synth.lj_fcc(cells=4)
    sd.params.r_core = 9.0
    path = synth.write_rbmd_input(sd, str(tmp_path))
    r = subprocess.run([RBMD, "cuda", "-j", path], cwd=str(tmp_path), capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "rbmd_system_add" in r.stderr
