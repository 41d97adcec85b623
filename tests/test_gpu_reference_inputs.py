"""The reference's bundled inputs on the GPU, against the FP64 oracle.

Each input the reference ships with all its files (see refinputs.INPUTS) is resolved by the `rbmd`
host (`--dump-system`) and run through the C ABI: FP64 forces within relative RMS 1e-6 of the
oracle, mixed precision within 1e-3, five steps of dynamics tracking it, and `rbmd cuda -j` itself
(five steps, outputs into a scratch copy of the input's directory) writing the energy.rbmd rows
the API's thermo gives.  Skipped where the reference tree is absent (RBMD_REFERENCE_ROOT names a
copy of it).
"""
import os
import subprocess

import numpy as np
import pytest

import refinputs as R
from rbmd_b200 import _abi as A

from conftest import rel_rms

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="reference tree not present")]

COLS = ["Step", "Time", "VanderWaalsEnergy", "NearCoulombicEnergy", "FarCoulombicEnergy", "KinticEnergy",
        "PotentialEnergy", "TotalEnergy", "BondEnergy", "AngleEnergy", "DihedralEnergy", "Temperature", "Pressure"]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(R.INPUTS))
def test_reference_input_forces(ctx_factory, oracle_mod, name, prec, tmp_path):
    _, j = R.resolve(R.INPUTS[name], tmp_path)
    sd = R.load(j)
    sd.params.precision = A.PREC_FP64 if prec == "fp64" else A.PREC_MIXED
    ctx = ctx_factory()
    sid = ctx.add_system(sd)
    ref = sd.copy()
    ref.params.precision = A.PREC_FP64
    o = oracle_mod.Oracle(ref)
    ctx.compute_forces(sid)
    o.compute_forces()
    err = rel_rms(ctx.forces(sid), o.forces())
    assert err < (1e-6 if prec == "fp64" else 1e-3), err


@pytest.mark.parametrize("name", sorted(R.INPUTS))
def test_reference_input_steps(ctx_factory, oracle_mod, name, tmp_path):
    _, j = R.resolve(R.INPUTS[name], tmp_path)
    sd = R.load(j)
    sd.params.precision = A.PREC_FP64
    ctx = ctx_factory()
    sid = ctx.add_system(sd)
    o = oracle_mod.Oracle(sd)
    ctx.init(sid)
    o.init()
    ctx.step(sid, 5)
    o.step(5)
    x, v, img = ctx.state(sid)
    ox, ov, oimg = o.state()
    assert rel_rms(x, ox) < 1e-9
    assert rel_rms(v, ov) < 1e-6
    assert np.array_equal(img, oimg)
    tg, to = ctx.thermo(sid), o.thermo()
    assert tg["status"] == 0
    for key in ("temperature", "e_lj", "e_coul_near", "e_coul_far", "e_bond", "e_angle", "e_eam", "total_energy"):
        assert tg[key] == pytest.approx(to[key], rel=1e-6, abs=1e-8), key


@pytest.mark.parametrize("name", ["h2o_box_305038", "eam_cu", "examples_ch4", "lj_inbuild"])
def test_reference_input_through_rbmd_cuda(ctx_factory, name, tmp_path):
    path, j = R.resolve(R.INPUTS[name], tmp_path, num_steps=5)
    cwd = os.path.dirname(path)
    r = subprocess.run([R.RBMD, "cuda", "-j", os.path.basename(path)], cwd=cwd, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [ln for ln in open(os.path.join(cwd, "energy.rbmd")).read().split("\n") if ln.strip()]
    assert lines[0].split() == COLS
    rows = [dict(zip(COLS, map(float, ln.split()))) for ln in lines[1:]]
    sd = R.load(j)
    ctx = ctx_factory()
    sid = ctx.add_system(sd)
    ctx.init(sid)
    api = [ctx.thermo(sid)]
    for _ in range(5):
        ctx.step(sid, 1)
        api.append(ctx.thermo(sid))
    assert [int(rw["Step"]) for rw in rows] == list(range(len(api)))
    for rw, t in zip(rows, api):
        assert rw["TotalEnergy"] == pytest.approx(t["total_energy"], rel=1e-8, abs=1e-9)
        assert rw["Temperature"] == pytest.approx(t["temperature"], rel=1e-8, abs=1e-9)
