"""setfl (eam/alloy) EAM on the sm_100a path against the FP64 oracle: per-type densities, embedding
functions and pair tables in every pair layout and both neighbour modes, dynamics and thermo, mixed
precision, and the rbmd host reading a setfl file."""
import json
import os
import subprocess

import numpy as np
import pytest

import rbmd_b200
from rbmd_b200 import _abi as A
from rbmd_b200 import synth

from conftest import rel_rms
from test_gpu_parity import LAYOUTS, pair

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RBMD = os.path.join(ROOT, "rbmd_b200", "_lib", "rbmd")


def alloy(oracle_mod, **kw):
    sd = synth.eam_alloy(cells=6, frac_b=0.35, build_splines=oracle_mod.setfl_splines, **kw)
    rng = np.random.default_rng(4)
    sd.pos = sd.pos + rng.normal(scale=0.05, size=sd.pos.shape)
    return sd


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("neigh", ["rbl", "verlet"])
def test_alloy_forces(ctx_factory, oracle_mod, layout, neigh):
    kw = {} if neigh == "rbl" else dict(neighbor=A.NEIGH_VERLET, r_core=5.0)
    sd = alloy(oracle_mod, **kw)
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd, layout=layout)
    ctx.compute_forces(sid)
    o.compute_forces()
    assert rel_rms(ctx.forces(sid), o.forces()) < 1e-9


def test_alloy_dynamics_and_thermo(ctx_factory, oracle_mod):
    sd = alloy(oracle_mod)
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd, graphs=False)
    ctx.init(sid)
    o.init()
    for n in (1, 9):
        ctx.step(sid, n)
        o.step(n)
        tg, to = ctx.thermo(sid), o.thermo()
        for key in ("e_eam", "potential_energy", "total_energy", "temperature"):
            assert tg[key] == pytest.approx(to[key], rel=1e-9, abs=1e-12), key
    x, v, _ = ctx.state(sid)
    ox, ov, _ = o.state()
    assert rel_rms(x, ox) < 1e-12 and rel_rms(v, ov) < 1e-9


def test_alloy_mixed_precision(ctx_factory, oracle_mod):
    sd = alloy(oracle_mod, precision=A.PREC_MIXED)
    ref = sd.copy()
    ref.params.precision = A.PREC_FP64
    ctx, sid, _ = pair(ctx_factory, oracle_mod, sd)
    o = oracle_mod.Oracle(ref)
    ctx.compute_forces(sid)
    o.compute_forces()
    assert rel_rms(ctx.forces(sid), o.forces()) < 1e-4


def test_host_reads_setfl(tmp_path, oracle_mod):
    body = synth.johnson_setfl(n=2000)
    synth.write_setfl(body, str(tmp_path / "ab.eam.alloy"))
    sd = synth.eam_alloy(cells=5, frac_b=0.35, build_splines=rbmd_b200.setfl_splines)
    sd.eam = rbmd_b200.setfl_splines(body, [0, 1])
    sd.params.num_steps = 5
    path = synth.write_rbmd_input(sd, str(tmp_path), atom_style="atomic", potential_file="ab.eam.alloy")
    r = subprocess.run([RBMD, "cuda", "-j", path], cwd=str(tmp_path), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [ln.split() for ln in open(tmp_path / "energy.rbmd").read().split("\n") if ln.strip()]
    head, rows = lines[0], np.array([[float(t) for t in ln] for ln in lines[1:]])
    ctx = rbmd_b200.Context(batched=False)
    sid = ctx.add_system(sd)
    ctx.init(sid)
    for s in range(6):
        t = ctx.thermo(sid)
        assert rows[s, head.index("VanderWaalsEnergy")] == pytest.approx(t["e_eam"], rel=1e-8)
        assert rows[s, head.index("TotalEnergy")] == pytest.approx(t["total_energy"], rel=1e-8)
        ctx.step(sid, 1)
    ctx.close()
