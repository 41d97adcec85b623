"""Harmonic dihedrals (CVFF with special bonds and a Dihedrals section) on the sm_100a path against
the FP64 oracle: forces in every pair layout, the one-step thermo with its dihedral energy and
virial, mixed precision, and the rbmd host's energy.rbmd column."""
import os
import subprocess

import numpy as np
import pytest

from rbmd_b200 import _abi as A
from rbmd_b200 import synth

from conftest import rel_rms
from test_gpu_parity import LAYOUTS, pair

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def chains(**kw):
    sd = synth.alkane_chains(n_side=6, length=6, **kw)
    sd.params.precision = A.PREC_FP64
    return sd


CASES = {
    "rbe_rbl": lambda: chains(),
    "ewald_verlet": lambda: chains(coulomb=A.COUL_EWALD, neighbor=A.NEIGH_VERLET, kmax=(4, 4, 4)),
}


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("case", list(CASES))
def test_forces_with_dihedrals(ctx_factory, oracle_mod, case, layout):
    sd = CASES[case]()
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd, layout=layout)
    ctx.compute_forces(sid)
    o.compute_forces()
    assert rel_rms(ctx.forces(sid), o.forces()) < 1e-6


@pytest.mark.parametrize("case", list(CASES))
def test_one_step_thermo_with_dihedrals(ctx_factory, oracle_mod, case):
    sd = CASES[case]()
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd, graphs=False)
    ctx.init(sid)
    o.init()
    ctx.step(sid, 1)
    o.step(1)
    tg, to = ctx.thermo(sid), o.thermo()
    assert to["e_dihedral"] > 0
    for key in ("e_dihedral", "e_bond", "e_angle", "potential_energy", "total_energy", "temperature"):
        assert tg[key] == pytest.approx(to[key], rel=1e-7, abs=1e-9), key
    assert tg["pressure"] == pytest.approx(to["pressure"], rel=1e-6, abs=1e-6)
    x, v, _ = ctx.state(sid)
    ox, ov, _ = o.state()
    assert rel_rms(x, ox) < 1e-10 and rel_rms(v, ov) < 1e-7


def test_mixed_precision_with_dihedrals(ctx_factory, oracle_mod):
    sd = chains()
    sd.params.precision = A.PREC_MIXED
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd)
    ctx.compute_forces(sid)
    o.compute_forces()
    assert rel_rms(ctx.forces(sid), o.forces()) < 1e-3


def test_host_writes_dihedral_energy(tmp_path):
    sd = chains()
    sd.params.num_steps = 3
    path = synth.write_rbmd_input(sd, str(tmp_path), atom_style="full")
    r = subprocess.run([os.path.join(ROOT, "rbmd_b200", "_lib", "rbmd"), "cuda", "-j", path], cwd=str(tmp_path),
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = open(os.path.join(str(tmp_path), "energy.rbmd")).read().split("\n")
    cols = lines[0].split()
    rows = [dict(zip(cols, map(float, ln.split()))) for ln in lines[1:] if ln.strip()]
    assert len(rows) == 4 and all(r["DihedralEnergy"] > 0 for r in rows)
