"""Parity with the FP64 oracle at the benchmark configurations' own sizes.

The other parity tests run shrunken systems; cell occupancy and stencil layout depend on the box,
so the five workloads are checked here at the sizes they are defined with:

  lj4000      LJ fluid, fcc 10^3 x 4 at rho* 0.8442, RBL r_core 1.2, 100 shell samples (nc 3, 20^3 cells)
  nacl8000    rock-salt melt, 20^3 ions at rho* 0.6, RBE alpha 0.6 with P = 200
  water9000   SPC/E, 3000 molecules, RBE beta 0.3 with P = 100, rc 10 / r_core 5 (8^3 cells), SHAKE
  eam32000    fcc Cu 20^3 x 4, Johnson funcfl tables of 10000 points to 5 A (28^3 cells)
  saline64k   one 64k-atom system of the serving stream (SPC/E + 0.15 M NaCl)

Each is checked at its lattice start and after ten FP64 steps: cell tables, RBL lists and RBE
samples bit-exact; FP64 forces within relative RMS 1e-6; mixed forces within the 1e-3 bar (and
below 1e-4, the level at which a single different RBL pick would show); ten steps of dynamics and
the thermo quantities against the oracle.  Force errors are relative to ||F||, or at a lattice
start (where the forces cancel by symmetry) to the ||F|| the system reaches ten steps later.
"""
import numpy as np
import pytest

from rbmd_b200 import _abi as A
from rbmd_b200 import synth

from conftest import rel_rms

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-6
MIXED_TOL = 1e-3
PICK_TOL = 1e-4   # one RBL pick different from the FP64 one moves the force by ~1e-3 or more
CAP = 256         # list row capacity: at most ~170 selected pairs per atom in these systems


def _config(name, oracle_mod):
    if name == "lj4000":
        return synth.lj_fcc()
    if name == "nacl8000":
        return synth.nacl_melt()
    if name == "water9000":
        return synth.spce_water()
    if name == "eam32000":
        return synth.eam_cu(build_splines=oracle_mod.eam_splines)
    if name == "saline64k":
        return synth.saline(64000, seed=5)
    raise KeyError(name)


CONFIGS = ["lj4000", "nacl8000", "water9000", "eam32000", "saline64k"]
RBE_CONFIGS = ["nacl8000", "water9000", "saline64k"]

_cache = {}


def _advanced(name, oracle_mod):
    """The configuration after ten FP64 oracle steps (lattice starts melt a little), cached."""
    if name not in _cache:
        sd = _config(name, oracle_mod)
        sd.params.precision = A.PREC_FP64
        o = oracle_mod.Oracle(sd)
        o.init()
        o.step(10)
        x, v, img = o.state()
        sd2 = sd.copy()
        sd2.pos = np.ascontiguousarray(x)
        sd2.vel = np.ascontiguousarray(v)
        sd2.image = np.ascontiguousarray(img, np.int32)
        _cache[name] = (sd2, o.thermo()["step"])
    sd2, step = _cache[name]
    return sd2.copy(), step


def _force_norm(name, oracle_mod):
    """||F|| of the configuration after ten steps: the force scale of the system.  At a perfect
    lattice start the forces cancel by symmetry (to round-off, plus the RBE noise), so errors there
    are measured against this scale instead of the vanishing ||F|| of the start."""
    key = ("norm", name)
    if key not in _cache:
        sd, step = _advanced(name, oracle_mod)
        sd.params.precision = A.PREC_FP64
        o = oracle_mod.Oracle(sd)
        o.set_step(step)
        o.compute_forces()
        _cache[key] = float(np.sqrt((o.forces() ** 2).sum()))
    return _cache[key]


def _err(f, fo, name, oracle_mod):
    return float(np.sqrt(((f - fo) ** 2).sum()) / max(np.sqrt((fo ** 2).sum()), _force_norm(name, oracle_mod)))


def _system(name, oracle_mod, state):
    if state == "start":
        return _config(name, oracle_mod), 0
    return _advanced(name, oracle_mod)


def _pair(ctx_factory, oracle_mod, sd, step, layout="auto"):
    import os
    ctx = ctx_factory()
    old = os.environ.get("RBMD_PAIR_LAYOUT")
    os.environ["RBMD_PAIR_LAYOUT"] = layout
    try:
        sid = ctx.add_system(sd)
    finally:
        if old is None:
            os.environ.pop("RBMD_PAIR_LAYOUT", None)
        else:
            os.environ["RBMD_PAIR_LAYOUT"] = old
    o = oracle_mod.Oracle(sd)
    if step:
        ctx.set_step(sid, step)
        o.set_step(step)
    return ctx, sid, o


def _tile_ok(sd):
    return all(2 * sd.params.cut_off <= h - lo for h, lo in zip(sd.box_hi, sd.box_lo))


def _lists_equal(g, o):
    gn, gs, gi = g
    on, os_, oi = o
    assert np.array_equal(gn, on), "core counts differ"
    assert np.array_equal(gs, os_), "shell counts differ"
    k = (gn + gs)[:, None]
    mask = np.arange(gi.shape[1])[None, :] < k
    bad = np.nonzero((np.where(mask, gi, -1) != np.where(mask, oi, -1)).any(1))[0]
    assert bad.size == 0, f"{bad.size} list rows differ, first atom {bad[:5]}"


@pytest.mark.parametrize("state", ["start", "advanced"])
@pytest.mark.parametrize("name", CONFIGS)
def test_full_cells_bit_exact(ctx_factory, oracle_mod, name, state):
    sd, step = _system(name, oracle_mod, state)
    ctx, sid, o = _pair(ctx_factory, oracle_mod, sd, step)
    for a, b in zip(ctx.cells(sid), o.cells()):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("layout", ["lean", "cell"])
@pytest.mark.parametrize("state", ["start", "advanced"])
@pytest.mark.parametrize("name", CONFIGS)
def test_full_rbl_lists_bit_exact(ctx_factory, oracle_mod, name, state, layout):
    sd, step = _system(name, oracle_mod, state)
    ctx, sid, o = _pair(ctx_factory, oracle_mod, sd, step, layout=layout)
    _lists_equal(ctx.rbl_lists(sid, cap=CAP), o.rbl_lists(cap=CAP))


@pytest.mark.parametrize("name", RBE_CONFIGS)
def test_full_rbe_samples_bit_exact(ctx_factory, oracle_mod, name):
    sd, step = _system(name, oracle_mod, "advanced")
    ctx, sid, o = _pair(ctx_factory, oracle_mod, sd, step)
    ctx.compute_forces(sid)
    o.compute_forces()
    m, rk = ctx.kspace(sid)
    om, ork = o.kspace()
    assert np.array_equal(m, om)
    assert rel_rms(rk, ork) < 1e-12


@pytest.mark.parametrize("layout", ["auto", "lean", "cell"])
@pytest.mark.parametrize("state", ["start", "advanced"])
@pytest.mark.parametrize("name", CONFIGS)
def test_full_forces_fp64(ctx_factory, oracle_mod, name, state, layout):
    sd, step = _system(name, oracle_mod, state)
    sd.params.precision = A.PREC_FP64
    ctx, sid, o = _pair(ctx_factory, oracle_mod, sd, step, layout=layout)
    ctx.compute_forces(sid)
    o.compute_forces()
    err = _err(ctx.forces(sid), o.forces(), name, oracle_mod)
    assert err < FP64_TOL, err


@pytest.mark.parametrize("layout", ["auto", "lean", "cell", "column"])
@pytest.mark.parametrize("state", ["start", "advanced"])
@pytest.mark.parametrize("name", CONFIGS)
def test_full_forces_mixed(ctx_factory, oracle_mod, name, state, layout):
    sd, step = _system(name, oracle_mod, state)
    if layout in ("cell", "column") and not _tile_ok(sd):
        pytest.skip("the tile layout needs edges of at least 2 rc")
    sd.params.precision = A.PREC_MIXED
    ctx, sid, o = _pair(ctx_factory, oracle_mod, sd, step, layout=layout)
    ref = sd.copy()
    ref.params.precision = A.PREC_FP64
    o = oracle_mod.Oracle(ref)
    if step:
        o.set_step(step)
    ctx.compute_forces(sid)
    o.compute_forces()
    err = _err(ctx.forces(sid), o.forces(), name, oracle_mod)
    assert err < MIXED_TOL, err
    assert err < PICK_TOL, f"{err}: above the FP32 arithmetic level (an RBL pick differs?)"


@pytest.mark.parametrize("name", CONFIGS)
def test_full_ten_steps_and_thermo(ctx_factory, oracle_mod, name):
    sd = _config(name, oracle_mod)
    sd.params.precision = A.PREC_FP64
    ctx, sid, o = _pair(ctx_factory, oracle_mod, sd, 0)
    ctx.init(sid)
    o.init()
    ctx.step(sid, 10)
    o.step(10)
    x, v, img = ctx.state(sid)
    ox, ov, oimg = o.state()
    assert rel_rms(x, ox) < 1e-9
    assert rel_rms(v, ov) < 1e-6
    assert np.array_equal(img, oimg)
    tg, to = ctx.thermo(sid), o.thermo()
    assert tg["step"] == to["step"] == 10
    assert tg["status"] == 0
    for key in ("temperature", "kinetic_energy", "e_lj", "e_coul_near", "e_coul_far", "e_bond", "e_angle",
                "e_eam", "total_energy"):
        assert tg[key] == pytest.approx(to[key], rel=1e-6, abs=1e-8), key
    assert tg["pressure"] == pytest.approx(to["pressure"], rel=1e-5, abs=1e-6)
