"""The pair-layout autotuner (rbmd_autotune) on the GPU: it times every usable layout per group,
keeps the fastest, leaves the state as it was, caches its decision by group signature, and the
forces after tuning still match the FP64 oracle."""
import numpy as np
import pytest

from rbmd_b200 import _abi as A
from rbmd_b200 import synth

from conftest import rel_rms

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-3


def _saline(n, seed):
    sd = synth.saline(n, seed=seed)
    sd.params.seed = 100 + seed
    return sd


def test_autotune_picks_the_fastest_and_keeps_state(ctx_factory, oracle_mod):
    systems = [_saline(4000, s) for s in (1, 2, 3)] + [synth.lj_fcc(cells=8, precision=A.PREC_MIXED)]
    ctx = ctx_factory()
    ids = [ctx.add_system(sd) for sd in systems]
    ctx.init(ids)
    ctx.step(ids, 3)
    before = [(ctx.state(i), ctx.forces(i)) for i in ids]
    res = ctx.autotune(ids)
    assert len(res) == 2 and sorted(r["n_systems"] for r in res) == [1, 3]
    for r in res:
        timed = {k: v for k, v in r["ms"].items() if v >= 0}
        assert set(timed) == {"column", "tile", "lean", "general"} and not r["from_cache"]
        assert r["layout"] == min(timed, key=timed.get)
    for i, ((x, v, img), f) in zip(ids, before):
        x2, v2, img2 = ctx.state(i)
        assert np.array_equal(x, x2) and np.array_equal(v, v2) and np.array_equal(img, img2)
        assert np.array_equal(f, ctx.forces(i))
    # a later call for the same signature takes the decision without timing
    again = ctx.autotune(ids)
    assert all(r["from_cache"] for r in again)
    assert [r["layout"] for r in again] == [r["layout"] for r in res]
    # forces in the chosen layout against the FP64 oracle on the same state
    for i, sd in zip(ids, systems):
        ctx.compute_forces(i)
        x, v, img = ctx.state(i)
        o = oracle_mod.Oracle(sd)
        o.set_state(x, v, img)
        o.set_step(ctx.thermo(i)["step"])
        o.compute_forces()
        assert rel_rms(ctx.forces(i), o.forces()) < MIXED_TOL


def test_autotune_on_first_step_then_cache(ctx_factory, oracle_mod):
    """Context(autotune=True): rbmd_init tunes new systems before their first force evaluation; a
    system added later with the same signature takes the cached layout."""
    ctx = ctx_factory(autotune=True)
    a = ctx.add_system(_saline(3000, 5))
    ctx.init(a)
    ctx.step(a, 4)
    assert ctx.thermo(a)["status"] == 0
    b = ctx.add_system(_saline(3000, 6))
    ctx.init(b)
    r = ctx.autotune([b])
    assert r[0]["from_cache"]


def test_autotune_fixed_layouts(ctx_factory):
    """NPT systems and boxes of nc cells per dimension (the least accepted) have a single usable
    layout; boxes of nc + 1 to 2 nc cells (a stencil that repeats cells) and edges of 2 rc have all
    three."""
    ctx = ctx_factory()
    npt = synth.lj_fcc(cells=6)
    p = npt.params
    p.ensemble, p.temp_ctrl, p.press_ctrl = A.ENS_NPT, A.TC_BERENDSEN, A.PC_BERENDSEN
    p.pressure[:] = (0.5, 0.5, 0.5)
    tiny = synth.lj_fcc(cells=2, rho=0.9, precision=A.PREC_MIXED)  # 3 cells per dimension = nc
    small = synth.lj_fcc(cells=3, precision=A.PREC_MIXED)  # 6 cells per dimension, edges 2 rc
    ids = [ctx.add_system(npt), ctx.add_system(tiny)]
    sid = ctx.add_system(small)
    ctx.init(ids + [sid])
    for r in ctx.autotune(ids):
        assert r["layout"] == "general" and all(v < 0 for v in r["ms"].values())
    (r,) = ctx.autotune([sid])
    assert all(v > 0 for v in r["ms"].values())
