"""Parity of the sm_100a path (through the C ABI) with the FP64 oracle on the same inputs.

Integer work (cell binning, RBL batch selection, RBE k samples) must be bit-exact; FP64 forces
within relative RMS 1e-6; mixed precision within 1e-3 of the FP64 oracle."""
import numpy as np
import pytest

from rbmd_b200 import _abi as A
from rbmd_b200 import synth

from conftest import rel_rms

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-6
MIXED_TOL = 1e-3


def _jiggle(sd, scale, seed=0):
    rng = np.random.default_rng(seed)
    sd.pos = np.ascontiguousarray((sd.pos + rng.normal(scale=scale, size=sd.pos.shape)) % sd.box_hi[0])
    return sd


def lj_small(**kw):
    return _jiggle(synth.lj_fcc(cells=6, **kw), 0.08)


def nacl_small(**kw):
    return _jiggle(synth.nacl_melt(n_side=10, **kw), 0.15)


def water_small(**kw):
    return synth.spce_water(n_mol=1000, **kw)


def eam_small(oracle_mod, **kw):
    sd = synth.eam_cu(cells=6, build_splines=oracle_mod.eam_splines, **kw)
    return _jiggle(sd, 0.05)


def pair(ctx_factory, oracle_mod, sd, layout="auto", **ctxkw):
    """GPU context + system and the oracle twin.  `layout` selects the pair kernel: "auto" (the
    library's choice), "atom" (general warp-per-atom traversal), "lean" (warp per atom with segment
    tables), "cell" (tile: warp per home cell, candidates shared by the cell's atoms), "column"
    (warp per column of home cells, lane per atom; mixed-precision RBL forces, else as "cell")."""
    import os
    ctx = ctx_factory(**ctxkw)
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
    return ctx, sid, o


LAYOUTS = ["auto", "atom", "lean", "cell", "column"]


CASES = {
    "lj_rbl": lambda om: lj_small(),
    "lj_verlet": lambda om: lj_small(neighbor=A.NEIGH_VERLET, cut_off=2.5, r_core=2.5),
    "nacl_rbe_rbl": lambda om: nacl_small(),
    "nacl_ewald_verlet": lambda om: nacl_small(coulomb=A.COUL_EWALD, neighbor=A.NEIGH_VERLET, kmax=(5, 5, 5)),
    "water_cvff_rbe_rbl": lambda om: water_small(),
    "water_cvff_verlet": lambda om: water_small(neighbor=A.NEIGH_VERLET, coulomb=A.COUL_EWALD, kmax=(4, 4, 4)),
    "eam_rbl": lambda om: eam_small(om, precision=A.PREC_FP64),
    "eam_verlet": lambda om: eam_small(om, precision=A.PREC_FP64, neighbor=A.NEIGH_VERLET),
}


@pytest.mark.parametrize("case", ["lj_rbl", "nacl_rbe_rbl", "water_cvff_rbe_rbl", "eam_rbl"])
def test_cells_bit_exact(ctx_factory, oracle_mod, case):
    sd = CASES[case](oracle_mod)
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd)
    g = ctx.cells(sid)
    r = o.cells()
    for a, b in zip(g, r):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("layout", ["lean", "cell"])
@pytest.mark.parametrize("case,mode", [("lj_rbl", A.RBL_STRIDE), ("nacl_rbe_rbl", A.RBL_STRIDE),
                                       ("water_cvff_rbe_rbl", A.RBL_STRIDE),
                                       ("water_cvff_rbe_rbl", A.RBL_PHILOX), ("eam_rbl", A.RBL_STRIDE)])
def test_rbl_lists_bit_exact(ctx_factory, oracle_mod, case, mode, layout):
    sd = CASES[case](oracle_mod)
    sd.params.rbl_mode = mode
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd, layout=layout)
    gn, gs, gi = ctx.rbl_lists(sid, cap=1024)
    on, os_, oi = o.rbl_lists(cap=1024)
    assert np.array_equal(gn, on)
    assert np.array_equal(gs, os_)
    for i in range(sd.n):
        k = gn[i] + gs[i]
        assert np.array_equal(gi[i, :k], oi[i, :k]), f"atom {i}"


@pytest.mark.parametrize("seed", [1, 2, 3, 77])
def test_rbe_samples_bit_exact(ctx_factory, oracle_mod, seed):
    sd = nacl_small(seed=seed)
    sd.params.seed = 1000 + seed
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd)
    ctx.compute_forces(sid)
    m, rk = ctx.kspace(sid)
    o.compute_forces()
    om, ork = o.kspace()
    assert np.array_equal(m, om)
    assert rel_rms(rk, ork) < 1e-12


def test_rbe_samples_test_mode(ctx_factory, oracle_mod):
    sd = nacl_small()
    sd.params.random_mode = A.RANDOM_TEST
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd)
    ctx.compute_forces(sid)
    m, _ = ctx.kspace(sid)
    o.compute_forces()
    om, _ = o.kspace()
    assert np.array_equal(m, om)


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("case", sorted(CASES))
def test_forces_fp64(ctx_factory, oracle_mod, case, layout):
    sd = CASES[case](oracle_mod)
    sd.params.precision = A.PREC_FP64
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd, layout=layout)
    ctx.compute_forces(sid)
    f = ctx.forces(sid)
    o.compute_forces()
    assert rel_rms(f, o.forces()) < FP64_TOL


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("case", ["lj_rbl", "nacl_rbe_rbl", "water_cvff_rbe_rbl", "eam_rbl"])
def test_forces_mixed_vs_fp64_oracle(ctx_factory, oracle_mod, case, layout):
    sd = CASES[case](oracle_mod)
    sd.params.precision = A.PREC_MIXED
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd, layout=layout)
    ctx.compute_forces(sid)
    f = ctx.forces(sid)
    o.compute_forces()
    err = rel_rms(f, o.forces())
    assert err < MIXED_TOL, err


@pytest.mark.parametrize("case", ["lj_rbl", "nacl_rbe_rbl", "water_cvff_rbe_rbl", "eam_rbl", "lj_verlet"])
def test_one_step_and_thermo(ctx_factory, oracle_mod, case):
    sd = CASES[case](oracle_mod)
    sd.params.precision = A.PREC_FP64
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd, graphs=False)
    ctx.init(sid)
    o.init()
    ctx.step(sid, 1)
    o.step(1)
    x, v, img = ctx.state(sid)
    ox, ov, oimg = o.state()
    assert rel_rms(x, ox) < 1e-10
    assert rel_rms(v, ov) < 1e-7
    assert np.array_equal(img, oimg)
    tg, to = ctx.thermo(sid), o.thermo()
    assert tg["step"] == to["step"] == 1
    for key in ("temperature", "kinetic_energy", "e_lj", "e_coul_near", "e_coul_far", "e_bond", "e_angle",
                "e_eam", "total_energy"):
        assert tg[key] == pytest.approx(to[key], rel=1e-7, abs=1e-9), key
    assert tg["pressure"] == pytest.approx(to["pressure"], rel=1e-6, abs=1e-6)
    for k in range(3):
        assert tg["nhc_eta"][k] == pytest.approx(to["nhc_eta"][k], rel=1e-8, abs=1e-14)


def _push_outside(sd):
    """Moves a few atoms outside [lo, hi): one exactly onto hi, one a whole box length past it, one
    below lo.  The reference bins them clamped but walks the neighbourhood of the unclamped cell."""
    L = sd.box_hi[0] - sd.box_lo[0]
    sd.pos = sd.pos.copy()
    sd.pos[0, 0] = sd.box_hi[0]
    sd.pos[7, 1] += L
    sd.pos[11, 2] -= 0.3 * L
    sd.pos[11, 2] = min(sd.pos[11, 2], sd.box_lo[2] - 0.05)
    return sd


@pytest.mark.parametrize("layout", ["atom", "lean", "cell"])
@pytest.mark.parametrize("case", ["lj_rbl", "nacl_rbe_rbl", "eam_rbl", "lj_verlet", "water_cvff_rbe_rbl"])
def test_forces_atoms_outside_box(ctx_factory, oracle_mod, case, layout):
    sd = _push_outside(CASES[case](oracle_mod))
    sd.params.precision = A.PREC_FP64
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd, layout=layout)
    ctx.compute_forces(sid)
    f = ctx.forces(sid)
    o.compute_forces()
    assert rel_rms(f, o.forces()) < FP64_TOL
    assert ctx.thermo(sid)["status"] == 0


@pytest.mark.parametrize("layout", ["lean", "cell"])
def test_rbl_lists_atoms_outside_box(ctx_factory, oracle_mod, layout):
    sd = _push_outside(CASES["water_cvff_rbe_rbl"](oracle_mod))
    sd.params.rbl_mode = A.RBL_PHILOX
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd, layout=layout)
    gn, gs, gi = ctx.rbl_lists(sid, cap=1024)
    on, os_, oi = o.rbl_lists(cap=1024)
    assert np.array_equal(gn, on) and np.array_equal(gs, os_)
    for i in range(sd.n):
        k = gn[i] + gs[i]
        assert np.array_equal(gi[i, :k], oi[i, :k]), f"atom {i}"


@pytest.mark.parametrize("case", ["nacl_rbe_rbl", "water_cvff_rbe_rbl"])
def test_ten_steps_track_oracle(ctx_factory, oracle_mod, case):
    sd = CASES[case](oracle_mod)
    sd.params.precision = A.PREC_FP64
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd)
    ctx.init(sid)
    o.init()
    ctx.step(sid, 10)
    o.step(10)
    x, v, _ = ctx.state(sid)
    ox, ov, _ = o.state()
    assert rel_rms(x, ox) < 1e-8
    assert rel_rms(v, ov) < 1e-5
    assert ctx.thermo(sid)["status"] == 0


def test_batched_equals_plain_and_alone(ctx_factory, oracle_mod):
    systems = [nacl_small(seed=s) for s in (1, 2)] + [water_small(seed=3, precision=A.PREC_MIXED)] + \
              [lj_small(seed=4)]
    for k, sd in enumerate(systems):
        sd.params.seed = 50 + k
    results = {}
    for mode in ("alone", "plain", "batched", "batched_graph"):
        ctx = ctx_factory(batched=mode.startswith("batched"), graphs=mode == "batched_graph")
        ids = [ctx.add_system(sd) for sd in systems]
        if mode == "alone":
            out = []
            for sid in ids:
                ctx.init(sid)
                ctx.step(sid, 7)
                out.append(ctx.state(sid))
        else:
            ctx.init(ids)
            ctx.step(ids, 7)
            out = [ctx.state(sid) for sid in ids]
        results[mode] = out
    for mode in ("plain", "batched", "batched_graph"):
        for a, b in zip(results["alone"], results[mode]):
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), mode


def test_net_force_vanishes_full_size_nacl(ctx_factory):
    """Size-independent property at the full 8000-ion melt: RBL near forces are mean-subtracted
    and the RBE force sums to zero analytically, so the net force is round-off."""
    sd = synth.nacl_melt()
    ctx = ctx_factory()
    sid = ctx.add_system(sd)
    ctx.compute_forces(sid)
    f = ctx.forces(sid)
    assert np.abs(f.sum(0)).max() < 1e-9 * np.abs(f).sum()


def test_errors_are_status_codes(ctx_factory):
    import rbmd_b200
    ctx = ctx_factory()
    with pytest.raises(rbmd_b200.RbmdError) as e:
        ctx.step([12345], 1)
    assert e.value.code == A.ERR_STATE
    sd = lj_small()
    sd.params.r_core = 5.0  # r_core > cut_off
    with pytest.raises(rbmd_b200.RbmdError) as e:
        ctx.add_system(sd)
    assert e.value.code == A.ERR_ARG
    sd = lj_small()
    sd.pos[3, 1] = np.nan
    with pytest.raises(rbmd_b200.RbmdError) as e:
        ctx.add_system(sd)
    assert e.value.code == A.ERR_NUMERIC


def test_energy_drift_mixed_matches_fp64():
    """The LJ fluid (4000 atoms, RBL, NVE, dt 0.005) over 1000 steps: mixed precision conserves
    energy as well as FP64 (drifts within 2e-4 of each other, both below 5e-3 of |E_0|)."""
    import bench
    d = bench.measure_drift(0)
    assert abs(d["fp64"]["drift"]) < 5e-3 and abs(d["mixed"]["drift"]) < 5e-3
    assert abs(d["mixed"]["drift"] - d["fp64"]["drift"]) < 2e-4
    assert d["energy_mixed_vs_fp64"] < 2e-3


def test_mixed_precision_classification_is_exact_along_trajectories(oracle_mod):
    """FP32 squared distances near rs^2 or rc^2 are classified again in FP64, so the mixed path
    picks the same RBL pairs as the FP64 oracle along a trajectory: its force error stays at the
    FP32 arithmetic level (a different pick would add ~1e-3 or more)."""
    import rbmd_b200
    for k, n in enumerate((1000, 4000, 12000)):
        sd = synth.saline(n, seed=40 + k)
        sd.params.seed = 900 + k
        ctx = rbmd_b200.Context()
        sid = ctx.add_system(sd)
        ctx.init(sid)
        for _ in range(3):
            ctx.step(sid, 5)
            x, v, img = ctx.state(sid)
            ctx.compute_forces(sid)
            o = oracle_mod.Oracle(sd)
            o.set_state(x, v, img)
            o.set_step(ctx.thermo(sid)["step"])
            o.compute_forces()
            assert rel_rms(ctx.forces(sid), o.forces()) < 1e-4
        ctx.close()


SMALL_BOXES = {
    # boxes holding more than nc but fewer than 2 nc + 1 cells per dimension: the stencil repeats
    # cells, and the tile and lean kernels walk a row's z cells in up to three ranges
    "water_dims4": lambda: synth.spce_water(n_mol=300),
    "nacl_dims4": lambda: _jiggle(synth.nacl_melt(n_side=6), 0.15),
    "lj_dims6_nc3": lambda: _jiggle(synth.lj_fcc(cells=3), 0.08),
    # edges below 2 rc: a pair within rc may not be at its nearest image (lean only)
    "water_dims3": lambda: synth.spce_water(n_mol=120),
}


@pytest.mark.parametrize("prec", [A.PREC_FP64, A.PREC_MIXED])
@pytest.mark.parametrize("layout", ["cell", "lean", "column"])
@pytest.mark.parametrize("case", list(SMALL_BOXES))
def test_small_box_layouts(ctx_factory, oracle_mod, case, layout, prec):
    sd = SMALL_BOXES[case]()
    short = any(2 * sd.params.cut_off > h - lo for h, lo in zip(sd.box_hi, sd.box_lo))
    if layout in ("cell", "column") and short:
        pytest.skip("the tile layout needs edges of at least 2 rc")
    sd.params.precision = prec
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd, layout=layout)
    d = ctx.derived(sid)
    nc = d["num_cycles"]
    assert all(nc < k for k in d["dims"]) and any(k < 2 * nc + 1 for k in d["dims"])
    gn, gs, gi = ctx.rbl_lists(sid, cap=1024)
    on, os_, oi = o.rbl_lists(cap=1024)
    assert np.array_equal(gn, on) and np.array_equal(gs, os_)
    for i in range(sd.n):
        k = gn[i] + gs[i]
        assert np.array_equal(gi[i, :k], oi[i, :k]), f"atom {i}"
    ctx.compute_forces(sid)
    ref = sd.copy()
    ref.params.precision = A.PREC_FP64
    o2 = oracle_mod.Oracle(ref)
    o2.compute_forces()
    assert rel_rms(ctx.forces(sid), o2.forces()) < (1e-9 if prec == A.PREC_FP64 else 1e-4)
