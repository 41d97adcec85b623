"""NPT barostats on the sm_100a path against the FP64 oracle: Berendsen (ExecutionNPT.cpp:90-122,
1334-1368, 1429-1447, 1506-1538) and the isotropic MTK barostat (:123-141, 1545-2066).

The box, its cell dims, the volume-dependent k-space tables and the remapped atoms are rebuilt on
the device every step; after a few steps they must agree with the oracle: box edges and volume to
1e-10 relative, positions within relative RMS 1e-8, velocities 1e-5, images and cell lists exactly,
RBE k samples exactly."""
import numpy as np
import pytest

from rbmd_b200 import _abi as A
from rbmd_b200 import synth

from conftest import rel_rms
from test_gpu_parity import eam_small, lj_small, pair, water_small

pytestmark = pytest.mark.gpu


def npt(sd, p_start, p_stop, p_damp, bulk, num_steps=200, mtk=False):
    p = sd.params
    p.ensemble = A.ENS_NPT
    p.temp_ctrl, p.press_ctrl = (A.TC_NOSE_HOOVER, A.PC_NOSE_HOOVER) if mtk else (A.TC_BERENDSEN, A.PC_BERENDSEN)
    p.pressure[:] = (p_start, p_stop, p_damp)
    p.bulk_modulus = bulk
    p.num_steps = num_steps
    p.precision = A.PREC_FP64
    return sd


# (system, P_start, P_stop, P_damp, bulk modulus) in each system's units
CASES = {
    "lj_rbl": lambda om: npt(lj_small(), 0.2, 0.4, 0.5, 10.0),
    "nacl_rbe_rbl": lambda om: npt(synth.nacl_melt(n_side=10), 0.0, 0.0, 0.5, 5.0),
    "nacl_ewald_verlet": lambda om: npt(synth.nacl_melt(n_side=10, coulomb=A.COUL_EWALD, neighbor=A.NEIGH_VERLET,
                                                        kmax=(5, 5, 5)), 0.0, 0.0, 0.5, 5.0),
    "water_cvff_rbe_rbl": lambda om: npt(water_small(), 1.0, 1.0, 1000.0, 2.0e4),
    "eam_rbl": lambda om: npt(eam_small(om), 0.0, 0.0, 1.0, 1.0e6),
}

# MTK: (system, P_start, P_stop, P_damp); P_damp about 100-1000 time steps
MTK_CASES = {
    "lj_rbl": lambda om: npt(lj_small(), 0.2, 0.6, 0.5, 0, mtk=True),
    "nacl_rbe_rbl": lambda om: npt(synth.nacl_melt(n_side=10), 0.0, 0.0, 0.5, 0, mtk=True),
    "nacl_ewald_verlet": lambda om: npt(synth.nacl_melt(n_side=10, coulomb=A.COUL_EWALD, neighbor=A.NEIGH_VERLET,
                                                        kmax=(5, 5, 5)), 0.0, 0.0, 0.5, 0, mtk=True),
    "water_cvff_rbe_rbl": lambda om: npt(water_small(), 1.0, 1.0, 200.0, 0, mtk=True),
    "eam_rbl": lambda om: npt(eam_small(om), 0.0, 0.0, 1.0, 0, mtk=True),
}


def compare(ctx, sid, o, x_tol=1e-8, v_tol=1e-5):
    tg, to = ctx.thermo(sid), o.thermo()
    assert tg["step"] == to["step"]
    assert tg["status"] == 0 and to["status"] == 0
    for k in range(3):
        assert tg["box_lo"][k] == pytest.approx(to["box_lo"][k], rel=1e-10, abs=1e-10)
        assert tg["box_hi"][k] == pytest.approx(to["box_hi"][k], rel=1e-10, abs=1e-10)
    assert tg["volume"] == pytest.approx(to["volume"], rel=1e-10)
    assert tg["pressure"] == pytest.approx(to["pressure"], rel=1e-6, abs=1e-6)
    for key in ("temperature", "potential_energy", "total_energy"):
        assert tg[key] == pytest.approx(to[key], rel=1e-6, abs=1e-8), key
    x, v, img = ctx.state(sid)
    ox, ov, oimg = o.state()
    assert rel_rms(x, ox) < x_tol
    assert rel_rms(v, ov) < v_tol
    assert np.array_equal(img, oimg)
    assert ctx.derived(sid)["dims"] == o.derived()["dims"]
    return tg, to


@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("case", list(CASES))
def test_npt_steps_track_oracle(ctx_factory, oracle_mod, case, graphs):
    sd = CASES[case](oracle_mod)
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd, graphs=graphs)
    ctx.init(sid)
    o.init()
    v0 = o.thermo()["volume"]
    ctx.step(sid, 4)
    o.step(4)
    ctx.step(sid, 4)
    o.step(4)
    tg, _ = compare(ctx, sid, o)
    assert tg["volume"] != v0  # the box moved


@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("case", list(MTK_CASES))
def test_mtk_steps_track_oracle(ctx_factory, oracle_mod, case, graphs):
    sd = MTK_CASES[case](oracle_mod)
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd, graphs=graphs)
    ctx.init(sid)
    o.init()
    v0 = o.thermo()["volume"]
    ctx.step(sid, 3)
    o.step(3)
    ctx.step(sid, 5)
    o.step(5)
    tg, _ = compare(ctx, sid, o)
    assert tg["volume"] != v0
    assert tg["nhc_eta"][0] == pytest.approx(o.thermo()["nhc_eta"][0], rel=1e-8, abs=1e-14)


def test_npt_cell_dims_change_and_cells_match(ctx_factory, oracle_mod):
    """A box just below 12 cells per edge grows past the boundary: dims go 11 -> 12 on the device
    and the cell list stays bit-exact."""
    rho = 4 * 6 ** 3 / 9.995 ** 3
    sd = npt(synth.lj_fcc(cells=6, rho=rho), 0.0, 0.0, 0.5, 10.0)
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd)
    ctx.init(sid)
    o.init()
    assert ctx.derived(sid)["dims"] == [11, 11, 11]
    ctx.step(sid, 6)
    o.step(6)
    compare(ctx, sid, o)
    assert ctx.derived(sid)["dims"] == [12, 12, 12]
    for a, b in zip(ctx.cells(sid), o.cells()):
        assert np.array_equal(a, b)


def test_npt_rbe_samples_after_remap(ctx_factory, oracle_mod):
    """The proposal tables rebuilt on the device for the new box drive the same Metropolis chain as
    the oracle's direct formulas."""
    sd = CASES["nacl_rbe_rbl"](oracle_mod)
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd)
    ctx.init(sid)
    o.init()
    ctx.step(sid, 5)
    o.step(5)
    m, _ = ctx.kspace(sid)
    om_, _ = o.kspace()
    assert np.array_equal(m, om_)


def test_npt_box_range_refused(ctx_factory, oracle_mod):
    """A dilation past the cell tables' range is refused on both sides: status bit, box unchanged."""
    sd = npt(lj_small(), -1e6, -1e6, 0.01, 1.0)
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd)
    ctx.init(sid)
    o.init()
    ctx.step(sid, 1)
    o.step(1)
    tg, to = ctx.thermo(sid), o.thermo()
    assert tg["status"] & A.STATUS_BOX_RANGE and to["status"] & A.STATUS_BOX_RANGE
    assert list(tg["box_lo"]) == list(sd.box_lo) and list(tg["box_hi"]) == list(sd.box_hi)
    x, _, _ = ctx.state(sid)
    ox, _, _ = o.state()
    assert rel_rms(x, ox) < 1e-10


def test_npt_mixed_precision(ctx_factory, oracle_mod):
    sd = CASES["water_cvff_rbe_rbl"](oracle_mod)
    sd.params.precision = A.PREC_MIXED
    ctx, sid, o = pair(ctx_factory, oracle_mod, sd)
    ctx.init(sid)
    o.init()
    ctx.step(sid, 5)
    o.step(5)
    tg, to = ctx.thermo(sid), o.thermo()
    assert tg["status"] == 0
    assert tg["volume"] == pytest.approx(to["volume"], rel=1e-4)
    x, _, _ = ctx.state(sid)
    ox, _, _ = o.state()
    assert rel_rms(x, ox) < 1e-5


def test_npt_batched_equals_alone(ctx_factory, oracle_mod):
    """NPT systems batch with each other (not with NVT ones or the other barostat) and give the same
    bits as alone."""
    systems = [npt(lj_small(seed=s), 0.2, 0.2, 0.5, 10.0) for s in (1, 2)] + [lj_small(seed=3)] + \
              [npt(lj_small(seed=s), 0.2, 0.2, 0.5, 0, mtk=True) for s in (4, 5)]
    for k, sd in enumerate(systems):
        sd.params.seed = 70 + k
    results = {}
    for mode in ("alone", "batched_graph"):
        ctx = ctx_factory(batched=mode != "alone", graphs=mode == "batched_graph")
        ids = [ctx.add_system(sd) for sd in systems]
        if mode == "alone":
            for sid in ids:
                ctx.init(sid)
                ctx.step(sid, 6)
        else:
            ctx.init(ids)
            ctx.step(ids, 6)
        results[mode] = [(ctx.state(sid), ctx.thermo(sid)) for sid in ids]
    for (sa, ta), (sb, tb) in zip(results["alone"], results["batched_graph"]):
        assert all(np.array_equal(a, b) for a, b in zip(sa, sb))
        assert list(ta["box_hi"]) == list(tb["box_hi"]) and ta["pressure"] == tb["pressure"]


def test_npt_validation(ctx_factory):
    ctx = ctx_factory()
    sd = npt(lj_small(), 0.2, 0.2, 0.5, 10.0)
    sd.params.temp_ctrl = A.TC_NOSE_HOOVER
    with pytest.raises(Exception, match="NOSE_HOOVER"):
        ctx.add_system(sd)
    sd = npt(lj_small(), 0.2, 0.2, 0.0, 0, mtk=True)
    with pytest.raises(Exception, match="damping"):
        ctx.add_system(sd)
    sd = npt(lj_small(), 0.2, 0.2, 0.5, 0.0)
    with pytest.raises(Exception, match="bulk_modulus"):
        ctx.add_system(sd)
