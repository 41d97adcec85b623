"""RBMD_NEAR_TABLE on the GPU: the reference's alpha = 0.1 lookup table for the RBL near Coulomb
force (ExecStaticTable::Extract / TableGnearValue, staticTable/ExecStaticTable.h:96-135, used by
ComputeNearForceRBLERF[SpecialBonds]Worklet, RunWorklet.cpp:1046-1047, 1171-1172), against the
FP64 oracle in the same mode, in every pair layout.  The reference's own table files are loaded
where the reference tree is present (RBMD_REFERENCE_ROOT names a copy of it)."""
import os

import numpy as np
import pytest

import rbmd_b200
from rbmd_b200 import _abi as A
from rbmd_b200 import synth

import refinputs as R
from conftest import rel_rms

pytestmark = pytest.mark.gpu

FILES = ("res/json_files/Gnear_table_leq2_2.txt", "res/json_files/Gnear_table_geq2_2.txt")


def _jiggle(sd, scale, seed=0):
    """Lattice starts cancel their forces to round-off and repeat each distance over whole shells of
    pairs (a shell near a key's edge would flip together); a small random displacement avoids both."""
    rng = np.random.default_rng(seed)
    lo, L = sd.box_lo, sd.box_hi - sd.box_lo
    sd.pos = np.ascontiguousarray((sd.pos - lo + rng.normal(scale=scale, size=sd.pos.shape)) % L + lo)
    return sd


def _systems():
    return {
        "nacl_rbe_rbl": _jiggle(synth.nacl_melt(n_side=10, seed=2), 0.03),       # LJ units, no special bonds
        "water_rbe_rbl": _jiggle(synth.spce_water(n_mol=1000, seed=4), 0.05),    # real units, special bonds
        "saline_rbe_rbl": _jiggle(synth.saline(4000, seed=5), 0.05),             # water + ions
    }


def _table(sd):
    sd.params.near_table = A.NEAR_TABLE
    return sd


def _add(ctx_factory, sd, layout):
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
    return ctx, sid


def _tile_ok(sd):
    return all(2 * sd.params.cut_off <= h - lo for h, lo in zip(sd.box_hi, sd.box_lo))


def _forces(ctx_factory, sd, layout="auto"):
    ctx, sid = _add(ctx_factory, sd, layout)
    ctx.compute_forces(sid)
    return ctx.forces(sid)


def _oracle_forces(oracle_mod, sd):
    ref = sd.copy()
    ref.params.precision = A.PREC_FP64
    o = oracle_mod.Oracle(ref)
    o.compute_forces()
    return o.forces()


@pytest.mark.parametrize("layout", ["auto", "lean", "cell"])
@pytest.mark.parametrize("name", ["nacl_rbe_rbl", "water_rbe_rbl", "saline_rbe_rbl"])
def test_near_table_forces_fp64(ctx_factory, oracle_mod, name, layout):
    sd = _table(_systems()[name])
    if layout == "cell" and not _tile_ok(sd):
        pytest.skip("the tile layout needs edges of at least 2 rc")
    sd.params.precision = A.PREC_FP64
    err = rel_rms(_forces(ctx_factory, sd, layout), _oracle_forces(oracle_mod, sd))
    assert err < 1e-6, err


@pytest.mark.parametrize("layout", ["auto", "lean", "cell", "column"])
@pytest.mark.parametrize("name", ["nacl_rbe_rbl", "water_rbe_rbl", "saline_rbe_rbl"])
def test_near_table_forces_mixed(ctx_factory, oracle_mod, name, layout):
    sd = _table(_systems()[name])
    if layout in ("cell", "column") and not _tile_ok(sd):
        pytest.skip("the tile layout needs edges of at least 2 rc")
    sd.params.precision = A.PREC_MIXED
    err = rel_rms(_forces(ctx_factory, sd, layout), _oracle_forces(oracle_mod, sd))
    assert err < 1e-3, err
    # the FP32 distance keys the table as the FP64 one does except within an ulp or so of a key's
    # edge (about one pair in 4e4, whose G then steps by about 0.8%)
    assert err < 5e-4, err


@pytest.mark.parametrize("name", ["nacl_rbe_rbl", "water_rbe_rbl"])
def test_near_table_is_the_lookup(ctx_factory, name):
    """At alpha = 0.1 the table holds the analytic G at one point per key, so the forces differ from
    the analytic ones by the lookup's step (no interpolation, up to 0.8% of G per pair): visibly,
    by less than 10% of the net forces (which are small residuals of the pair forces)."""
    sd = _systems()[name]
    sd.params.alpha = 0.1
    sd.params.precision = A.PREC_FP64
    fa = _forces(ctx_factory, sd)
    ft = _forces(ctx_factory, _table(sd.copy()))
    d = rel_rms(ft, fa)
    assert 1e-5 < d < 0.1, d


@pytest.mark.skipif(not R.available(), reason="reference tree not present")
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_near_table_reference_values(ctx_factory, oracle_mod, prec):
    """The reference's own table values (its two files, G by key), given through
    rbmd_system_desc.near_table_values, on the GPU and in the oracle."""
    import ctypes as C
    tab = np.zeros(2048, np.float32)
    assert rbmd_b200.lib().rbmd_near_table_default(tab.ctypes.data_as(C.POINTER(C.c_float))) == A.OK
    for rel in FILES:
        for row in (ln.split() for ln in open(os.path.join(R.REF_ROOT, rel)) if ln.strip()):
            tab[int(row[0])] = np.float32(float(row[3]))
    sd = _table(_systems()["water_rbe_rbl"])
    sd.near_table_values = tab
    sd.params.precision = A.PREC_FP64 if prec == "fp64" else A.PREC_MIXED
    f = _forces(ctx_factory, sd)
    err = rel_rms(f, _oracle_forces(oracle_mod, sd))
    assert err < (1e-6 if prec == "fp64" else 5e-4), err
    # the files' values are the library's to six digits where G matters (r < 8)
    sd2 = _table(_systems()["water_rbe_rbl"])
    sd2.params.precision = sd.params.precision
    assert rel_rms(f, _forces(ctx_factory, sd2)) < 1e-5


def test_near_table_steps(ctx_factory, oracle_mod):
    sd = _table(_systems()["water_rbe_rbl"])
    sd.params.precision = A.PREC_FP64
    ctx, sid = _add(ctx_factory, sd, "auto")
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


def test_near_table_refuses_cutoff_beyond_table(ctx_factory):
    sd = _table(synth.spce_water(n_mol=1500, seed=4))
    sd.params.cut_off = 12.5
    ctx = ctx_factory()
    with pytest.raises(rbmd_b200.RbmdError) as e:
        ctx.add_system(sd)
    assert e.value.code == A.ERR_UNSUPPORTED
