"""Trajectory observables on the sm_100a path: MSD / VACF against the oracle's restatement on the
states the device reports, RDF pair counts bit for bit against the oracle (molecule exclusion, the
inbuild halves, radii beyond half the box, shared-memory and global bin counters, empty lists),
argument errors, and the msd.rbmd / vacf.rbmd / rdf.rbmd files of the rbmd host against the
Python API on the same run."""
import json
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


def _box(sd):
    return np.asarray(sd.box_hi, np.float64) - np.asarray(sd.box_lo, np.float64)


def _mol(sd):
    return np.arange(sd.n) if sd.molecule is None else np.asarray(sd.molecule)


def _lj():
    sd = synth.lj_fcc(cells=5, T=1.44)
    sd.params.precision = A.PREC_FP64
    return sd


def _water():
    sd = synth.spce_water(n_mol=300)
    return sd


@pytest.mark.parametrize("make", [_lj, _water], ids=["lj", "water"])
def test_msd_vacf_against_oracle(ctx_factory, oracle_mod, make):
    sd = make()
    ctx = ctx_factory()
    sid = ctx.add_system(sd)
    with pytest.raises(rbmd_b200.RbmdError):
        ctx.observe(sid)  # no reference configuration yet
    ctx.init(sid)
    ctx.step(sid, 5)
    x0, v0, i0 = ctx.state(sid)
    ctx.observe_reset(sid)
    ctx.step(sid, 60)
    x, v, img = ctx.state(sid)
    msd, vacf = ctx.observe(sid)
    om, ov = oracle_mod.msd_vacf(x0, i0, v0, x, img, v, _box(sd))
    assert (img != i0).any()  # some atoms crossed the box
    assert msd[3] > 0
    np.testing.assert_allclose(msd, om, rtol=1e-12, atol=1e-300)
    np.testing.assert_allclose(vacf, ov, rtol=1e-12, atol=1e-14 * np.abs(ov).max())
    # a later velocity reference leaves the position reference alone
    ctx.observe_reset(sid, msd=False, vacf=True)
    m2, v2 = ctx.observe(sid)
    np.testing.assert_allclose(m2, om, rtol=1e-12, atol=1e-300)
    assert v2[3] == pytest.approx((v * v).sum(1).mean(), rel=1e-12)


def _rdf_case(name):
    if name == "water_O_O":
        sd = _water()
        c = t = np.flatnonzero(sd.types == 0)
        return sd, c, t, 6.0, 0.05, True
    if name == "water_O_H":
        sd = _water()
        return sd, np.flatnonzero(sd.types == 0), np.flatnonzero(sd.types == 1), 6.0, 0.05, True
    if name == "lj_halves":
        sd = _lj()
        h = sd.n // 2
        return sd, np.arange(h), np.arange(h, 2 * h), 3.0, 0.01, False
    if name == "lj_beyond_half_box":
        sd = _lj()
        ids = np.arange(sd.n)
        return sd, ids[:200], ids, 6.5, 0.05, False
    if name == "lj_global_bins":
        sd = _lj()
        ids = np.arange(sd.n)
        return sd, ids[::3], ids, 3.0, 0.0003, True  # 10000 bins: counters in global memory
    raise KeyError(name)


@pytest.mark.parametrize("name", ["water_O_O", "water_O_H", "lj_halves", "lj_beyond_half_box", "lj_global_bins"])
def test_rdf_counts_bit_exact(ctx_factory, oracle_mod, name):
    sd, c, t, radius, dr, excl = _rdf_case(name)
    ctx = ctx_factory()
    sid = ctx.add_system(sd)
    ctx.init(sid)
    ctx.step(sid, 3)
    x, _, _ = ctx.state(sid)
    counts, vol = ctx.rdf_counts(sid, c, t, radius, dr, excl)
    ref = oracle_mod.rdf_counts(x, _mol(sd), _box(sd), c, t, radius, dr, excl)
    assert counts.sum() > 0
    assert np.array_equal(counts, ref)
    assert vol == pytest.approx(np.prod(_box(sd)), rel=1e-12)
    assert np.array_equal(rbmd_b200.rdf_bins(radius, dr), oracle_mod.rdf_bins(radius, dr))


def test_rdf_empty_lists_and_errors(ctx_factory):
    sd = _lj()
    ctx = ctx_factory()
    sid = ctx.add_system(sd)
    ctx.init(sid)
    counts, _ = ctx.rdf_counts(sid, [], np.arange(sd.n), 2.0, 0.1)
    assert counts.shape == (20,) and not counts.any()
    g = rbmd_b200.rdf_snapshot(counts, rbmd_b200.rdf_bins(2.0, 0.1), 0, sd.n, 1000.0)
    assert np.isnan(g).all()  # 0 / 0, printed as a blank by the reference
    for bad in (dict(centers=[sd.n]), dict(targets=[-1]), dict(radius=0.0), dict(dr=-0.1), dict(radius=0.05)):
        kw = dict(centers=[0], targets=[1], radius=2.0, dr=0.1)
        kw.update(bad)
        with pytest.raises(rbmd_b200.RbmdError):
            ctx.rdf_counts(sid, kw["centers"], kw["targets"], kw["radius"], kw["dr"])
    with pytest.raises(rbmd_b200.RbmdError):
        ctx.observe_reset(sid, msd=False, vacf=False)


def _table(path):
    lines = [ln for ln in open(path).read().split("\n") if ln.strip()]
    return lines[0].split(), [[float(v) for v in ln.split()] for ln in lines[1:]]


def test_host_writes_observable_files(tmp_path):
    """rbmd cuda -j with msd_out, vacf_out and rdf_out: every file row equals the same quantities
    taken through the Python API at the same steps of the same run (6 significant digits, the
    reference's stream precision)."""
    sd = _water()
    sd.params.num_steps = 8
    path = synth.write_rbmd_input(sd, str(tmp_path))
    cfg = json.load(open(path))
    cfg["outputs"].update(
        msd_out={"interval": 2, "start_step": 0, "end_step": 6},
        vacf_out={"interval": 1, "start_step": 2, "end_step": 5},
        rdf_out={"radius": 6.0, "dr": 0.1, "statistics_rdf_steps": 3, "atoms_pair": [[0, 0], [0, 1]]})
    json.dump(cfg, open(path, "w"))
    r = subprocess.run([RBMD, "cuda", "-j", path], cwd=str(tmp_path), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr

    # the same run through the API: outputs before each of num_steps + 1 steps, thermo first
    N, S = 8, 3
    ctx = rbmd_b200.Context(graphs=True, batched=False)
    sid = ctx.add_system(sd)
    ctx.init(sid)
    oxy, hyd = np.flatnonzero(sd.types == 0), np.flatnonzero(sd.types == 1)
    radii = rbmd_b200.rdf_bins(6.0, 0.1)
    acc = [np.zeros(radii.size), np.zeros(radii.size)]
    msd_rows, vacf_rows, rdf_final = [], [], None
    m = np.zeros(4)
    w = np.zeros(4)
    for s in range(N + 1):
        ctx.thermo(sid)
        if N - S <= s < N + 1:
            for k, (c, t) in enumerate(((oxy, oxy), (oxy, hyd))):
                counts, vol = ctx.rdf_counts(sid, c, t, 6.0, 0.1, True)
                acc[k] += rbmd_b200.rdf_snapshot(counts, radii, c.size, t.size, vol)
        if s == N - 1:
            rdf_final = [a / S for a in acc]
        if s == 0:
            ctx.observe_reset(sid, msd=True, vacf=False)
        if s <= 6:
            m, _ = ctx.observe(sid, msd=True, vacf=False)
        if s == 2:
            ctx.observe_reset(sid, msd=False, vacf=True)
        if 2 <= s <= 5:
            _, w = ctx.observe(sid, msd=False, vacf=True)
        if s >= 1 and s % 2 == 0:
            msd_rows.append([s, s * sd.params.timestep, *m, np.sqrt(m[3])])
        if s >= 1:
            vacf_rows.append([s, s * sd.params.timestep, *(w if s >= 2 else np.zeros(4))])
        ctx.step(sid, 1)
    ctx.close()

    head, rows = _table(tmp_path / "msd.rbmd")
    assert head == ["Step", "Time", "MSD_x", "MSD_y", "MSD_z", "MSD_total", "sqrt(MSD_total)"]
    np.testing.assert_allclose(rows, msd_rows, rtol=2e-5, atol=1e-12)
    head, rows = _table(tmp_path / "vacf.rbmd")
    assert head == ["Step", "Time", "VACFx", "VACFy", "VACFz", "VACF_total"]
    np.testing.assert_allclose(rows, vacf_rows, rtol=2e-5, atol=1e-9)
    head, rows = _table(tmp_path / "rdf.rbmd")
    assert head == ["Radius", "RDF:0-0", "RDF:0-1"]
    rows = np.array(rows)
    np.testing.assert_allclose(rows[:, 0], radii, rtol=1e-5)
    np.testing.assert_allclose(rows[:, 1:], np.stack(rdf_final, 1), rtol=2e-5, atol=1e-9)
    assert rows[:, 1:].max() > 1.0  # structure: water's first O-O / O-H shells stand above 1
