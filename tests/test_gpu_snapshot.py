"""Asynchronous state snapshots (rbmd_snapshot_begin / _poll / _wait) and the outputs the rbmd host
writes from them: the snapshot holds the state as of the work queued before it even when more
steps are queued before the wait; rbmd.trj (the reference's LAMMPS dump layout), temperature.rbmd
and the checkpoint data file, which reads back to the exact state of its step."""
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


def _water():
    return synth.spce_water(n_mol=300)


def _npt_nacl():
    """Berendsen NPT: the box moves every step, so the snapshot's box is the device's."""
    sd = synth.nacl_melt(n_side=10)
    p = sd.params
    p.ensemble, p.temp_ctrl, p.press_ctrl = A.ENS_NPT, A.TC_BERENDSEN, A.PC_BERENDSEN
    p.pressure[:] = (0.0, 0.0, 0.5)
    p.bulk_modulus = 5.0
    p.num_steps = 200
    p.precision = A.PREC_FP64
    return sd


@pytest.mark.parametrize("make", [_water, _npt_nacl], ids=["water", "npt_nacl"])
def test_snapshot_is_the_state_when_queued(ctx_factory, make):
    sd = make()
    a, b = ctx_factory(batched=False), ctx_factory(batched=False)
    sa, sb = a.add_system(sd), b.add_system(sd)
    a.init(sa)
    b.init(sb)
    a.step(sa, 7)
    snap = a.snapshot_begin(sa)
    a.step(sa, 30)  # queued before the wait: the snapshot must not see them
    x, v, img, box, step = snap.wait()
    b.step(sb, 7)
    xb, vb, ib = b.state(sb)
    tb = b.thermo(sb)
    assert np.array_equal(x, xb) and np.array_equal(v, vb) and np.array_equal(img, ib)
    assert step == tb["step"] == 7
    assert np.array_equal(box[0], tb["box_lo"]) and np.array_equal(box[1], tb["box_hi"])
    xa, _, _ = a.state(sa)
    assert not np.array_equal(xa, x)
    if sd.params.ensemble == A.ENS_NPT:
        assert not np.array_equal(box[1] - box[0], np.asarray(sd.box_hi) - np.asarray(sd.box_lo))


def test_snapshots_in_flight_and_poll(ctx_factory):
    sd = _water()
    ctx = ctx_factory()
    sid = ctx.add_system(sd)
    ctx.init(sid)
    snaps = []
    for _ in range(6):
        ctx.step(sid, 2)
        snaps.append(ctx.snapshot_begin(sid))
    ctx.sync()
    assert all(s.done() for s in snaps)
    steps = [s.wait()[4] for s in snaps]
    assert steps == [2, 4, 6, 8, 10, 12]
    with pytest.raises(rbmd_b200.RbmdError):
        snaps[0].wait()  # a ticket is consumed by its wait


def _blocks(path):
    lines = open(path).read().split("\n")
    out, k = [], 0
    while k < len(lines) and lines[k].strip():
        assert lines[k] == "ITEM: TIMESTEP"
        step = int(lines[k + 1])
        assert lines[k + 2] == "ITEM: NUMBER OF ATOMS"
        n = int(lines[k + 3])
        assert lines[k + 4] == "ITEM: BOX BOUNDS pp pp pp"
        box = np.array([[float(t) for t in lines[k + 5 + d].split()] for d in range(3)])
        assert lines[k + 8] == "ITEM: ATOMS id type x y z"
        atoms = np.array([[float(t) for t in ln.split()] for ln in lines[k + 9:k + 9 + n]])
        out.append((step, box, atoms))
        k += 9 + n
    return out


def test_host_trajectory_temperature_and_checkpoint(tmp_path):
    sd = _water()
    sd.params.num_steps = 8
    path = synth.write_rbmd_input(sd, str(tmp_path))
    cfg = json.load(open(path))
    cfg["outputs"].update(trajectory_out={"interval": 2}, checkpoint_out={"interval": 4, "file": "ck.data"})
    json.dump(cfg, open(path, "w"))
    r = subprocess.run([RBMD, "cuda", "-j", path], cwd=str(tmp_path), capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr

    ctx = rbmd_b200.Context(batched=False)
    sid = ctx.add_system(sd)
    ctx.init(sid)
    states, thermos = {}, {}
    for s in range(9):
        thermos[s] = ctx.thermo(sid)
        states[s] = ctx.state(sid)
        ctx.step(sid, 1)
    ctx.close()

    blocks = _blocks(tmp_path / "rbmd.trj")
    assert [b[0] for b in blocks] == [2, 4, 6, 8]
    for step, box, atoms in blocks:
        assert atoms.shape == (sd.n, 5)
        assert np.array_equal(atoms[:, 0], np.arange(1, sd.n + 1))
        assert np.array_equal(atoms[:, 1], sd.types + 1)
        np.testing.assert_allclose(atoms[:, 2:], states[step][0], rtol=1e-5, atol=1e-4)
        np.testing.assert_allclose(box, np.stack([sd.box_lo, sd.box_hi], 1), rtol=5e-6)  # %g: 6 digits

    lines = [ln.split() for ln in open(tmp_path / "temperature.rbmd").read().split("\n") if ln.strip()]
    assert lines[0] == ["Step", "Temperature", "Pressure"]
    rows = np.array([[float(t) for t in ln] for ln in lines[1:]])
    assert np.array_equal(rows[:, 0], np.arange(9))
    np.testing.assert_allclose(rows[:, 1], [thermos[s]["temperature"] for s in range(9)], rtol=1e-5)

    # the checkpoint of the last step reads back as the exact state (17 significant digits)
    ck = str(tmp_path / "ck.data")
    head = open(ck).readline()
    assert "step 8" in head and "atom_style full" in head
    cfg["init_configuration"]["read_data"]["file"] = ck
    cfg["outputs"] = {}
    json.dump(cfg, open(path, "w"))
    dump = tmp_path / "d.json"
    r = subprocess.run([RBMD, "-j", path, "--dump-system", str(dump)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    d = json.load(open(dump))
    x8, v8, _ = states[8]
    assert np.array_equal(np.array(d["position"]).reshape(-1, 3), x8)
    assert np.array_equal(np.array(d["velocity"]).reshape(-1, 3), v8)
    assert np.array_equal(np.array(d["bond_atoms"]), sd.bond_atoms)
    assert np.array_equal(np.array(d["charge"]), sd.charge)
