"""Continuous batching (rbmd_serve_*): every request's result must be the one the same system gives
run alone, whatever it was batched with, whenever it was admitted and however its steps were cut
into rounds.  Results are compared bit for bit: the per-system arithmetic does not depend on the
batch (segment-indexed launches, per-system reductions in a fixed order)."""
import time

import numpy as np
import pytest

import rbmd_b200
from rbmd_b200 import _abi as A
from rbmd_b200 import synth

pytestmark = pytest.mark.gpu


def _mix():
    """Uneven sizes and kinds: mixed-precision saline, FP64 NaCl melt, LJ fcc, mixed water."""
    out = [
        (synth.saline(1500, seed=5), 9),
        (synth.nacl_melt(n_side=8, seed=2), 14),
        (synth.lj_fcc(cells=5, seed=3), 6),
        (synth.spce_water(n_mol=600, seed=4, precision=A.PREC_MIXED), 11),
        (synth.saline(3000, seed=6), 7),
    ]
    for k, (sd, _) in enumerate(out):
        sd.params.seed = 100 + k
    return out


def _alone(sd, nsteps):
    ctx = rbmd_b200.Context()
    sid = ctx.add_system(sd)
    ctx.init(sid)
    ctx.step(sid, nsteps)
    x, v, _ = ctx.state(sid)
    th = ctx.thermo(sid)
    ctx.close()
    return x, v, th


@pytest.fixture(scope="module")
def alone_results():
    return [_alone(sd, n) for sd, n in _mix()]


def _serve(mix, wait_between=None, **cfg):
    ctx = rbmd_b200.Context()
    ctx.serve_start(**cfg)
    rids = []
    for k, (sd, n) in enumerate(mix):
        rids.append(ctx.serve_submit(sd, n))
        if wait_between is not None and k == wait_between:
            assert ctx.serve_wait(rids[0], 120.0) == 0  # later requests arrive after the first is done
    out = []
    for rid in rids:
        assert ctx.serve_wait(rid, 300.0) == 0
        x, v, th, st = ctx.serve_result(rid)
        out.append((x, v, th, st))
    ctx.serve_stop()
    ctx.close()
    return out


@pytest.mark.parametrize("cfg", [dict(steps_per_round=4), dict(steps_per_round=50, max_systems=2),
                                 dict(steps_per_round=3, max_systems=1),
                                 dict(steps_per_round=4, round_atoms=3500)],
                         ids=["all_at_once", "two_slots", "one_slot", "least_work_first"])
def test_serve_results_equal_alone(alone_results, cfg):
    mix = _mix()
    got = _serve(mix, **cfg)
    for (sd, n), (xa, va, tha), (x, v, th, st) in zip(mix, alone_results, got):
        assert st["status"] == 0 and th["status"] == 0
        assert st["atom_steps"] == sd.n * n
        assert np.array_equal(x, xa) and np.array_equal(v, va), sd.name
        # the thermo of systems retired together (one batched evaluation) equals the thermo alone
        for key in ("potential_energy", "kinetic_energy", "total_energy", "pressure", "e_lj", "e_coul_near",
                    "e_coul_far", "e_bond", "e_angle", "temperature", "step"):
            assert th[key] == tha[key], (sd.name, key)


def test_serve_late_arrivals(alone_results):
    mix = _mix()
    got = _serve(mix, wait_between=1, steps_per_round=5)
    for (xa, va, _), (x, v, _, st) in zip(alone_results, got):
        assert np.array_equal(x, xa) and np.array_equal(v, va)


def test_serve_hbm_budget_admission(alone_results):
    """A budget that holds the largest request but not all of them: requests wait for memory,
    are admitted in arrival order, and still give the alone results."""
    mix = _mix()
    sizes = [rbmd_b200.system_bytes(sd) for sd, _ in mix]
    got = _serve(mix, hbm_budget_bytes=max(sizes) + min(sizes), steps_per_round=4)
    admits = [st["t_admit"] for _, _, _, st in got]
    assert admits == sorted(admits)
    for (xa, va, _), (x, v, _, st) in zip(alone_results, got):
        assert np.array_equal(x, xa) and np.array_equal(v, va)


def test_serve_rejects_request_over_budget():
    ctx = rbmd_b200.Context()
    sd = synth.saline(2000, seed=1)
    ctx.serve_start(hbm_budget_bytes=1024)
    with pytest.raises(rbmd_b200.RbmdError) as e:
        ctx.serve_submit(sd, 5)
    assert e.value.code == A.ERR_BUDGET
    ctx.serve_stop()
    ctx.close()


def test_serve_poll_states():
    ctx = rbmd_b200.Context()
    ctx.serve_start(steps_per_round=2)
    sd = synth.lj_fcc(cells=4, seed=9)
    rid = ctx.serve_submit(sd, 6)
    t0 = time.monotonic()
    while ctx.serve_poll(rid) != A.REQ_DONE:
        assert time.monotonic() - t0 < 60.0
        time.sleep(0.005)
    x, v, th, st = ctx.serve_result(rid)
    assert th["step"] == 6 and st["t_done"] >= st["t_admit"] >= st["t_submit"]
    ctx.serve_stop()
    ctx.close()


def test_serve_least_work_first_rounds():
    """round_atoms: a round steps the requests with the least remaining work up to that many atoms,
    so a small request submitted with large ones finishes first; results stay the alone ones."""
    big = [synth.saline(3000, seed=20 + k) for k in range(3)]
    small = synth.saline(1000, seed=30)
    ctx = rbmd_b200.Context()
    ctx.serve_start(steps_per_round=5, round_atoms=3500)
    rids = [ctx.serve_submit(sd, 30) for sd in big] + [ctx.serve_submit(small, 30)]
    out = []
    for rid in rids:
        assert ctx.serve_wait(rid, 300.0) == 0
        out.append(ctx.serve_result(rid))
    ctx.serve_stop()
    ctx.close()
    done = [st["t_done"] for _, _, _, st in out]
    assert done[3] < min(done[:3])
    xa, va, _ = _alone(small, 30)
    assert np.array_equal(out[3][0], xa) and np.array_equal(out[3][1], va)
