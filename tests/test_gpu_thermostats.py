"""NVT Berendsen and velocity-rescale thermostats against the FP64 oracle.

ExecutionNVT::Solve (run/ExecutionNVT.cpp:93-119) applies `UpdateVelocityByTempConType`
(:270-291) after the second half kick: the temperature is computed from the new velocities
(after RATTLE where water is constrained) and every velocity is scaled by
sqrt(1 + dt/Tdamp (T0/T - 1)) (BERENDSEN) or sqrt(T0/T) (TEMP_RESCALE).  The device applies the
factor in the force-assembly kernel's last block, or in the kinetic-energy kernel after RATTLE,
and hands it to the next step (`vscale_pending`), so both the order and the handoff are checked
here over one and ten steps, with and without constrained triples.
"""
import numpy as np
import pytest

from rbmd_b200 import _abi as A
from rbmd_b200 import synth

from conftest import rel_rms

pytestmark = pytest.mark.gpu


def _jiggle(sd, scale, seed=0):
    rng = np.random.default_rng(seed)
    sd.pos = np.ascontiguousarray((sd.pos + rng.normal(scale=scale, size=sd.pos.shape)) % sd.box_hi[0])
    return sd


def _lj(tc):
    # NVT (the LJ config itself is NVE): T0 1.44 with a short damping time so the factor is far from 1
    return _jiggle(synth.lj_fcc(cells=6, temp_ctrl=tc, ensemble=A.ENS_NVT, temperature=(1.8, 1.8, 0.05)), 0.08)


def _nacl(tc):
    return _jiggle(synth.nacl_melt(n_side=10, temp_ctrl=tc, temperature=(2.4, 2.4, 0.02)), 0.03)


def _water(tc):
    return synth.spce_water(n_mol=1000, temp_ctrl=tc, temperature=(340.0, 340.0, 20.0))


def _water_unconstrained(tc):
    return synth.spce_water(n_mol=1000, temp_ctrl=tc, temperature=(340.0, 340.0, 20.0), fix_shake=A.SHAKE_NULL,
                            timestep=0.5)


SYSTEMS = {"lj_rbl": _lj, "nacl_rbe_rbl": _nacl, "water_shake": _water, "water_free": _water_unconstrained}
THERMOSTATS = {"berendsen": A.TC_BERENDSEN, "rescale": A.TC_RESCALE}


@pytest.mark.parametrize("nsteps", [1, 10])
@pytest.mark.parametrize("tc", sorted(THERMOSTATS))
@pytest.mark.parametrize("case", sorted(SYSTEMS))
def test_thermostat_tracks_oracle(ctx_factory, oracle_mod, case, tc, nsteps):
    sd = SYSTEMS[case](THERMOSTATS[tc])
    sd.params.precision = A.PREC_FP64
    ctx = ctx_factory(graphs=nsteps > 1)
    sid = ctx.add_system(sd)
    o = oracle_mod.Oracle(sd)
    ctx.init(sid)
    o.init()
    ctx.step(sid, nsteps)
    o.step(nsteps)
    x, v, img = ctx.state(sid)
    ox, ov, oimg = o.state()
    assert rel_rms(x, ox) < 1e-9
    assert rel_rms(v, ov) < 1e-6
    assert np.array_equal(img, oimg)
    tg, to = ctx.thermo(sid), o.thermo()
    assert tg["status"] == 0
    assert tg["temperature"] == pytest.approx(to["temperature"], rel=1e-7)
    assert tg["kinetic_energy"] == pytest.approx(to["kinetic_energy"], rel=1e-7)
    assert tg["total_energy"] == pytest.approx(to["total_energy"], rel=1e-6, abs=1e-9)


@pytest.mark.parametrize("tc", sorted(THERMOSTATS))
def test_thermostat_batched_equals_alone(ctx_factory, tc):
    """Two thermostatted systems stepped in one batch give the same bits as each alone."""
    systems = [_nacl(THERMOSTATS[tc]), _water(THERMOSTATS[tc])]
    for k, sd in enumerate(systems):
        sd.params.seed = 70 + k
    out = {}
    for mode in ("alone", "batched"):
        ctx = ctx_factory(batched=mode == "batched", graphs=True)
        ids = [ctx.add_system(sd) for sd in systems]
        if mode == "alone":
            res = []
            for sid in ids:
                ctx.init(sid)
                ctx.step(sid, 6)
                res.append(ctx.state(sid))
        else:
            ctx.init(ids)
            ctx.step(ids, 6)
            res = [ctx.state(sid) for sid in ids]
        out[mode] = res
    for a, b in zip(out["alone"], out["batched"]):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
