"""rbmd_get_rbl_lists_static, the list entry point for callers that must not allocate device memory
while systems run (an observer thread beside running steps, a serving host whose HBM budget is
spent), against the allocating rbmd_get_rbl_lists, both through the C ABI.

The file is named to be collected last: a run that stops at the first failure has run every other
test before this one, and in a full run it executes after the others have used device memory in
the same process."""
import numpy as np
import pytest

import rbmd_b200
from rbmd_b200 import _abi as A
from rbmd_b200 import synth

pytestmark = pytest.mark.gpu

CAP = 256


def _nacl():
    sd = synth.nacl_melt(n_side=10)
    rng = np.random.default_rng(0)
    sd.pos = np.ascontiguousarray((sd.pos + rng.normal(scale=0.15, size=sd.pos.shape)) % sd.box_hi[0])
    return sd


def _water_philox():
    sd = synth.spce_water(n_mol=1000)
    sd.params.rbl_mode = A.RBL_PHILOX
    return sd


def _same_lists(alloc, static):
    """Lists are integer work: counts and picked ids must be identical; the static rows end in -1."""
    gn, gs, gi = alloc
    sn, ss, si = static
    assert np.array_equal(gn, sn)
    assert np.array_equal(gs, ss)
    for i in range(len(gn)):
        k = gn[i] + gs[i]
        assert np.array_equal(gi[i, :k], si[i, :k]), f"atom {i}"
        assert (si[i, k:] == -1).all(), f"atom {i} tail"


@pytest.mark.parametrize("make", [_nacl, _water_philox], ids=["nacl_stride", "water_philox"])
def test_static_lists_match_allocating_entry(ctx_factory, make):
    sd = make()
    ctx = ctx_factory()
    sid = ctx.add_system(sd)
    ctx.init(sid)
    for _ in range(2):  # two calls in a row: the second finds the first call's data in the scratch
        _same_lists(ctx.rbl_lists(sid, cap=CAP), ctx.rbl_lists_static(sid, cap=CAP))
    ctx.step(sid, 3)
    _same_lists(ctx.rbl_lists(sid, cap=CAP), ctx.rbl_lists_static(sid, cap=CAP))


def test_static_lists_reject_oversize(ctx_factory):
    ctx = ctx_factory()
    sid = ctx.add_system(_nacl())  # 1000 atoms at cap 2048 need about 4.1 M ints > 2^21
    with pytest.raises(rbmd_b200.RbmdError) as e:
        ctx.rbl_lists_static(sid, cap=2048)
    assert e.value.code == A.ERR_ARG
    assert "8 MiB" in str(e.value)
    _same_lists(ctx.rbl_lists(sid, cap=CAP), ctx.rbl_lists_static(sid, cap=CAP))
