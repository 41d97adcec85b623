"""Known-answer tests that pin the FP64 oracle (the reference itself cannot run here: VTK-m is
absent, and its own tests pin an older framework).  CPU only."""
import math

import numpy as np
import pytest

from rbmd_b200 import _abi as A
from rbmd_b200 import synth


def test_philox_known_answers(oracle_mod):
    """Philox4x32-10 against the published known-answer vectors of Salmon et al. (Random123)."""
    import ctypes as C
    from rbmd_b200._abi import Params  # noqa: F401  (ensures the ABI module imports)
    L = oracle_mod.lib()
    # the oracle exports no raw Philox entry; exercise it through a tiny helper compiled in
    import oracle_ffi
    kat = oracle_ffi.philox_kat
    assert kat([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert kat([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert kat([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == \
        [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def _two_atoms(r, eps=1.0, sig=1.0):
    pos = np.array([[5.0, 5.0, 5.0], [5.0 + r, 5.0, 5.0]])
    sd = synth.SystemData(pos, [1.0, 1.0], [0, 0], [eps], [sig], [0, 0, 0], [10, 10, 10])
    sd.params = A.default_params(neighbor=A.NEIGH_VERLET, cut_off=2.5, r_core=2.5)
    return sd


@pytest.mark.parametrize("r", [0.95, 1.1224620483, 1.5, 2.4])
def test_two_atom_lj_closed_form(oracle_mod, r):
    o = oracle_mod.Oracle(_two_atoms(r))
    o.compute_forces()
    f = o.forces()
    fmag = 24 * (2 * r ** -12 - r ** -6) / r  # repulsive along +x on atom 1
    assert f[1, 0] == pytest.approx(fmag, rel=1e-12, abs=1e-12)
    assert f[0, 0] == pytest.approx(-fmag, rel=1e-12, abs=1e-12)
    th = o.thermo()
    e = 4 * (r ** -12 - r ** -6)
    assert th["e_lj"] * 2 == pytest.approx(e, rel=1e-12, abs=1e-14)


def _rocksalt(n_side, spacing=1.0, alpha=1.2, rc=None, kmax=13):
    n = n_side ** 3
    g = np.arange(n_side)
    ijk = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos = (ijk + 0.5) * spacing
    q = np.where(ijk.sum(1) % 2 == 0, 1.0, -1.0)
    L = n_side * spacing
    sd = synth.SystemData(pos, np.ones(n), (q < 0).astype(int), [0.0, 0.0], [1.0, 1.0], [0, 0, 0],
                          [L, L, L], charge=q)
    sd.params = A.default_params(force_field=A.FF_LJ_CUT_COUL_LONG, neighbor=A.NEIGH_VERLET,
                                 coulomb=A.COUL_EWALD, alpha=alpha, kmax=(kmax,) * 3,
                                 cut_off=rc if rc else L / 2 - 0.1, r_core=rc if rc else L / 2 - 0.1)
    return sd


def test_madelung_constant(oracle_mod):
    """Rock salt: Coulomb energy per ion = -M q^2 / (2 r0) with M = 1.747565 (NaCl)."""
    o = oracle_mod.Oracle(_rocksalt(8))
    o.init()
    th = o.thermo()
    e_atom = th["e_coul_near"] + th["e_coul_far"]
    M = -2.0 * e_atom
    assert M == pytest.approx(1.747565, abs=2e-6)


def test_ewald_alpha_independence(oracle_mod):
    """Total Coulomb energy and force of a disordered charge set do not depend on alpha once the
    real- and reciprocal-space sums converge."""
    rng = np.random.default_rng(3)
    sd = _rocksalt(6, spacing=1.2, alpha=2.0, kmax=18)
    sd.pos += rng.normal(scale=0.15, size=sd.pos.shape)
    sd.pos %= sd.box_hi[0]
    res = []
    for alpha in (2.0, 2.6):
        sd2 = sd.copy()
        sd2.params.alpha = alpha
        o = oracle_mod.Oracle(sd2)
        o.init()
        th = o.thermo()
        f = o.forces()
        res.append((th["e_coul_near"] + th["e_coul_far"], f))
    assert res[0][0] == pytest.approx(res[1][0], rel=1e-8)
    df = np.abs(res[0][1] - res[1][1]).max() / np.abs(res[0][1]).max()
    assert df < 1e-6


def test_rbl_lists_partition_full_list(oracle_mod):
    """With pice_num 1 the RBL core and shell lists partition the full list (RunWorklet.cpp:955-970)."""
    sd = synth.lj_fcc(cells=4, seed=5)
    rng = np.random.default_rng(0)
    sd.pos += rng.normal(scale=0.1, size=sd.pos.shape)
    sd.pos %= sd.box_hi[0]
    o = oracle_mod.Oracle(sd)
    assert o.derived()["pice_num"] == 1
    nc, ns, ids = o.rbl_lists()
    L = sd.box_hi[0]
    for i in range(0, sd.n, 7):
        d = sd.pos - sd.pos[i]
        d -= L * np.round(d / L)
        r2 = (d * d).sum(1)
        full = set(np.nonzero((2.5 ** 2 - r2 > 1e-4) & (r2 > 1e-4))[0])
        core = set(np.nonzero((1.2 ** 2 - r2 > 1e-4) & (r2 > 1e-4))[0])
        got_core = set(ids[i, :nc[i]])
        got_all = set(ids[i, :nc[i] + ns[i]])
        assert got_core == core
        assert got_all == full


def test_rbl_stride_pick_counts(oracle_mod):
    """pice_num > 1: the shell list holds every pice-th shell atom, ceil(n_shell / pice) of them."""
    sd = synth.spce_water(n_mol=1000, seed=2)
    o = oracle_mod.Oracle(sd)
    d = o.derived()
    assert d["pice_num"] > 1
    nc, ns, ids = o.rbl_lists(cap=2048)
    L = sd.box_hi[0]
    for i in range(0, sd.n, 97):
        dd = sd.pos - sd.pos[i]
        dd -= L * np.round(dd / L)
        r2 = (dd * dd).sum(1)
        nshell = int(((100.0 - r2 > 1e-4) & (r2 - 25.0 > 1e-4)).sum())
        assert ns[i] == (nshell + d["pice_num"] - 1) // d["pice_num"]


def test_eam_splines_match_johnson(oracle_mod):
    """funcfl tabulation + file2array/array2spline reproduce the analytic Johnson functions, one grid
    step ahead: ReadPotentialFile stores funcfl values 0-based (ExecutionNVT.cpp:915-928) while
    file2array interpolates them as 1-based (:952-965), so the table at r holds f(r + dr)."""
    body = synth.johnson_funcfl()
    eam = oracle_mod.eam_splines(body)
    f, phi, F, df, dphi, dF = synth.johnson_functions()
    rr = np.linspace(1.8, 4.9, 17)
    rs = eam["rhor_spline"].reshape(-1, 7)
    zs = eam["z2r_spline"].reshape(-1, 7)
    for r in rr:
        p = r / eam["dr"] + 1.0
        m = min(int(p), eam["nr"] - 1)
        p = min(p - m, 1.0)
        c = rs[m]
        rho = ((c[3] * p + c[4]) * p + c[5]) * p + c[6]
        drho = (c[0] * p + c[1]) * p + c[2]
        rs_ = r + eam["dr"]
        assert rho == pytest.approx(f(rs_), rel=1e-7)
        assert drho == pytest.approx(df(rs_), rel=1e-5)
        z = zs[m]
        z2 = ((z[3] * p + z[4]) * p + z[5]) * p + z[6]
        assert z2 == pytest.approx(rs_ * phi(rs_), rel=1e-7)
    fs = eam["frho_spline"].reshape(-1, 7)
    for rho in (6.0, 12.0, 18.0):
        p = rho / eam["drho"] + 1.0
        m = max(1, min(int(p), eam["nrho"] - 1))
        p = min(p - m, 1.0)
        c = fs[m]
        rr_ = rho + eam["drho"]
        assert ((c[3] * p + c[4]) * p + c[5]) * p + c[6] == pytest.approx(F(rr_), rel=1e-7)
        assert (c[0] * p + c[1]) * p + c[2] == pytest.approx(dF(rr_), rel=1e-4)


def test_rbe_mean_force_is_unbiased(oracle_mod):
    """The RBE k-space force averaged over independent Philox streams converges to the Ewald
    k-space force (RBE is an unbiased estimator).  For an unbiased estimator the squared error of
    the mean of K samples is tr(Cov) / K, with tr(Cov) estimated from the samples' own spread, so
    z = |mean - Ewald|^2 / (V / K) is about 1 (1.1 here); a bias b adds |b|^2 K / V, so z < 3 rejects
    a bias of 1.5% of the Ewald force and more (a 2% scale error gives z = 4.8 at K = 2400)."""
    sd = synth.nacl_melt(n_side=4, rho=0.6, P=40, alpha=0.6)
    rng = np.random.default_rng(1)
    sd.pos += rng.normal(scale=0.2, size=sd.pos.shape)
    sd.pos %= sd.box_hi[0]
    sd.params.kmax[:] = (12, 12, 12)
    sd.params.coulomb = A.COUL_EWALD
    ew = oracle_mod.Oracle(sd)
    ewald = ew.ewald_kspace_force()
    sd.params.coulomb = A.COUL_RBE
    K = 4000
    samples = np.empty((K,) + ewald.shape)
    for k in range(K):
        sd2 = sd.copy()
        sd2.params.seed = 1000 + k
        o = oracle_mod.Oracle(sd2)
        o.compute_forces()
        samples[k] = o.force_part(1)
    mean = samples.mean(0)
    var = ((samples - mean) ** 2).sum() / (K - 1)
    z = ((mean - ewald) ** 2).sum() / (var / K)
    assert z < 3.0, z
    err = np.sqrt(((mean - ewald) ** 2).sum() / (ewald ** 2).sum())
    assert err < 0.02, err


def test_shake_holds_water_geometry(oracle_mod):
    sd = synth.spce_water(n_mol=64, seed=3, P=20)
    o = oracle_mod.Oracle(sd)
    o.init()
    o.step(5)
    assert o.status() == 0
    x, v, _ = o.state()
    L = sd.box_hi[0]
    tri = sd.angle_atoms.reshape(-1, 3)
    def dist(a, b):
        d = x[a] - x[b]
        d -= L * np.round(d / L)
        return np.sqrt((d * d).sum(1))
    hh = math.sqrt(2 - 2 * math.cos(math.radians(109.47)))
    assert np.abs(dist(tri[:, 0], tri[:, 1]) - 1.0).max() < 1e-4
    assert np.abs(dist(tri[:, 2], tri[:, 1]) - 1.0).max() < 1e-4
    assert np.abs(dist(tri[:, 0], tri[:, 2]) - hh).max() < 1e-4


def test_nve_energy_drift_small(oracle_mod):
    sd = synth.lj_fcc(cells=4, T=0.7)
    sd.params.neighbor = A.NEIGH_VERLET
    sd.params.cut_off = sd.params.r_core = 2.5
    sd.params.timestep = 0.002
    o = oracle_mod.Oracle(sd)
    o.init()
    e0 = o.thermo()["total_energy"]
    o.step(100)
    e1 = o.thermo()["total_energy"]
    assert abs(e1 - e0) / abs(e0) < 2e-3


def test_nose_hoover_moves_toward_target(oracle_mod):
    sd = synth.lj_fcc(cells=4, T=0.5)
    sd.params.temp_ctrl = A.TC_NOSE_HOOVER
    sd.params.temperature[:] = (1.5, 1.5, 0.05)
    o = oracle_mod.Oracle(sd)
    o.init()
    t0 = o.thermo()["temperature"]
    o.step(200)
    t1 = o.thermo()["temperature"]
    assert abs(t1 - 1.5) < abs(t0 - 1.5)


def _npt(sd, p_start=0.5, p_stop=0.5, p_damp=0.5, bulk=10.0, num_steps=100):
    p = sd.params
    p.ensemble, p.temp_ctrl, p.press_ctrl = A.ENS_NPT, A.TC_BERENDSEN, A.PC_BERENDSEN
    p.pressure[:] = (p_start, p_stop, p_damp)
    p.bulk_modulus = bulk
    p.num_steps = num_steps
    return sd


def test_berendsen_barostat_one_step_closed_form(oracle_mod):
    """One NPT step = the Berendsen NVT step followed by the dilation
    mu = (1 - dt/P_damp (P_target - P) / B)^(1/3) about the box centre, atoms carried along in
    reduced coordinates (ExecutionNPT.cpp:1334-1368, 1506-1538)."""
    base = synth.lj_fcc(cells=5)
    base.params.temp_ctrl = A.TC_BERENDSEN
    nvt = oracle_mod.Oracle(base.copy())
    nvt.init()
    nvt.step(1)
    x_nvt, v_nvt, img_nvt = nvt.state()
    sd = _npt(base.copy(), p_start=0.2, p_stop=1.2, num_steps=50)
    o = oracle_mod.Oracle(sd)
    o.init()
    o.step(1)
    t = o.thermo()
    P = t["pressure"]
    assert P == pytest.approx(nvt.thermo()["pressure"], rel=1e-12)  # the NVT step's own pressure
    target = 0.2 + (1 / 50) * (1.2 - 0.2)
    mu = (1 - sd.params.timestep / 0.5 * (target - P) / 10.0) ** (1 / 3)
    lo0, hi0 = base.box_lo, base.box_hi
    ctr = 0.5 * (lo0 + hi0)
    lo1, hi1 = (lo0 - ctr) * mu + ctr, (hi0 - ctr) * mu + ctr
    assert np.allclose(t["box_lo"], lo1, rtol=0, atol=1e-13) and np.allclose(t["box_hi"], hi1, rtol=0, atol=1e-13)
    assert t["volume"] == pytest.approx(np.prod(hi1 - lo1), rel=1e-13)
    lam = (x_nvt - lo0) / (hi0 - lo0)
    x1 = lam * (hi1 - lo1) + lo1
    x, v, img = o.state()
    wrap = np.floor((x1 - lo1) / (hi1 - lo1))
    assert np.allclose(x, x1 - wrap * (hi1 - lo1), rtol=0, atol=1e-12)
    assert np.array_equal(img, img_nvt + wrap.astype(np.int32))
    assert np.array_equal(v, v_nvt)  # the barostat leaves velocities alone
    assert t["status"] == 0


def test_berendsen_barostat_moves_volume_toward_target(oracle_mod):
    """While the pressure stays above the target the box grows every step; below it, it shrinks
    (the fcc start melts within these steps, so the pressure itself is not monotone)."""
    for target, grows in ((0.2, True), (3.0, False)):
        o = oracle_mod.Oracle(_npt(synth.lj_fcc(cells=5), p_start=target, p_stop=target, p_damp=0.2))
        o.init()
        vols = [o.thermo()["volume"]]
        for _ in range(30):
            o.step(1)
            t = o.thermo()
            assert (t["pressure"] > target) == grows
            vols.append(t["volume"])
        d = np.diff(vols)
        assert (d > 0).all() if grows else (d < 0).all()


def test_barostat_refuses_boxes_outside_the_cell_range(oracle_mod):
    """A dilation past 1.25x (or below 0.8x) the initial edge leaves the box alone and sets
    RBMD_STATUS_BOX_RANGE."""
    sd = _npt(synth.lj_fcc(cells=5), p_start=-1e6, p_stop=-1e6, p_damp=0.01, bulk=1.0)
    o = oracle_mod.Oracle(sd)
    o.init()
    o.step(1)
    t = o.thermo()
    assert t["status"] & A.STATUS_BOX_RANGE
    assert list(t["box_lo"]) == list(sd.box_lo) and list(t["box_hi"]) == list(sd.box_hi)


def _mtk(sd, p_target, p_damp, num_steps=100):
    p = sd.params
    p.ensemble, p.temp_ctrl, p.press_ctrl = A.ENS_NPT, A.TC_NOSE_HOOVER, A.PC_NOSE_HOOVER
    p.pressure[:] = (p_target, p_target, p_damp)
    p.num_steps = num_steps
    return sd


def test_mtk_with_a_heavy_barostat_is_the_nose_hoover_step(oracle_mod):
    """With P_damp huge the barostat mass (N+1) kT P_damp^2 freezes omega_dot at ~0: the MTK step
    (ExecutionNPT.cpp:1671-1741) must then reduce to the NVT Nose-Hoover step."""
    base = synth.nacl_melt(n_side=8)
    base.params.temp_ctrl = A.TC_NOSE_HOOVER
    nvt = oracle_mod.Oracle(base.copy())
    o = oracle_mod.Oracle(_mtk(base.copy(), 0.0, 1e9))
    for s in (nvt, o):
        s.init()
        s.step(10)
    x0, v0, _ = nvt.state()
    x1, v1, _ = o.state()
    assert np.abs(x1 - x0).max() < 1e-9 and np.abs(v1 - v0).max() < 1e-9
    assert o.thermo()["volume"] == pytest.approx(nvt.thermo()["volume"], rel=1e-12)


def test_mtk_volume_follows_the_pressure(oracle_mod):
    """The barostat velocity integrates (P - p_hydro) V / W: a box under a pressure above the
    (reference-weighted) target grows, below it shrinks."""
    for target, grows in ((0.0, True), (6.0, False)):
        o = oracle_mod.Oracle(_mtk(synth.lj_fcc(cells=5), target, 0.5))
        o.init()
        v0 = o.thermo()["volume"]
        o.step(20)
        t = o.thermo()
        assert (t["volume"] > v0) == grows and t["status"] == 0


def _one_dihedral(pos, K=1.7, sign=1, mult=3):
    """Four CVFF atoms with every term but one harmonic dihedral switched off."""
    sd = synth.alkane_chains(n_side=1, length=4, jiggle=0.0, coulomb=A.COUL_EWALD, neighbor=A.NEIGH_VERLET,
                             cut_off=8.0, r_core=8.0, kmax=(2, 2, 2))
    sd.box_hi = np.array([30.0, 30.0, 30.0])
    sd.pos = np.ascontiguousarray(pos, np.float64)
    sd.charge = np.zeros(4)
    sd.eps = np.array([0.0])
    sd.bond_k = np.array([0.0])
    sd.angle_k = np.array([0.0])
    sd.dihedral_k = np.array([K])
    sd.dihedral_sign = np.array([sign], np.int32)
    sd.dihedral_multiplicity = np.array([mult], np.int32)
    return sd


@pytest.mark.parametrize("sign,mult", [(1, 3), (-1, 1), (1, 2), (-1, 0)])
def test_harmonic_dihedral_closed_form(oracle_mod, sign, mult):
    """E = K [1 + d cos(n phi)] with phi the IUPAC torsion, and F = -dE/dx by central differences
    (ComputeDihedralHarmonicWorklet, MolecularWorklet.h:669-973)."""
    rng = np.random.default_rng(3 + mult)
    pos = np.array([[10.0, 10.0, 10.0], [11.5, 10.2, 10.1], [12.1, 11.6, 10.0], [13.4, 11.9, 11.1]])
    pos += rng.normal(scale=0.2, size=pos.shape)
    K = 1.7
    sd = _one_dihedral(pos, K, sign, mult)
    o = oracle_mod.Oracle(sd)
    o.compute_forces()
    b1, b2, b3 = pos[1] - pos[0], pos[2] - pos[1], pos[3] - pos[2]
    n1, n2 = np.cross(b1, b2), np.cross(b2, b3)
    phi = np.arctan2(np.dot(np.cross(n1, n2), b2 / np.linalg.norm(b2)), np.dot(n1, n2))
    e = o.thermo()["e_dihedral"]
    expect = K * (1 + (1.0 if sign == 1 else -1.0) * np.cos(mult * phi)) if mult > 0 else K * (1 + (1.0 if sign == 1 else -1.0))
    assert e == pytest.approx(expect, rel=1e-12, abs=1e-12)
    f = o.forces()
    h = 1e-6
    for a in range(4):
        for k in range(3):
            ep, em = pos.copy(), pos.copy()
            ep[a, k] += h
            em[a, k] -= h
            energies = []
            for q in (ep, em):
                oq = oracle_mod.Oracle(_one_dihedral(q, K, sign, mult))
                oq.compute_forces()
                energies.append(oq.thermo()["e_dihedral"])
            assert f[a, k] == pytest.approx(-(energies[0] - energies[1]) / (2 * h), rel=1e-5, abs=1e-7)
    assert np.abs(f.sum(0)).max() < 1e-12  # no net force


# ------------------------------------------------------------------ trajectory observables
def _radii(radius, dr):
    """RDFOutput.cpp:42-53: (int)(radius / dr) values, dr added once per bin."""
    out, r = [], 0.0
    for _ in range(int(radius / dr)):
        r += dr
        out.append(r)
    return np.array(out)


@pytest.mark.parametrize("radius,dr", [(10.0, 0.1), (2.5, 0.01), (1.0, 0.3), (3.0, 3.0)])
def test_rdf_bins_accumulate(oracle_mod, radius, dr):
    r = oracle_mod.rdf_bins(radius, dr)
    assert np.array_equal(r, _radii(radius, dr))
    with pytest.raises(ValueError):
        oracle_mod.rdf_bins(0.05, 0.1)


def test_rdf_counts_simple_cubic_shells(oracle_mod):
    """Known answer: a simple cubic lattice of spacing a in a periodic box of 4 a has, around every
    atom, 6 / 12 / 8 / 6 / 24 / 24 images at a sqrt(1..6); a bin counts a shell when
    r_b < a sqrt(m) < 1.01 r_b.  a = 1.003 keeps every shell away from the bin edges."""
    a, m = 1.003, 4
    g = np.arange(m) * a + 0.5 * a
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    n = x.shape[0]
    radius, dr = 2.5, 0.01
    r = _radii(radius, dr)
    counts = oracle_mod.rdf_counts(x, np.arange(n), [m * a] * 3, np.arange(n), np.arange(n), radius, dr)
    expect = np.zeros(r.size, np.int64)
    for mm, z in ((1, 6), (2, 12), (3, 8), (4, 6), (5, 24), (6, 24)):
        d = a * math.sqrt(mm)
        expect[(r < d) & (d < r + r * 0.01)] += n * z
    assert counts.sum() > 0 and np.array_equal(counts, expect)


def _rdf_numpy(x, mol, L, centers, targets, radius, dr, exclude):
    """Independent restatement (vectorised over pairs, images -2..2) of the RDF pair count."""
    r = _radii(radius, dr)
    u = r + r * 0.01
    R = u[-1]
    counts = np.zeros(r.size, np.int64)
    xc, xt = x[centers], x[targets]
    base = xt[None, :, :] - xc[:, None, :]
    keep = np.ones((len(centers), len(targets)), bool)
    if exclude:
        keep = mol[centers][:, None] != mol[targets][None, :]
    for nx in range(-2, 3):
        for ny in range(-2, 3):
            for nz in range(-2, 3):
                d = base + np.array([nx * L[0], ny * L[1], nz * L[2]])
                inside = keep & (np.abs(d) < R).all(-1)
                dis = np.sqrt(d[..., 0] * d[..., 0] + d[..., 1] * d[..., 1] + d[..., 2] * d[..., 2])[inside]
                counts += ((dis[:, None] > r[None, :]) & (dis[:, None] < u[None, :])).sum(0)
    return counts


@pytest.mark.parametrize("exclude", [True, False])
def test_rdf_counts_match_independent_count(oracle_mod, exclude):
    rng = np.random.default_rng(7)
    n = 120
    L = np.array([6.0, 7.0, 5.5])
    x = rng.uniform(0, 1, (n, 3)) * L
    mol = np.repeat(np.arange(n // 3), 3)
    types = rng.integers(0, 2, n)
    c, t = np.flatnonzero(types == 0), np.flatnonzero(types == 1)
    got = oracle_mod.rdf_counts(x, mol, L, c, t, 3.0, 0.05, exclude)
    assert np.array_equal(got, _rdf_numpy(x, mol, L, c, t, 3.0, 0.05, exclude))
    # a radius beyond half the box reaches more than one image of a pair
    got = oracle_mod.rdf_counts(x, mol, L, c, t, 4.5, 0.1, exclude)
    assert np.array_equal(got, _rdf_numpy(x, mol, L, c, t, 4.5, 0.1, exclude))


def test_rdf_ideal_gas_is_flat(oracle_mod):
    """Uniform random points: the normalised RDF (OutPutWorklet.cpp:303-306) averages to 1."""
    from rbmd_b200 import rdf_snapshot
    rng = np.random.default_rng(3)
    n, Lb = 400, 8.0
    x = rng.uniform(0, Lb, (n, 3))
    ids = np.arange(n)
    radius, dr = 3.5, 0.05
    counts = oracle_mod.rdf_counts(x, ids, [Lb] * 3, ids, ids, radius, dr, True)
    g = rdf_snapshot(counts, _radii(radius, dr), n, n, Lb ** 3)
    assert abs(g[20:].mean() - 1.0) < 0.03


def test_msd_vacf_match_numpy(oracle_mod):
    rng = np.random.default_rng(5)
    n = 64
    L = np.array([4.0, 5.0, 6.0])
    x0, x = rng.uniform(0, 1, (n, 3)) * L, rng.uniform(0, 1, (n, 3)) * L
    img0, img = rng.integers(-2, 3, (n, 3)), rng.integers(-2, 3, (n, 3))
    v0, v = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
    msd, vacf = oracle_mod.msd_vacf(x0, img0, v0, x, img, v, L)
    d = x + (img - img0) * L - x0
    assert np.allclose(msd, [*(d ** 2).mean(0), (d ** 2).sum(1).mean()], rtol=1e-13)
    w = v0 * v
    assert np.allclose(vacf, [*w.mean(0), w.sum(1).mean()], rtol=1e-13)


# ------------------------------------------------------------------ setfl (eam/alloy) EAM
def _row(tab, x, delta, n):
    p = x / delta + 1.0
    m = min(int(p), n - 1)
    p = min(p - m, 1.0)
    c = tab[m]
    return ((c[3] * p + c[4]) * p + c[5]) * p + c[6], (c[0] * p + c[1]) * p + c[2]


def test_setfl_splines_match_johnson(oracle_mod):
    """setfl tables are splined on the file's grid with no resampling (LAMMPS eam/alloy
    file2array), so unlike funcfl they reproduce f(r), r phi(r) and F(rho) at r itself; the
    cross pair carries the mixing rule; type t takes element type_element[t]."""
    body = synth.johnson_setfl(n=4000)
    te = [1, 0]  # type 0 is element B, type 1 is Cu
    eam = oracle_mod.setfl_splines(body, te)
    nr, nrho, dr, drho = eam["nr"], eam["nrho"], eam["dr"], eam["drho"]
    rs = eam["rhor_spline"].reshape(2, -1, 7)
    zs = eam["z2r_spline"].reshape(3, -1, 7)
    fs = eam["frho_spline"].reshape(2, -1, 7)
    funcs = [synth.johnson_functions(synth.JOHNSON_B), synth.johnson_functions(synth.JOHNSON_CU)]
    for r in np.linspace(1.8, 4.9, 13):
        for t in range(2):
            f, phi, F, df, dphi, dF = funcs[t]
            rho, drho_dr = _row(rs[t], r, dr, nr)
            assert rho == pytest.approx(f(r), rel=1e-7)
            assert drho_dr == pytest.approx(df(r), rel=1e-4)
            z2, _ = _row(zs[t * (t + 1) // 2 + t], r, dr, nr)
            assert z2 == pytest.approx(r * phi(r), rel=1e-7)
        fa, pa = funcs[0][0](r), funcs[0][1](r)
        fb, pb = funcs[1][0](r), funcs[1][1](r)
        z2, _ = _row(zs[1], r, dr, nr)  # types (1, 0)
        assert z2 == pytest.approx(r * 0.5 * (fb / fa * pa + fa / fb * pb), rel=1e-7)
    for t in range(2):
        F = funcs[t][2]
        for rho in (6.0, 12.0, 18.0):
            v, _ = _row(fs[t], rho, drho, nrho)
            assert v == pytest.approx(F(rho), rel=1e-6)
    assert eam["rhomax"] == pytest.approx((nrho - 1) * drho)


def test_setfl_alloy_forces_are_energy_gradients(oracle_mod):
    """Per-type densities, embedding and pair tables: the oracle's forces are minus the gradient
    of its EAM energy (Verlet neighbours, so every pair within the cutoff counts)."""
    sd = synth.eam_alloy(cells=3, frac_b=0.4, build_splines=oracle_mod.setfl_splines,
                         neighbor=A.NEIGH_VERLET, cut_off=4.9, r_core=4.9)
    sd.eam["cut"] = 4.9
    rng = np.random.default_rng(2)
    sd.pos = sd.pos + rng.normal(scale=0.05, size=sd.pos.shape)
    assert (sd.types == 1).any() and (sd.types == 0).any()
    o = oracle_mod.Oracle(sd)
    o.compute_forces()
    f = o.forces()
    n = sd.n

    def energy(pos):
        s2 = sd.copy()
        s2.pos = pos
        oo = oracle_mod.Oracle(s2)
        oo.compute_forces()
        return oo.thermo()["e_eam"] * n

    h = 1e-5
    for i, k in ((0, 0), (7, 1), (31, 2), (50, 0)):
        p1, p2 = sd.pos.copy(), sd.pos.copy()
        p1[i, k] += h
        p2[i, k] -= h
        g = -(energy(p1) - energy(p2)) / (2 * h)
        assert f[i, k] == pytest.approx(g, rel=2e-5, abs=1e-6)
