"""Seeded synthetic systems for the five benchmark workloads and the tests.

Each builder returns a `SystemData` holding numpy arrays in the layout of `rbmd_system_desc`
(include/rbmd_gpu.h) plus the matching `rbmd_params`.  No public dataset is involved: every system
is generated from a seed (the reference ships no benchmark inputs, and its bundled data files are
read by the data-file reader, not by these builders).

Workloads (sizes exactly as named):
  * lj_fcc        LJ fluid, 4000 atoms, fcc 10x10x10x4, rho* 0.8442, T* 1.44, rc 2.5, RBL rs 1.2
  * nacl_melt     rock-salt melt, 20^3 simple-cubic alternating +1/-1, rho 0.6, RBE alpha 0.6 P 200
  * spce_water    3000 SPC/E molecules, 1.0 g/cm^3, RBE alpha 0.09 (beta 0.3/A) P 100, SHAKE
  * eam_cu        fcc Cu 20^3 x 4 = 32000 atoms, Johnson-form EAM tabulated to 5.0 A
  * saline        SPC/E + 0.15 M NaCl (Joung-Cheatham 2008 SPC/E ion parameters)
"""
import ctypes as C
import math

import numpy as np

from . import _abi as A

# physical constants for REAL units (g/mol, A, fs, kcal/mol)
AVOGADRO = 6.02214076e23
KB_REAL = 1.9872067e-3
MVV2E_REAL = 1.0 / 4.186e-4

M_O, M_H, M_NA, M_CL, M_CU = 15.9994, 1.008, 22.98977, 35.453, 63.546
SPCE = dict(q_o=-0.8476, q_h=0.4238, sigma_o=3.166, eps_o=0.1553, r_oh=1.0, theta=109.47)
# Joung & Cheatham, J. Phys. Chem. B 112, 9020 (2008), SPC/E set: sigma = Rmin / 2^(1/6)
ION_NA = dict(sigma=2.1595, eps=0.3526418, q=1.0, mass=M_NA)
ION_CL = dict(sigma=4.8305, eps=0.0127850, q=-1.0, mass=M_CL)


class SystemData:
    """Host-side arrays of one system; `desc()` returns an rbmd_system_desc pointing into them."""

    def __init__(self, pos, mass, types, eps, sig, box_lo, box_hi, vel=None, charge=None,
                 molecule=None, params=None, name="system"):
        self.name = name
        self.pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        n = self.pos.shape[0]
        self.mass = np.ascontiguousarray(mass, dtype=np.float64).reshape(n)
        self.types = np.ascontiguousarray(types, dtype=np.int32).reshape(n)
        self.eps = np.ascontiguousarray(eps, dtype=np.float64)
        self.sig = np.ascontiguousarray(sig, dtype=np.float64)
        self.box_lo = np.asarray(box_lo, dtype=np.float64)
        self.box_hi = np.asarray(box_hi, dtype=np.float64)
        self.vel = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64).reshape(n, 3)
        self.charge = None if charge is None else np.ascontiguousarray(charge, dtype=np.float64)
        self.molecule = None if molecule is None else np.ascontiguousarray(molecule, dtype=np.int32)
        self.image = None
        self.bond_atoms = self.bond_type = self.bond_k = self.bond_r0 = None
        self.angle_atoms = self.angle_type = self.angle_k = self.angle_theta0 = None
        self.special_offsets = self.special_ids = self.special_weights = None
        self.dihedral_atoms = self.dihedral_type = self.dihedral_k = None
        self.dihedral_sign = self.dihedral_multiplicity = None
        self.eam = None
        self.near_table_values = None  # float32 [2048] G by key (params.near_table), or None: the library's
        self.params = params if params is not None else A.default_params()
        self._desc = None

    @property
    def n(self):
        return self.pos.shape[0]

    def copy(self):
        import copy
        other = copy.copy(self)
        for k, v in self.__dict__.items():
            if isinstance(v, np.ndarray):
                setattr(other, k, v.copy())
        other.params = A.Params.from_buffer_copy(self.params)
        other._desc = None
        if self.eam is not None:
            other.eam = dict(self.eam)
        return other

    def desc(self):
        def dp(a):
            return None if a is None else a.ctypes.data_as(A.dptr)

        def ip(a):
            return None if a is None else a.ctypes.data_as(A.iptr)

        d = A.SystemDesc()
        d.n_atoms = self.n
        d.n_types = len(self.eps)
        d.box_lo[:] = list(self.box_lo)
        d.box_hi[:] = list(self.box_hi)
        d.position = dp(self.pos)
        d.velocity = dp(self.vel)
        d.charge = dp(self.charge)
        d.mass = dp(self.mass)
        d.type = ip(self.types)
        d.molecule = ip(self.molecule)
        d.image = ip(self.image)
        d.epsilon = dp(self.eps)
        d.sigma = dp(self.sig)
        if self.bond_atoms is not None:
            d.n_bonds = len(self.bond_type)
            d.n_bond_types = len(self.bond_k)
            d.bond_atoms = ip(self.bond_atoms)
            d.bond_type = ip(self.bond_type)
            d.bond_k = dp(self.bond_k)
            d.bond_r0 = dp(self.bond_r0)
        if self.angle_atoms is not None:
            d.n_angles = len(self.angle_atoms) // 3
            d.angle_atoms = ip(self.angle_atoms)
            if self.angle_type is not None:
                d.n_angle_types = len(self.angle_k)
                d.angle_type = ip(self.angle_type)
                d.angle_k = dp(self.angle_k)
                d.angle_theta0 = dp(self.angle_theta0)
        if self.special_offsets is not None:
            d.special_offsets = ip(self.special_offsets)
            d.special_ids = ip(self.special_ids)
            d.special_weights = dp(self.special_weights)
        if self.eam is not None:
            e = self.eam
            d.eam_nrho, d.eam_nr = e["nrho"], e["nr"]
            d.eam_drho, d.eam_dr = e["drho"], e["dr"]
            d.eam_rhomax, d.eam_cut = e["rhomax"], e["cut"]
            d.eam_frho_spline = dp(e["frho_spline"])
            d.eam_rhor_spline = dp(e["rhor_spline"])
            d.eam_z2r_spline = dp(e["z2r_spline"])
            d.eam_per_type = int(e.get("per_type", 0))
        if self.near_table_values is not None:
            tab = np.ascontiguousarray(self.near_table_values, dtype=np.float32)
            assert tab.shape == (2048,)
            self.near_table_values = tab
            d.near_table_values = tab.ctypes.data_as(C.POINTER(C.c_float))
        if self.dihedral_atoms is not None:
            d.n_dihedrals = len(self.dihedral_type)
            d.n_dihedral_types = len(self.dihedral_k)
            d.dihedral_atoms = ip(self.dihedral_atoms)
            d.dihedral_type = ip(self.dihedral_type)
            d.dihedral_k = dp(self.dihedral_k)
            d.dihedral_sign = ip(self.dihedral_sign)
            d.dihedral_multiplicity = ip(self.dihedral_multiplicity)
        self._desc = d
        return d


def maxwell(mass, T, kB, mvv2e, rng):
    """Maxwell-Boltzmann velocities at T with zero centre-of-mass momentum."""
    n = len(mass)
    sd = np.sqrt(kB * T / (mass * mvv2e))
    v = rng.standard_normal((n, 3)) * sd[:, None]
    p = (v * mass[:, None]).sum(0) / mass.sum()
    return v - p[None, :]


def special_lists(n, bonds, weights):
    """special_ids/weights/offsets as ModelFileInitCondition::SetSpecialBonds builds them
    (framework/InitCondition/ModelFileInitCondition.cpp:848-923): 1-2, 1-3 and 1-4 partners
    through a symmetric multimap of the bond list, in insertion order; atoms without bonds carry
    their own id with weight 1."""
    links = [[] for _ in range(n)]
    for a, b in bonds:
        links[a].append(b)
        links[b].append(a)
    ids, ws, counts = [], [], []
    for i in range(n):
        if not links[i]:
            ids.append(i)
            ws.append(1.0)
            counts.append(1)
            continue
        c = 0
        for k1 in links[i]:
            ids.append(k1)
            ws.append(weights[0])
            c += 1
            for k2 in links[k1]:
                if k2 == i:
                    continue
                ids.append(k2)
                ws.append(weights[1])
                c += 1
                for k3 in links[k2]:
                    if k3 == k1:
                        continue
                    ids.append(k3)
                    ws.append(weights[2])
                    c += 1
        counts.append(c)
    off = np.zeros(n + 1, dtype=np.int32)
    off[1:] = np.cumsum(counts)
    return off, np.asarray(ids, dtype=np.int32), np.asarray(ws, dtype=np.float64)


# ---------------------------------------------------------------------------------- configs 1-4
def lj_fcc(cells=10, rho=0.8442, T=1.44, seed=1, **kw):
    """LJ fluid start: fcc cells^3 x 4 atoms, reduced density rho, Maxwell velocities at T."""
    a = (4.0 / rho) ** (1.0 / 3.0)
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.arange(cells)
    cell = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 1, 3)
    pos = ((cell + base[None]) * a).reshape(-1, 3) + 0.25 * a
    L = cells * a
    rng = np.random.default_rng(seed)
    n = pos.shape[0]
    mass = np.ones(n)
    vel = maxwell(mass, T, 1.0, 1.0, rng)
    params = A.default_params(force_field=A.FF_LJ_CUT, neighbor=A.NEIGH_RBL, cut_off=2.5, r_core=1.2,
                              neighbor_sample_num=100, units=A.UNITS_LJ, timestep=0.005,
                              temp_ctrl=A.TC_NONE, ensemble=A.ENS_NVE, temperature=(T, T, 1.0),
                              num_steps=1000, seed=seed)
    for k, v in kw.items():
        _set(params, k, v)
    return SystemData(pos, mass, np.zeros(n), [1.0], [1.0], [0, 0, 0], [L, L, L], vel=vel,
                      params=params, name=f"lj_fcc_{n}")


def nacl_melt(n_side=20, rho=0.6, T=2.0, seed=1, P=200, alpha=0.6, **kw):
    """Molten rock salt: n_side^3 simple cubic with alternating +1/-1 charges at reduced density."""
    n = n_side ** 3
    L = (n / rho) ** (1.0 / 3.0)
    sp = L / n_side
    g = np.arange(n_side)
    ijk = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos = (ijk + 0.5) * sp
    charge = np.where(ijk.sum(1) % 2 == 0, 1.0, -1.0)
    types = (charge < 0).astype(np.int32)
    rng = np.random.default_rng(seed)
    mass = np.ones(n)
    vel = maxwell(mass, T, 1.0, 1.0, rng)
    params = A.default_params(force_field=A.FF_LJ_CUT_COUL_LONG, neighbor=A.NEIGH_RBL, cut_off=3.0,
                              r_core=1.5, neighbor_sample_num=100, coulomb=A.COUL_RBE,
                              coulomb_sample_num=P, alpha=alpha, kmax=(6, 6, 6), units=A.UNITS_LJ,
                              timestep=0.002, temp_ctrl=A.TC_NOSE_HOOVER, temperature=(T, T, 0.2),
                              num_steps=500, seed=seed)
    for k, v in kw.items():
        _set(params, k, v)
    return SystemData(pos, mass, types, [1.0, 1.0], [1.0, 1.0], [0, 0, 0], [L, L, L], vel=vel,
                      charge=charge, params=params, name=f"nacl_{n}")


def _rotations(rng, m):
    q = rng.standard_normal((m, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((m, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z)
    R[:, 0, 1] = 2 * (x * y - z * w)
    R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w)
    R[:, 1, 1] = 1 - 2 * (x * x + z * z)
    R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w)
    R[:, 2, 1] = 2 * (y * z + x * w)
    R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def _water_block(n_sites, L, rng, water_sites, ion_sites=(), ions=()):
    """Water molecules (H, O, H order per molecule) on the cubic-lattice sites `water_sites`, ions
    on `ion_sites`.  Returns arrays in atom order: all waters first, then ions."""
    side = int(round(n_sites ** (1.0 / 3.0)))
    sp = L / side
    water_sites = np.asarray(water_sites, dtype=np.int64)
    ion_sites = np.asarray(ion_sites, dtype=np.int64)

    def site_xyz(s):
        i, r = np.divmod(s, side * side)
        j, k = np.divmod(r, side)
        return (np.stack([i, j, k], -1) + 0.5) * sp

    th = math.radians(SPCE["theta"])
    r = SPCE["r_oh"]
    local = np.array([[r * math.sin(th / 2), 0.0, r * math.cos(th / 2)], [0.0, 0.0, 0.0],
                      [-r * math.sin(th / 2), 0.0, r * math.cos(th / 2)]])
    com = (M_H * local[0] + M_H * local[2]) / (M_O + 2 * M_H)
    nw = len(water_sites)
    R = _rotations(rng, nw)
    centers = site_xyz(water_sites)
    wpos = centers[:, None, :] + np.einsum("mij,aj->mai", R, local - com[None, :])
    pos = [wpos.reshape(-1, 3)]
    types = [np.tile(np.array([1, 0, 1], np.int32), nw)]
    mass = [np.tile(np.array([M_H, M_O, M_H]), nw)]
    charge = [np.tile(np.array([SPCE["q_h"], SPCE["q_o"], SPCE["q_h"]]), nw)]
    mol = [np.repeat(np.arange(nw, dtype=np.int32), 3)]
    if len(ion_sites):
        pos.append(site_xyz(ion_sites))
        types.append(np.array([ion["type"] for ion in ions], np.int32))
        mass.append(np.array([ion["mass"] for ion in ions]))
        charge.append(np.array([ion["q"] for ion in ions]))
        mol.append(nw + np.arange(len(ion_sites), dtype=np.int32))
    pos = np.mod(np.concatenate(pos), L)
    return (pos, np.concatenate(mass), np.concatenate(types), np.concatenate(charge),
            np.concatenate(mol).astype(np.int32))


def water_special_lists(n_water, n_other, weights):
    """special_lists() of the water topology built by _water_topology, vectorised: O carries its two
    H (1-2), each H carries its O (1-2) and the other H (1-3); other atoms carry themselves."""
    w12, w13 = float(weights[0]), float(weights[1])
    m = np.arange(n_water, dtype=np.int32)
    h1, o, h2 = 3 * m, 3 * m + 1, 3 * m + 2
    ids = np.stack([o, h2, h1, h2, o, h1], -1)  # rows: H1 (o, h2), O (h1, h2), H2 (o, h1)
    ws = np.tile(np.array([w12, w13, w12, w12, w12, w13]), (n_water, 1))
    ids = ids.reshape(-1)
    ws = ws.reshape(-1)
    n = 3 * n_water + n_other
    other = np.arange(3 * n_water, n, dtype=np.int32)
    ids = np.concatenate([ids, other]).astype(np.int32)
    ws = np.concatenate([ws, np.ones(n_other)])
    counts = np.concatenate([np.full(3 * n_water, 2, np.int32), np.ones(n_other, np.int32)])
    off = np.zeros(n + 1, dtype=np.int32)
    off[1:] = np.cumsum(counts)
    return off, ids, ws


def _water_topology(sd, n_water, special=(0.0, 0.0, 0.0)):
    """Harmonic O-H bonds and H-O-H angles (SPC/E geometry) and the SHAKE triples."""
    m = np.arange(n_water, dtype=np.int32)
    h1, o, h2 = 3 * m, 3 * m + 1, 3 * m + 2
    sd.bond_atoms = np.stack([o, h1, o, h2], -1).reshape(-1).astype(np.int32)
    sd.bond_type = np.zeros(2 * n_water, np.int32)
    sd.bond_k = np.array([554.1349])
    sd.bond_r0 = np.array([SPCE["r_oh"]])
    sd.angle_atoms = np.stack([h1, o, h2], -1).reshape(-1).astype(np.int32)
    sd.angle_type = np.zeros(n_water, np.int32)
    sd.angle_k = np.array([45.7696])
    sd.angle_theta0 = np.array([SPCE["theta"]])
    sd.special_offsets, sd.special_ids, sd.special_weights = water_special_lists(
        n_water, sd.n - 3 * n_water, special)


def spce_water(n_mol=3000, density=1.0, T=300.0, seed=1, P=100, beta=0.3, **kw):
    """SPC/E water: n_mol molecules at randomly rotated simple-cubic sites, density in g/cm^3."""
    mass_tot = n_mol * (M_O + 2 * M_H) / AVOGADRO  # g
    L = (mass_tot / density) ** (1.0 / 3.0) * 1e8  # A
    side = int(math.ceil(n_mol ** (1.0 / 3.0) - 1e-9))
    n_sites = side ** 3
    rng = np.random.default_rng(seed)
    sites = np.sort(rng.choice(n_sites, size=n_mol, replace=False))
    pos, mass, types, charge, mol = _water_block(n_sites, L, rng, sites)
    vel = maxwell(mass, T, KB_REAL, MVV2E_REAL, rng)
    params = A.default_params(force_field=A.FF_CVFF, neighbor=A.NEIGH_RBL, cut_off=10.0, r_core=5.0,
                              neighbor_sample_num=100, coulomb=A.COUL_RBE, coulomb_sample_num=P,
                              alpha=beta * beta, kmax=(3, 3, 3), units=A.UNITS_REAL, timestep=1.0,
                              temp_ctrl=A.TC_NOSE_HOOVER, temperature=(T, T, 100.0),
                              fix_shake=A.SHAKE_TRUE, num_steps=1000, seed=seed,
                              special_bonds=(0.0, 0.0, 0.0))
    for k, v in kw.items():
        _set(params, k, v)
    sd = SystemData(pos, mass, types, [SPCE["eps_o"], 0.0], [SPCE["sigma_o"], 0.0], [0, 0, 0],
                    [L, L, L], vel=vel, charge=charge, molecule=mol, params=params,
                    name=f"spce_{3 * n_mol}")
    _water_topology(sd, n_mol, tuple(params.special_bonds))
    return sd


# united-atom CH2 chains (TraPPE-like LJ, CVFF harmonic bonds and angles, harmonic dihedrals
# K [1 + d cos(n phi)] with n = 3) for the bonded terms that water lacks
CH2 = dict(mass=14.027, sigma=3.95, eps=0.0914, r0=1.54, k_bond=260.0, theta=114.0, k_angle=62.1,
           k_dih=1.4, sign=1, mult=3, q=0.1)


def alkane_chains(n_side=5, length=6, spacing=11.0, T=300.0, seed=1, P=100, beta=0.3, jiggle=0.03, **kw):
    """n_side^3 all-trans CH2 chains of `length` sites at randomly rotated simple-cubic sites
    `spacing` A apart, positions jiggled by `jiggle` A so that the dihedrals carry forces, charges
    +-q alternating along each chain; bonds, angles, dihedrals and 1-2/1-3/1-4 special lists
    (weights 0, 0, 0: the reference reads special_bonds as integers) from the chain graph."""
    rng = np.random.default_rng(seed)
    half = np.deg2rad(CH2["theta"]) / 2
    step_x, step_y = CH2["r0"] * np.sin(half), CH2["r0"] * np.cos(half)
    base = np.array([[k * step_x, (k % 2) * step_y, 0.0] for k in range(length)])
    base -= base.mean(0)
    rot = _rotations(rng, n_side ** 3)
    g = np.arange(n_side)
    sites = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) * spacing + spacing / 2
    pos = (sites[:, None, :] + np.einsum("mij,kj->mki", rot, base)).reshape(-1, 3)
    pos += rng.normal(scale=jiggle, size=pos.shape)
    L = n_side * spacing
    pos %= L
    nmol = n_side ** 3
    n = nmol * length
    mass = np.full(n, CH2["mass"])
    charge = np.tile(np.where(np.arange(length) % 2 == 0, CH2["q"], -CH2["q"]), nmol)
    mol = np.repeat(np.arange(nmol), length).astype(np.int32)
    vel = maxwell(mass, T, KB_REAL, MVV2E_REAL, rng)
    params = A.default_params(force_field=A.FF_CVFF, neighbor=A.NEIGH_RBL, cut_off=10.0, r_core=5.0,
                              neighbor_sample_num=100, coulomb=A.COUL_RBE, coulomb_sample_num=P,
                              alpha=beta * beta, kmax=(3, 3, 3), units=A.UNITS_REAL, timestep=1.0,
                              temp_ctrl=A.TC_NOSE_HOOVER, temperature=(T, T, 100.0), num_steps=1000, seed=seed,
                              special_bonds=(0.0, 0.0, 0.0))
    for k, v in kw.items():
        _set(params, k, v)
    sd = SystemData(pos, mass, np.zeros(n, np.int32), [CH2["eps"]], [CH2["sigma"]], [0, 0, 0], [L, L, L], vel=vel,
                    charge=charge, molecule=mol, params=params, name=f"alkane_{n}")
    first = (np.arange(nmol) * length)[:, None, None]
    sd.bond_atoms = (first + np.stack([np.arange(length - 1), np.arange(1, length)], -1)[None]).reshape(-1).astype(np.int32)
    sd.bond_type = np.zeros(nmol * (length - 1), np.int32)
    sd.bond_k, sd.bond_r0 = np.array([CH2["k_bond"]]), np.array([CH2["r0"]])
    tri = np.stack([np.arange(length - 2), np.arange(1, length - 1), np.arange(2, length)], -1)
    sd.angle_atoms = (first + tri[None]).reshape(-1).astype(np.int32)
    sd.angle_type = np.zeros(nmol * (length - 2), np.int32)
    sd.angle_k, sd.angle_theta0 = np.array([CH2["k_angle"]]), np.array([CH2["theta"]])
    quad = np.stack([np.arange(length - 3), np.arange(1, length - 2), np.arange(2, length - 1), np.arange(3, length)], -1)
    sd.dihedral_atoms = (first + quad[None]).reshape(-1).astype(np.int32)
    sd.dihedral_type = np.zeros(nmol * (length - 3), np.int32)
    sd.dihedral_k = np.array([CH2["k_dih"]])
    sd.dihedral_sign = np.array([CH2["sign"]], np.int32)
    sd.dihedral_multiplicity = np.array([CH2["mult"]], np.int32)
    sp = tuple(params.special_bonds)
    sd.special_offsets, sd.special_ids, sd.special_weights = special_lists(n, sd.bond_atoms.reshape(-1, 2), sp)
    return sd


def saline(n_atoms_target, T=300.0, seed=1, P=100, beta=0.3, molar=0.15, precision=A.PREC_MIXED, **kw):
    """SPC/E water with `molar` NaCl at random lattice sites, close to n_atoms_target atoms."""
    waters_per_pair = 55.5 / molar
    n_pairs = max(1, int(round(n_atoms_target / (3 * waters_per_pair + 2))))
    n_water = max(8, (n_atoms_target - 2 * n_pairs) // 3)
    n_mol = n_water + 2 * n_pairs
    mass_tot = (n_water * (M_O + 2 * M_H) + n_pairs * (M_NA + M_CL)) / AVOGADRO
    L = (mass_tot / 1.0) ** (1.0 / 3.0) * 1e8
    side = int(math.ceil(n_mol ** (1.0 / 3.0) - 1e-9))
    n_sites = side ** 3
    rng = np.random.default_rng(seed)
    sites = rng.choice(n_sites, size=n_mol, replace=False)
    water_sites = np.sort(sites[:n_water])
    ion_sites = sites[n_water:]
    ions = [dict(type=2, **ION_NA)] * n_pairs + [dict(type=3, **ION_CL)] * n_pairs
    pos, mass, types, charge, mol = _water_block(n_sites, L, rng, water_sites, ion_sites, ions)
    vel = maxwell(mass, T, KB_REAL, MVV2E_REAL, rng)
    params = A.default_params(force_field=A.FF_CVFF, neighbor=A.NEIGH_RBL, cut_off=10.0, r_core=5.0,
                              neighbor_sample_num=100, coulomb=A.COUL_RBE, coulomb_sample_num=P,
                              alpha=beta * beta, kmax=(3, 3, 3), units=A.UNITS_REAL, timestep=1.0,
                              temp_ctrl=A.TC_NOSE_HOOVER, temperature=(T, T, 100.0),
                              fix_shake=A.SHAKE_TRUE, num_steps=1000, seed=seed,
                              special_bonds=(0.0, 0.0, 0.0), precision=precision)
    for k, v in kw.items():
        _set(params, k, v)
    eps = [SPCE["eps_o"], 0.0, ION_NA["eps"], ION_CL["eps"]]
    sig = [SPCE["sigma_o"], 0.0, ION_NA["sigma"], ION_CL["sigma"]]
    sd = SystemData(pos, mass, types, eps, sig, [0, 0, 0], [L, L, L], vel=vel, charge=charge,
                    molecule=mol, params=params, name=f"saline_{len(mass)}")
    _water_topology(sd, n_water, tuple(params.special_bonds))
    return sd


# Johnson-form analytic EAM for Cu (parameters as named by the benchmark configuration)
JOHNSON_CU = dict(re=2.556, fe=1.0, beta=5.85, gamma=8.0, phi_e=0.59, E_c=3.54, rho_e=12.0)


def johnson_functions(par=JOHNSON_CU):
    re, fe, be, ga, phe, Ec, rhe = (par[k] for k in ("re", "fe", "beta", "gamma", "phi_e", "E_c", "rho_e"))
    f = lambda r: fe * np.exp(-be * (r / re - 1.0))
    phi = lambda r: phe * np.exp(-ga * (r / re - 1.0))
    F = lambda rho: -Ec * np.sqrt(np.maximum(rho, 0.0) / rhe)
    df = lambda r: -be / re * f(r)
    dphi = lambda r: -ga / re * phi(r)
    dF = lambda rho: -Ec * 0.5 / np.sqrt(np.maximum(rho, 1e-300) * rhe)
    return f, phi, F, df, dphi, dF


def johnson_funcfl(n=10000, cut=5.0, rho_max=None, par=JOHNSON_CU):
    """Tabulate the Johnson functions as a funcfl file body: F on an nrho grid, Z(r) with
    27.2*0.529*Z^2 = r*phi(r) (so the funcfl z2r conversion of the reader gives r*phi), rho(r)."""
    f, phi, F, *_ = johnson_functions(par)
    if rho_max is None:
        rho_max = 3.0 * par["rho_e"]
    dr = cut / (n - 1)
    drho = rho_max / (n - 1)
    r = np.arange(n) * dr
    rr = np.where(r > 0, r, dr * 1e-3)
    rhor = f(rr)
    z = np.sqrt(rr * phi(rr) / (27.2 * 0.529))
    frho = F(np.arange(n) * drho)
    return dict(nrho=n, drho=drho, nr=n, dr=dr, cut=cut, frho=frho, zr=z, rhor=rhor)


def eam_cu(cells=20, a=3.615, T=600.0, seed=1, build_splines=None, **kw):
    """fcc Cu, cells^3 x 4 atoms, Johnson EAM; `build_splines(file_dict) -> eam dict` turns the
    tabulated functions into the reference's Vec7 spline rows (rbmd_eam_build_splines)."""
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.arange(cells)
    cell = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 1, 3)
    pos = ((cell + base[None]) * a).reshape(-1, 3) + 0.25 * a
    L = cells * a
    n = pos.shape[0]
    rng = np.random.default_rng(seed)
    mass = np.full(n, M_CU)
    kB, mvv2e = 8.617343e-5, 1.0364269e-4
    vel = maxwell(mass, T, kB, mvv2e, rng)
    params = A.default_params(force_field=A.FF_EAM, neighbor=A.NEIGH_RBL, cut_off=5.0, r_core=2.5,
                              neighbor_sample_num=100, units=A.UNITS_METAL, timestep=0.002,
                              temp_ctrl=A.TC_NOSE_HOOVER, temperature=(T, T, 0.1), num_steps=1000,
                              seed=seed, precision=A.PREC_MIXED)
    for k, v in kw.items():
        _set(params, k, v)
    sd = SystemData(pos, mass, np.zeros(n), [0.0], [0.0], [0, 0, 0], [L, L, L], vel=vel,
                    params=params, name=f"eam_cu_{n}")
    if build_splines is not None:
        sd.eam = build_splines(johnson_funcfl())
    return sd


# A second Johnson-form element for two-element (setfl) tests: synthetic parameters, not fitted to
# any metal.
JOHNSON_B = dict(re=2.49, fe=1.15, beta=6.1, gamma=8.6, phi_e=0.52, E_c=4.1, rho_e=13.5)
M_B = 58.69


def johnson_setfl(elements=(JOHNSON_CU, JOHNSON_B), masses=(M_CU, M_B), names=("Cu", "B"), n=2000, cut=5.0):
    """Tabulate Johnson functions of several elements as a setfl body: F_e on the nrho grid,
    rho_e(r) on the nr grid, and r phi_ab(r) for every pair a >= b in setfl order, the cross pair
    mixed as phi_ab = (f_b / f_a phi_a + f_a / f_b phi_b) / 2 (Johnson's alloy rule)."""
    fs = [johnson_functions(par) for par in elements]
    rho_max = 3.0 * max(par["rho_e"] for par in elements)
    dr, drho = cut / (n - 1), rho_max / (n - 1)
    r = np.arange(n) * dr
    rr = np.where(r > 0, r, dr * 1e-3)
    frho = np.stack([F(np.arange(n) * drho) for (_, _, F, *_) in fs])
    rhor = np.stack([f(rr) for (f, *_) in fs])
    z2r = []
    for a in range(len(fs)):
        for b in range(a + 1):
            fa, pa = fs[a][0](rr), fs[a][1](rr)
            fb, pb = fs[b][0](rr), fs[b][1](rr)
            phi = pa if a == b else 0.5 * (fb / fa * pa + fa / fb * pb)
            z2r.append(rr * phi)
    return dict(n_elements=len(fs), names=list(names), mass=np.array(masses, np.float64), nrho=n, drho=drho,
                nr=n, dr=dr, cut=cut, frho=frho, rhor=rhor, z2r=np.stack(z2r))


def write_setfl(body, path):
    """Writes a setfl body (johnson_setfl() or read_setfl() dict) as a LAMMPS eam/alloy file."""
    with open(path, "w") as f:
        f.write("setfl written by rbmd_b200.synth\n\n\n")
        f.write(f"{body['n_elements']} " + " ".join(body["names"]) + "\n")
        f.write(f"{int(body['nrho'])} {float(body['drho'])!r} {int(body['nr'])} {float(body['dr'])!r} "
                f"{float(body['cut'])!r}\n")

        def block(v):
            v = np.asarray(v, np.float64)
            for k in range(0, len(v), 5):
                f.write(" ".join(repr(float(x)) for x in v[k:k + 5]) + "\n")

        for e in range(body["n_elements"]):
            f.write(f"{29 + e} {float(body['mass'][e])!r} 3.6 fcc\n")
            block(body["frho"][e])
            block(body["rhor"][e])
        for q in range(len(body["z2r"])):
            block(body["z2r"][q])
    return path


def eam_alloy(cells=6, a=3.6, frac_b=0.3, T=600.0, seed=1, build_splines=None, **kw):
    """fcc lattice of two Johnson elements (johnson_setfl), a random fraction frac_b of type 1;
    `build_splines(setfl_body, type_element) -> eam dict` makes the per-type tables
    (rbmd_eam_build_setfl_splines)."""
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.arange(cells)
    cell = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 1, 3)
    pos = ((cell + base[None]) * a).reshape(-1, 3) + 0.25 * a
    L = cells * a
    n = pos.shape[0]
    rng = np.random.default_rng(seed)
    types = (rng.uniform(size=n) < frac_b).astype(np.int32)
    mass = np.where(types == 1, M_B, M_CU)
    kB, mvv2e = 8.617343e-5, 1.0364269e-4
    vel = maxwell(mass, T, kB, mvv2e, rng)
    params = A.default_params(force_field=A.FF_EAM, neighbor=A.NEIGH_RBL, cut_off=5.0, r_core=2.5,
                              neighbor_sample_num=100, units=A.UNITS_METAL, timestep=0.002,
                              temp_ctrl=A.TC_NOSE_HOOVER, temperature=(T, T, 0.1), num_steps=1000,
                              seed=seed, precision=A.PREC_FP64)
    for k, v in kw.items():
        _set(params, k, v)
    sd = SystemData(pos, mass, types, [0.0, 0.0], [0.0, 0.0], [0, 0, 0], [L, L, L], vel=vel,
                    params=params, name=f"eam_alloy_{n}")
    if build_splines is not None:
        sd.eam = build_splines(johnson_setfl(), [0, 1])
    return sd


def _set(params, k, v):
    cur = getattr(params, k)
    if hasattr(cur, "__len__"):
        cur[:] = v
    else:
        setattr(params, k, v)


def serving_stream(n_requests=512, n_min=1000, n_max=64000, rate=50.0, seed=7):
    """Request sizes log-uniform in [n_min, n_max] and Poisson arrival times at `rate` per s."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(n_min), math.log(n_max), n_requests)).astype(int)
    gaps = rng.exponential(1.0 / rate, n_requests)
    arrivals = np.cumsum(gaps) - gaps[0]
    return sizes, arrivals


def write_funcfl(body, path, z=29, mass=63.55, a0=3.615, lattice="fcc"):
    """Writes a funcfl body (johnson_funcfl() or read_funcfl() dict) as a funcfl file: comment,
    "Z mass a0 lattice", "nrho drho nr dr cut", then F(rho), Z(r) and rho(r), five per line."""
    with open(path, "w") as f:
        f.write("funcfl written by rbmd_b200.synth\n")
        f.write(f"{z} {mass!r} {a0!r} {lattice}\n")
        f.write(f"{int(body['nrho'])} {float(body['drho'])!r} {int(body['nr'])} {float(body['dr'])!r} "
                f"{float(body['cut'])!r}\n")
        for key in ("frho", "zr", "rhor"):
            v = np.asarray(body[key], np.float64)
            for k in range(0, len(v), 5):
                f.write(" ".join(repr(float(x)) for x in v[k:k + 5]) + "\n")
    return path


def write_rbmd_input(sd, directory, atom_style=None, thermo_interval=1, name="rbmd", potential_file=None):
    """Writes `sd` as the reference's inputs: a LAMMPS data file (every double at full precision,
    velocities included) and an rbmd.json in the reference schema that runs it with sd.params
    (plus the optional keys seed, precision and rbl_mode).  Returns the json path.  The data file
    carries per-type masses, so sd's masses must be uniform within each type."""
    import json as _json
    import os as _os
    p = sd.params
    n, nt = sd.n, len(sd.eps)
    if atom_style is None:
        atom_style = "full" if sd.molecule is not None else ("charge" if sd.charge is not None else "atomic")
    tmass = np.zeros(nt)
    for t in range(nt):
        m = sd.mass[sd.types == t]
        if len(m) and not np.all(m == m[0]):
            raise ValueError(f"type {t} has more than one mass")
        tmass[t] = m[0] if len(m) else 1.0
    units = {A.UNITS_LJ: "LJ", A.UNITS_REAL: "REAL", A.UNITS_METAL: "METAL"}[p.units]
    _os.makedirs(directory, exist_ok=True)
    data = _os.path.join(directory, f"{name}.data")
    q = sd.charge if sd.charge is not None else np.zeros(n)
    mol = sd.molecule if sd.molecule is not None else np.arange(n)
    nb = 0 if sd.bond_atoms is None else len(sd.bond_type)
    na = 0 if sd.angle_atoms is None or sd.angle_type is None else len(sd.angle_type)
    nd = 0 if sd.dihedral_atoms is None else len(sd.dihedral_type)
    with open(data, "w") as f:
        f.write(f"LAMMPS data file written by rbmd_b200.synth ({sd.name})\n\n")
        f.write(f"{n} atoms\n{nt} atom types\n")
        if nb:
            f.write(f"{nb} bonds\n{len(sd.bond_k)} bond types\n")
        if na:
            f.write(f"{na} angles\n{len(sd.angle_k)} angle types\n")
        if nd:
            f.write(f"{nd} dihedrals\n{len(sd.dihedral_k)} dihedral types\n")
        f.write("\n")
        for k, ax in enumerate("xyz"):
            f.write(f"{float(sd.box_lo[k])!r} {float(sd.box_hi[k])!r} {ax}lo {ax}hi\n")
        f.write("\nMasses\n\n")
        for t in range(nt):
            f.write(f"{t + 1} {float(tmass[t])!r}\n")
        f.write("\nPair Coeffs # lj/cut\n\n")
        for t in range(nt):
            f.write(f"{t + 1} {float(sd.eps[t])!r} {float(sd.sig[t])!r}\n")
        if nb:
            f.write("\nBond Coeffs # harmonic\n\n")
            for t in range(len(sd.bond_k)):
                f.write(f"{t + 1} {float(sd.bond_k[t])!r} {float(sd.bond_r0[t])!r}\n")
        if na:
            f.write("\nAngle Coeffs # harmonic\n\n")
            for t in range(len(sd.angle_k)):
                f.write(f"{t + 1} {float(sd.angle_k[t])!r} {float(sd.angle_theta0[t])!r}\n")
        if nd:
            f.write("\nDihedral Coeffs # harmonic\n\n")
            for t in range(len(sd.dihedral_k)):
                f.write(f"{t + 1} {float(sd.dihedral_k[t])!r} {int(sd.dihedral_sign[t])} "
                        f"{int(sd.dihedral_multiplicity[t])}\n")
        f.write(f"\nAtoms # {atom_style}\n\n")
        for i in range(n):
            x, y, z = (repr(float(c)) for c in sd.pos[i])
            if atom_style == "full":
                f.write(f"{i + 1} {int(mol[i]) + 1} {int(sd.types[i]) + 1} {float(q[i])!r} {x} {y} {z} 0 0 0\n")
            elif atom_style == "charge":
                f.write(f"{i + 1} {int(sd.types[i]) + 1} {float(q[i])!r} {x} {y} {z} 0 0 0\n")
            else:
                f.write(f"{i + 1} {int(sd.types[i]) + 1} {x} {y} {z} 0 0 0\n")
        if sd.vel is not None:
            f.write("\nVelocities\n\n")
            for i in range(n):
                f.write(f"{i + 1} " + " ".join(repr(float(c)) for c in sd.vel[i]) + "\n")
        if nb:
            f.write("\nBonds\n\n")
            for b in range(nb):
                f.write(f"{b + 1} {int(sd.bond_type[b]) + 1} {int(sd.bond_atoms[2 * b]) + 1} "
                        f"{int(sd.bond_atoms[2 * b + 1]) + 1}\n")
        if na:
            f.write("\nAngles\n\n")
            for a in range(na):
                i3 = sd.angle_atoms[3 * a:3 * a + 3] + 1
                f.write(f"{a + 1} {int(sd.angle_type[a]) + 1} {i3[0]} {i3[1]} {i3[2]}\n")
        if nd:
            f.write("\nDihedrals\n\n")
            for q in range(nd):
                i4 = sd.dihedral_atoms[4 * q:4 * q + 4] + 1
                f.write(f"{q + 1} {int(sd.dihedral_type[q]) + 1} {i4[0]} {i4[1]} {i4[2]} {i4[3]}\n")
    ff = {v: k for k, v in A.FORCE_FIELDS.items()}[p.force_field]
    hp = {"force_field": {"type": ff} if potential_file is None else {"type": ff, "potential_file": potential_file},
          "neighbor": {"type": "RBL" if p.neighbor == A.NEIGH_RBL else "VERLETLIST", "cut_off": p.cut_off,
                       "r_core": p.r_core, "neighbor_sample_num": p.neighbor_sample_num},
          "extend": {}}
    if nd:
        hp["force_field"]["dihedral_type"] = "Harmonic"
    if p.coulomb != A.COUL_NONE:
        hp["coulomb"] = {"type": "RBE" if p.coulomb == A.COUL_RBE else "EWALD",
                         "coulomb_sample_num": p.coulomb_sample_num, "alpha": p.alpha,
                         "kmax": [int(k) for k in p.kmax]}
    if p.fix_shake != A.SHAKE_NULL:
        hp["extend"]["fix_shake"] = bool(p.fix_shake == A.SHAKE_TRUE)
    if sd.special_offsets is not None:
        hp["extend"]["special_bonds"] = [int(w) for w in p.special_bonds]
    tc = {v: k for k, v in A.TEMP_CTRLS.items()}.get(p.temp_ctrl, "NOSE_HOOVER")
    cfg = {"init_configuration": {"read_data": {"file": f"{name}.data", "unit": units, "atom_style": atom_style,
                                                "velocity_type": "GAUSS"}},
           "hyper_parameters": hp,
           "execution": {"ensemble": "NVE" if p.temp_ctrl == A.TC_NONE else "NVT",
                         "temperature": list(p.temperature), "temp_ctrl_type": tc, "timestep": p.timestep,
                         "num_steps": int(p.num_steps), "seed": int(p.seed),
                         "precision": "MIXED" if p.precision == A.PREC_MIXED else "FP64",
                         "rbl_mode": "PHILOX" if p.rbl_mode == A.RBL_PHILOX else "STRIDE"},
           "outputs": {"thermo_out": {"interval": int(thermo_interval)}}}
    path = _os.path.join(directory, f"{name}.json")
    with open(path, "w") as f:
        _json.dump(cfg, f, indent=2)
    return path
