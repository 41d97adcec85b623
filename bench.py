#!/usr/bin/env python
"""bench.py -- atom-steps/s of batched mixed-precision RBMD serving on B200, against the plain FP64
one-system-per-launch path, with force error, p50/p99 latency, roofline and a CPU baseline.

Workload (synthetic, seeded): the batched serving stream -- 512 independent SPC/E water systems
with 0.15 M NaCl, atom counts log-uniform in [1k, 64k], Poisson arrivals at 50 req/s, each asking
for 1000 RBE + RBL NVT steps at 300 K (RBE alpha 0.09 A^-2 [beta 0.3/A], P = 100; RBL rc 10 A, r_core
5 A, 100 shell samples; SHAKE water; FP32 pair/RBE arithmetic with FP64 integration, rho(k) and
reductions).

Lines printed by rank 0 (one JSON line):
  value  -- device-resident throughput: all 512 systems resident in HBM, K batched steps timed with
            CUDA events on the library stream (max over ranks), atom-steps/s summed over ranks.
  e2e    -- the same stream through the public serving API (rbmd_serve_submit with host arrays at
            the Poisson arrival times; results read back to host), wall clock, with p50/p99
            request latency.
  plain_fp64 -- the same size distribution (every 4th request) run FP64, one system per launch.
  --impl reference -- the CPU restatement of the reference's algorithm (the reference itself needs
            VTK-m, which this environment lacks) on a bounded sample of the same workload.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-steps/s batched vs plain on 1 B200 at <=1e-3 force err; p50/p99 latency"
UNIT = "atom-steps/s"
WORKLOAD = ("saline serving stream: 512 SPC/E + 0.15 M NaCl systems, N log-uniform 1k-64k, Poisson 50 req/s, "
            "1000 RBE(P=100)+RBL NVT steps each, mixed FP32/FP64")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20, help="timed batched steps of the resident batch")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--requests", type=int, default=512)
    ap.add_argument("--request-steps", type=int, default=1000)
    ap.add_argument("--rate", type=float, default=50.0)
    ap.add_argument("--round-atoms", type=int, default=4_000_000,
                    help="serving rounds step the requests with the least remaining work up to this many atoms "
                         "(0: every active request each round)")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-accuracy", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--out", default=None, help="also write the JSON line here")
    return ap.parse_args()


# ------------------------------------------------------------------------------------------ utils
class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


class Dist:
    """One process per GPU from torchrun's environment.  Systems are independent, so the only
    collectives are the barriers around the timed region and the max / sum of the timing.  The
    backend is NCCL (RBMD_DIST_BACKEND=gloo runs the same logic on host tensors, for CPU tests)."""

    def __init__(self, backend=None, timeout_s=600):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend or os.environ.get("RBMD_DIST_BACKEND", "nccl")
        self.torch = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as td
            if self.backend == "nccl":
                torch.cuda.set_device(self.local)
            td.init_process_group(self.backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.torch = torch
            self.td = td

    def barrier(self):
        if self.world > 1:
            self.td.barrier()

    def reduce(self, x, op="max"):
        if self.world == 1:
            return x
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = self.torch.tensor([float(x)], device=dev, dtype=self.torch.float64)
        self.td.all_reduce(t, op=self.td.ReduceOp.MAX if op == "max" else self.td.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self.td.destroy_process_group()


def build_stream(args, rank):
    from rbmd_b200 import synth
    sizes, arrivals = synth.serving_stream(n_requests=args.requests, rate=args.rate, seed=7 + 1000 * rank)
    systems = [synth.saline(int(n), seed=100000 * rank + k) for k, n in enumerate(sizes)]
    for k, sd in enumerate(systems):
        sd.params.num_steps = args.request_steps
        sd.params.seed = 1 + k + 100000 * rank
    return systems, arrivals


def desc_bytes(sd):
    b = 0
    for name in ("pos", "vel", "charge", "mass", "types", "molecule", "bond_atoms", "bond_type", "angle_atoms",
                 "angle_type", "special_offsets", "special_ids", "special_weights", "eps", "sig"):
        a = getattr(sd, name, None)
        if a is not None:
            b += a.nbytes
    return b


# ------------------------------------------------------------------------------------------ parts
def measure_resident(ctx, systems, args, dist, clocks):
    ids = [ctx.add_system(sd) for sd in systems]
    ctx.init(ids)
    ctx.step(ids, args.warmup)  # captures the batched step graph
    ctx.sync()
    launches0 = ctx.launch_count()
    dist.barrier()
    clocks.start()
    ms = ctx.step_timed(ids, args.steps)
    clk = clocks.stop()
    launches = ctx.launch_count() - launches0
    dist.barrier()
    atoms = sum(sd.n for sd in systems)
    ms_max = dist.reduce(ms, "max")
    atoms_all = dist.reduce(atoms, "sum")
    status = [ctx.thermo(i)["status"] for i in ids[:4]]
    return ids, dict(ms=ms_max, atoms_rank=atoms, atoms_all=atoms_all, launches=launches, clocks=clk,
                     value=atoms_all * args.steps / (ms_max * 1e-3), status=status)


def kernel_profile(ctx, ids, systems):
    """Per-kernel device time (CUDA events on the library stream) of two eager batched steps."""
    ctx.profile(True)
    ctx.step(ids, 2)
    ctx.sync()
    out = {}
    for name in ("nhc", "kick_drift", "cells", "shake", "rbe_sample", "rho", "bonded", "pair_col", "pair_tile", "pair_lean",
                 "pair_atom", "final", "rattle"):
        ms, n, units = ctx.profile_get(name)
        if n:
            out[name] = dict(avg_ms=ms, launches=n, units_per_launch=units)
    ctx.profile(False)
    return out


def pair_stats(ctx, sid, n):
    """Selected pairs per atom (core + sampled shell) of one representative system."""
    nc, ns, _ = ctx.rbl_lists(sid, cap=1024)
    return float((nc + ns).mean()), float(nc.mean()), float(ns.mean())


def measure_plain(systems, args, device):
    """FP64, one system per launch, eager: the plain path the batched mixed path is compared to."""
    import rbmd_b200
    from rbmd_b200 import _abi as A
    sample = systems[::4]
    ctx = rbmd_b200.Context(device=device, batched=False, graphs=False)
    tot_ms, tot_as = 0.0, 0
    steps = 20
    for sd in sample:
        s2 = sd.copy()
        s2.params.precision = A.PREC_FP64
        sid = ctx.add_system(s2)
        ctx.init(sid)
        ctx.step(sid, 2)
        ms = ctx.step_timed(sid, steps)
        tot_ms += ms
        tot_as += s2.n * steps
        ctx.remove_system(sid)
    ctx.close()
    return dict(value=tot_as / (tot_ms * 1e-3), systems=len(sample), steps_each=steps,
                atoms=sum(sd.n for sd in sample))


def measure_accuracy(device):
    """(i) mixed vs FP64 on the same Philox stream; (ii) RBE vs full Ewald (FP64, converged kmax)."""
    import rbmd_b200
    from rbmd_b200 import _abi as A, synth
    sd = synth.saline(4000, seed=11)
    ctx = rbmd_b200.Context(device=device)
    f = {}
    for tag, prec, coul, km in (("mixed", A.PREC_MIXED, A.COUL_RBE, 3), ("fp64", A.PREC_FP64, A.COUL_RBE, 3),
                                ("ewald", A.PREC_FP64, A.COUL_EWALD, 17)):
        s2 = sd.copy()
        s2.params.precision = prec
        s2.params.coulomb = coul
        s2.params.kmax[:] = (km, km, km)
        sid = ctx.add_system(s2)
        ctx.compute_forces(sid)
        f[tag] = ctx.forces(sid)
        ctx.remove_system(sid)
    ctx.close()

    def rr(a, b):
        return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))
    return dict(mixed_vs_fp64=rr(f["mixed"], f["fp64"]), rbe_vs_ewald_fp64=rr(f["fp64"], f["ewald"]),
                mixed_vs_ewald=rr(f["mixed"], f["ewald"]), atoms=sd.n)


def measure_traj_accuracy(device, sizes=(1000, 4000, 16000, 64000), checkpoints=2, every=5):
    """Mixed-vs-FP64 force error along trajectories: saline systems of the stream's sizes run in
    mixed precision; at each checkpoint the FP64 path evaluates the same state at the same step
    (same RBE draws and RBL stride), so the difference is the mixed path's error alone.  Reports
    the relative RMS per system and over all checkpoints of all systems."""
    import rbmd_b200
    from rbmd_b200 import _abi as A, synth
    num = den = 0.0
    per = []
    ctx = rbmd_b200.Context(device=device)
    for k, n in enumerate(sizes):
        sd = synth.saline(n, seed=60 + k)
        sd.params.seed = 700 + k
        sid = ctx.add_system(sd)
        s64 = sd.copy()
        s64.params.precision = A.PREC_FP64
        ref = ctx.add_system(s64)
        ctx.init(sid)
        worst = 0.0
        for _ in range(checkpoints):
            ctx.step(sid, every)
            x, v, img = ctx.state(sid)
            step = ctx.thermo(sid)["step"]
            ctx.compute_forces(sid)
            fm = ctx.forces(sid)
            ctx.set_state(ref, x, v, img)
            ctx.set_step(ref, step)
            ctx.compute_forces(ref)
            f64 = ctx.forces(ref)
            a, b = float(((fm - f64) ** 2).sum()), float((f64 ** 2).sum())
            num += a
            den += b
            worst = max(worst, (a / b) ** 0.5)
        per.append({"atoms": sd.n, "max_rel_rms": worst})
        ctx.remove_system(sid)
        ctx.remove_system(ref)
    ctx.close()
    return {"aggregate_rel_rms": (num / den) ** 0.5, "systems": per, "steps_between": every}


def ewald_kspace_forces(x, q, L, alpha, kmax, qqr2e=1.0, chunk=4096):
    """The reciprocal-space Ewald force alone, F_i = (4 pi / V) qqr2e q_i sum_k exp(-k^2 / 4 alpha)
    / k^2 k Im(exp(i k.r_i) conj(rho_k)), rho_k = sum_j q_j exp(i k.r_j), over m in
    [-kmax, kmax]^3 without 0 (the k-space part of ExecutionMD::ComputeChargeStructureFactorEwald +
    ComputeNewFarElectrostaticsWorklet, RunWorklet.cpp:2492-2540), in numpy: the denominator of the
    k-space-only RBE error."""
    L = np.asarray(L, np.float64)
    g = [np.arange(-k, k + 1) for k in kmax]
    m = np.stack(np.meshgrid(*g, indexing="ij"), -1).reshape(-1, 3)
    m = m[(m != 0).any(1)]
    kv = 2 * np.pi * m / L
    k2 = (kv * kv).sum(1)
    w = np.exp(-k2 / (4 * alpha)) / k2
    V = float(np.prod(L))
    F = np.zeros_like(x)
    for a in range(0, len(kv), chunk):
        kk, ww = kv[a:a + chunk], w[a:a + chunk]
        e = np.exp(1j * (x @ kk.T))                     # [n, k]
        rho = (q[:, None] * e).sum(0)                   # [k]
        im = (e * np.conj(rho)[None, :]).imag * ww[None, :]
        F += im @ kk
    return F * (4 * np.pi / V) * qqr2e * q[:, None]


def converged_kmax(L, alpha, tol=1e-12):
    """Smallest |m| per dimension with exp(-k^2 / 4 alpha) < tol beyond it."""
    kc = math.sqrt(-4.0 * alpha * math.log(tol))
    return [int(math.ceil(kc * l / (2 * math.pi))) for l in L]


def measure_rbe_curve(device, n=1000, Ps=(100, 400, 1600, 6400), seeds=(1, 2, 3)):
    """RBE against full Ewald on one saline system of the stream's parameters (FP64 on both sides,
    converged Ewald kmax, the same RBL picks): total-force relative RMS ||F_rbe - F_ewald|| /
    ||F_ewald|| and k-space-only ||F_rbe - F_ewald|| / ||F_k|| (F_k the reciprocal-space Ewald force
    alone) at P = 100 ... 6400 k samples, averaged over Philox seeds, with the least-squares slope of
    log(error) against log(P) (-0.5 for a variance-limited estimator) and the P at which the
    total-force error would reach 1e-3 on that line."""
    import rbmd_b200
    from rbmd_b200 import _abi as A, synth
    sd = synth.saline(n, seed=11, precision=A.PREC_FP64)
    L = sd.box_hi - sd.box_lo
    km = converged_kmax(L, sd.params.alpha)
    ctx = rbmd_b200.Context(device=device)
    ew = sd.copy()
    ew.params.coulomb = A.COUL_EWALD
    ew.params.kmax[:] = km
    sid = ctx.add_system(ew)
    ctx.compute_forces(sid)
    f_ew = ctx.forces(sid)
    ctx.remove_system(sid)
    f_k = ewald_kspace_forces(sd.pos, sd.charge, L, sd.params.alpha, km, qqr2e=332.06371)
    rows = []
    for P in Ps:
        tot, ks = [], []
        for seed in seeds:
            s2 = sd.copy()
            s2.params.coulomb_sample_num = P
            s2.params.seed = seed
            sid = ctx.add_system(s2)
            ctx.compute_forces(sid)
            d = ctx.forces(sid) - f_ew
            ctx.remove_system(sid)
            tot.append(float(np.sqrt((d * d).sum() / (f_ew * f_ew).sum())))
            ks.append(float(np.sqrt((d * d).sum() / (f_k * f_k).sum())))
        rows.append({"P": P, "total_rel_rms": float(np.mean(tot)), "kspace_rel_rms": float(np.mean(ks)),
                     "seeds": len(seeds)})
    ctx.close()
    lp = np.log([r["P"] for r in rows])
    slope, icpt = np.polyfit(lp, np.log([r["total_rel_rms"] for r in rows]), 1)
    kslope, _ = np.polyfit(lp, np.log([r["kspace_rel_rms"] for r in rows]), 1)
    p_needed = float(math.exp((math.log(1e-3) - icpt) / slope)) if slope < 0 else None
    return {"atoms": sd.n, "ewald_kmax": km, "curve": rows, "slope_total": float(slope), "slope_kspace": float(kslope),
            "P_for_1e-3_total": p_needed}


def measure_saline_energy(device, n=4000, steps=1000, every=50):
    """Energies of the served configuration (saline, RBE P = 100 + RBL, SHAKE, dt 1 fs), per atom in
    kcal/mol: (i) NVT (Nose-Hoover, the served ensemble) in mixed precision against FP64 on the same
    Philox stream: the largest |E_mixed - E_fp64| along the run, absolute and relative to |PE_0| (the
    mixed path's energy error; the two trajectories decorrelate chaotically over the run);
    (ii) NVE drift E_end - E_0 for RBE + RBL in mixed precision and in FP64 (same draws: the mixed
    path's drift must match the FP64 one) and for FP64 full Ewald with Verlet lists, a force that is
    the gradient of the reported energy (the integrator and SHAKE alone).  RBL's sampled shells and
    RBE's sampled k vectors make the served force a random estimate of that gradient, so its NVE
    energy is not conserved: that heating is the method's, equal in both precisions."""
    import rbmd_b200
    from rbmd_b200 import _abi as A, synth
    base = synth.saline(n, seed=21)
    base.params.seed = 5
    L = base.box_hi - base.box_lo

    def run(prec, coul, nve, verlet=False):
        sd = base.copy()
        sd.params.precision = prec
        if nve:
            sd.params.temp_ctrl = A.TC_NONE
            sd.params.ensemble = A.ENS_NVE
        if coul == A.COUL_EWALD:
            sd.params.coulomb = A.COUL_EWALD
            sd.params.kmax[:] = converged_kmax(L, sd.params.alpha)
        if verlet:
            sd.params.neighbor = A.NEIGH_VERLET
        ctx = rbmd_b200.Context(device=device)
        sid = ctx.add_system(sd)
        ctx.init(sid)
        th = ctx.thermo(sid)
        e, pe0 = [th["total_energy"]], th["potential_energy"]
        for _ in range(steps // every):
            ctx.step(sid, every)
            e.append(ctx.thermo(sid)["total_energy"])
        st = ctx.thermo(sid)["status"]
        ctx.close()
        return np.array(e), pe0, st

    ps = steps * float(base.params.timestep) * 1e-3
    out = {"atoms": base.n, "steps": steps, "every": every, "ps": ps, "unit": "kcal/mol per atom"}
    e_m, pe0, s1 = run(A.PREC_MIXED, A.COUL_RBE, False)
    e_d, _, s2 = run(A.PREC_FP64, A.COUL_RBE, False)
    d = float(np.abs(e_m - e_d).max())
    out["nvt_mixed_vs_fp64"] = {"max_abs": d, "rel_to_pe0": d / abs(pe0), "pe0": pe0, "e0": float(e_d[0])}
    drift = {}
    for tag, prec, coul, verlet in (("rbe_rbl_mixed", A.PREC_MIXED, A.COUL_RBE, False),
                                    ("rbe_rbl_fp64", A.PREC_FP64, A.COUL_RBE, False),
                                    ("ewald_verlet_fp64", A.PREC_FP64, A.COUL_EWALD, True)):
        e, _, st = run(prec, coul, True, verlet)
        drift[tag] = {"drift": float(e[-1] - e[0]), "per_ps": float((e[-1] - e[0]) / ps),
                      "max_excursion": float(np.abs(e - e[0]).max()), "status": int(st)}
    out["nve"] = drift
    out["nve_drift_mixed_minus_fp64"] = drift["rbe_rbl_mixed"]["drift"] - drift["rbe_rbl_fp64"]["drift"]
    out["status"] = [int(s1), int(s2)]
    return out


def measure_drift(device, steps=1000, every=100):
    """Energy conservation of the LJ fluid (4000 atoms, RBL rs 1.2 with 100 shell samples, NVE,
    dt 0.005): total energy per atom every `every` steps in FP64 and in mixed precision.  Reports
    the relative drift (E_end - E_0) / |E_0|, the largest excursion and the mixed-vs-FP64 energy
    difference along the run."""
    import rbmd_b200
    from rbmd_b200 import _abi as A, synth
    out = {}
    traj = {}
    for tag, prec in (("fp64", A.PREC_FP64), ("mixed", A.PREC_MIXED)):
        sd = synth.lj_fcc(precision=prec)
        ctx = rbmd_b200.Context(device=device)
        sid = ctx.add_system(sd)
        ctx.init(sid)
        e = [ctx.thermo(sid)["total_energy"]]
        for _ in range(steps // every):
            ctx.step(sid, every)
            e.append(ctx.thermo(sid)["total_energy"])
        ctx.close()
        e = np.array(e)
        traj[tag] = e
        out[tag] = dict(drift=float((e[-1] - e[0]) / abs(e[0])), max_excursion=float(np.abs(e - e[0]).max() / abs(e[0])))
    out["energy_mixed_vs_fp64"] = float(np.abs(traj["mixed"] - traj["fp64"]).max() / abs(traj["fp64"][0]))
    out.update(atoms=4000, steps=steps, ensemble="NVE", e0_per_atom=float(traj["fp64"][0]))
    return out


def measure_e2e(systems, arrivals, args, device):
    """The stream through rbmd_serve_*: submissions at the Poisson times, results back to host."""
    import rbmd_b200
    ctx = rbmd_b200.Context(device=device)
    ctx.serve_start(steps_per_round=50, round_atoms=args.round_atoms)
    rids = []
    h2d = 0
    t0 = time.monotonic()
    for sd, ta in zip(systems, arrivals):
        now = time.monotonic() - t0
        if ta > now:
            time.sleep(ta - now)
        rids.append(ctx.serve_submit(sd, args.request_steps))
        h2d += desc_bytes(sd)
    lat, d2h, atom_steps, sizes = [], 0, 0, []
    for rid, sd in zip(rids, systems):
        rc = ctx.serve_wait(rid, 3600.0)
        x, v, th, st = ctx.serve_result(rid)
        if rc or st["status"]:
            raise RuntimeError(f"request {rid} failed with {rc}/{st['status']}")
        lat.append(st["t_done"] - st["t_submit"])
        sizes.append(sd.n)
        d2h += x.nbytes + v.nbytes
        atom_steps += st["atom_steps"]
    wall = time.monotonic() - t0
    ctx.serve_stop()
    ctx.close()
    total_steps = len(systems) * args.request_steps
    lat, sizes = np.array(lat), np.array(sizes)
    bands = {}
    for lo, hi in STRATA:
        m = (sizes >= lo) & (sizes < hi)
        if m.any():
            bands[f"{lo}-{hi - 1}"] = {"requests": int(m.sum()), "p50_s": float(np.percentile(lat[m], 50)),
                                      "p99_s": float(np.percentile(lat[m], 99))}
    return dict(value=atom_steps / wall, wall_s=wall, p50_s=float(np.percentile(lat, 50)),
                p99_s=float(np.percentile(lat, 99)), h2d=h2d / total_steps, d2h=d2h / total_steps,
                atom_steps=atom_steps, bands=bands)


STRATA = ((1000, 4000), (4000, 16000), (16000, 64001))  # log-thirds of the stream's size range


def stream_strata(n_requests, seed=7):
    """The serving stream's sizes in three log-size strata: per stratum the request nearest its
    median size (the system the CPU runs) and the stratum's share of the stream's atoms (its
    weight in the throughput)."""
    from rbmd_b200 import synth
    sizes, _ = synth.serving_stream(n_requests=n_requests, seed=seed)
    out = []
    for lo, hi in STRATA:
        s = np.sort(sizes[(sizes >= lo) & (sizes < hi)])
        if s.size == 0:
            continue
        out.append(dict(lo=lo, hi=hi, requests=int(s.size), atoms=int(s.sum()), size=int(s[s.size // 2])))
    return out


def cpu_stream_rate(n_requests, steps=None, warmup=1, seconds=None, threads=None):
    """The FP64 CPU restatement of the reference algorithm on a size-stratified sample of the
    serving stream: one system per stratum (the stratum's median size, the stream's own
    parameters), `warmup` untimed then `steps` timed steps of each (or steps until `seconds` of
    wall time), on `threads` host threads.  The stream's throughput follows from the per-stratum
    rates r_k weighted by the strata's atoms w_k: sum(w) / sum(w / r), the rate at which the CPU
    would work through the stream's atom-steps."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_ffi
    from rbmd_b200 import _abi as A, synth
    # the oracle's loops run on RBMD_ORACLE_THREADS std::threads, fixed at its first parallel loop
    threads = threads or (os.cpu_count() or 1)
    os.environ["RBMD_ORACLE_THREADS"] = str(threads)
    strata = stream_strata(n_requests)
    systems = []
    for k, st in enumerate(strata):
        sd = synth.saline(st["size"], seed=3 + k)
        sd.params.precision = A.PREC_FP64
        o = oracle_ffi.Oracle(sd)
        o.init()
        o.step(warmup)
        systems.append((sd, o))
    per_step = [0.0] * len(systems)
    done = 0
    t_all = time.perf_counter()
    while True:
        for k, (sd, o) in enumerate(systems):
            t0 = time.perf_counter()
            o.step(1)
            per_step[k] += time.perf_counter() - t0
        done += 1
        if steps is not None and done >= steps:
            break
        if steps is None and time.perf_counter() - t_all >= (seconds or 10.0) and done >= 2:
            break
    rates = [sd.n * done / t for (sd, _), t in zip(systems, per_step)]
    w = [st["atoms"] for st in strata]
    value = sum(w) / sum(wk / rk for wk, rk in zip(w, rates))
    desc = ", ".join(f"{sd.n} atoms for [{st['lo']}, {st['hi']}) ({st['requests']} requests, "
                     f"{r:.3g} atom-steps/s)" for (sd, _), st, r in zip(systems, strata, rates))
    return dict(value=value, unit=UNIT, cores=threads, kind="port",
                sample=f"size-stratified sample of the stream: {done} FP64 NVT steps each of {desc}; "
                       "throughput weighted by each stratum's atoms",
                strata=[dict(st, rate=r) for st, r in zip(strata, rates)], steps=done)


PAIR_KERNELS = {"pair_col": "k_pair_col (warp per column of home cells, lane per atom over a staged row: RBL picks, LJ + erfc), "
                            "timed with the stray pass k_pair_col_strays before it",
                "pair_tile": "k_pair_tile (warp per home cell: shared candidate batches, RBL picks, LJ + erfc)",
                "pair_lean": "k_pair2 (warp per atom with segment tables)", "pair_atom": "k_pair (general warp per atom)"}


def profiled_figures(name):
    """Machine-readable figures ("key: value" lines) of a pair kernel's committed ncu summary
    profiles/k_<name>_saline_small.md: traffic_bytes_per_atom, issue_active_pct,
    warp_inst_per_atom; {} without one."""
    path = os.path.join(ROOT, "profiles", f"k_{name}_saline_small.md")
    out = {}
    if not os.path.exists(path):
        return out
    for line in open(path):
        key, sep, val = line.strip().partition(":")
        if sep and key in ("traffic_bytes_per_atom", "issue_active_pct", "warp_inst_per_atom"):
            try:
                out[key] = float(val)
            except ValueError:
                pass
    out["source"] = f"profiles/k_{name}_saline_small.md"
    return out


def roofline(prof, pairs_per_atom, peaks, fp32_peak):
    """Roofline of the dominant pair kernel (largest device time over the profiled steps).  Its
    bound is the FP32 pipe (the pair arithmetic and the selection around it are FP32 / integer
    issue; SFU ops -- rsqrt, ex2, rcp -- are counted as one flop each, not separately weighted):
    achieved = 40 flops per selected pair (26 LJ + 14 real-space Coulomb) x pairs per atom x
    atoms per launch / the launch's CUDA-event time.  The HBM view (64 algorithmic bytes per atom)
    is the secondary entry."""
    recs = {k: v for k, v in prof.items() if k in PAIR_KERNELS}
    if not recs:
        return None, None
    name = max(recs, key=lambda k: recs[k]["avg_ms"] * recs[k]["launches"])
    p = recs[name]
    atoms = p["units_per_launch"]
    secs = p["avg_ms"] * 1e-3
    # algorithmic HBM bytes per atom: its sorted FP32 position + charge (16 B), sorted metadata
    # (16 B) and the FP64 force written (32 B); neighbour reuse is cache traffic, not counted
    bytes_alg = 64.0 * atoms
    flops = (26 + 14) * pairs_per_atom * atoms  # LJ + Coulomb pair convention (flops per pair)
    hbm = peaks.get("hbm_gbs", 6650.0)
    achieved_gbs = bytes_alg / secs / 1e9
    fig = profiled_figures(name)
    tpa = fig.get("traffic_bytes_per_atom")
    traffic = None if tpa is None else tpa * atoms
    traffic_src = None if tpa is None else \
        f"{fig['source']} (ncu dram__bytes_read.sum + dram__bytes_write.sum on 64 stream systems), scaled by atoms"
    tf = flops / secs / 1e12
    r_fp32 = {"bound": "fp32", "achieved": tf, "peak": fp32_peak, "unit": "TFLOP/s",
              "frac": tf / fp32_peak if fp32_peak else None, "traffic": traffic, "traffic_source": traffic_src,
              "kernel": PAIR_KERNELS[name], "launch_ms": p["avg_ms"], "atoms_per_launch": atoms,
              "peak_source": "FFMA-chain microbenchmark in this run (rbmd_fma_peak), of measured",
              "flops_per_pair": 40, "pairs_per_atom": pairs_per_atom,
              "issue_active_pct": fig.get("issue_active_pct"), "warp_inst_per_atom": fig.get("warp_inst_per_atom"),
              "issue_source": fig.get("source")}
    r_hbm = {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm, "unit": "GB/s", "frac": achieved_gbs / hbm,
             "traffic": traffic, "traffic_source": traffic_src, "bytes_alg_per_atom": 64.0,
             "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks else "fallback 6650 GB/s"}
    return r_fp32, r_hbm


def run_reference(args, dist):
    """--impl reference: the CPU restatement of the reference algorithm on all host cores, on a
    size-stratified sample of the same stream (each step one FP64 step of each stratum's system)."""
    if dist.rank != 0:
        return
    cores = os.cpu_count() or 1
    r = cpu_stream_rate(args.requests, steps=args.steps, warmup=args.warmup, threads=cores)
    line = {"metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "impl": "reference", "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD + "; CPU: size-stratified sample (one system per log-size third, "
                       "weighted by the stream's atoms in it)", "parallelism": "cpu"},
            "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["cores"], "kind": "port",
                             "sample": r["sample"]},
            "strata": r["strata"],
            "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference binary needs VTK-m 1.9 (absent); this is the FP64 C++ restatement of its algorithm"}
    print(json.dumps(line), flush=True)


def launch_ranks(args):
    """`--gpus N` without a torchrun environment: start N ranks (one process per GPU, rendezvous on
    127.0.0.1) through torch.distributed.run and return its exit code; None when this process is
    already a rank (or N is 1).  A rank whose WORLD_SIZE differs from --gpus is an error."""
    world = os.environ.get("WORLD_SIZE")
    if world is not None:
        if int(world) != args.gpus:
            raise SystemExit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}")
        return None
    if args.gpus <= 1:
        return None
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = parse()
    rc = launch_ranks(args)
    if rc is not None:
        sys.exit(rc)
    dist = Dist()
    if args.impl == "reference":
        run_reference(args, dist)
        dist.close()
        return
    import rbmd_b200
    device = dist.local
    peaks = {}
    pk = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk):
        peaks = json.load(open(pk))
    systems, arrivals = build_stream(args, dist.rank)
    ctx = rbmd_b200.Context(device=device)
    fp32_peak = ctx.fma_peak(False)
    fp64_peak = ctx.fma_peak(True)
    clocks = Clocks(device)
    ids, res = measure_resident(ctx, systems, args, dist, clocks)
    prof = kernel_profile(ctx, ids, systems)
    rep = int(np.argsort([sd.n for sd in systems])[len(systems) // 2])
    ppa, pcore, pshell = pair_stats(ctx, ids[rep], systems[rep].n)
    for sid in ids:
        ctx.remove_system(sid)
    ctx.close()
    r_fp32, r_hbm = roofline(prof, ppa, peaks, fp32_peak)
    extra = {}
    if dist.rank == 0:
        if not args.skip_accuracy:
            extra["accuracy"] = measure_accuracy(device)
            extra["accuracy"]["trajectory_mixed_vs_fp64"] = measure_traj_accuracy(device)
            extra["drift"] = measure_drift(device)
            extra["rbe_curve"] = measure_rbe_curve(device)
            extra["saline_energy"] = measure_saline_energy(device)
        if not args.skip_plain:
            extra["plain_fp64"] = measure_plain(systems, args, device)
    e2e = None
    if not args.skip_e2e:
        e2e = measure_e2e(systems, arrivals, args, device)
        e2e_val = dist.reduce(e2e["value"], "sum")
    dist.barrier()
    if dist.rank == 0:
        cpu = None if args.skip_cpu else cpu_stream_rate(args.requests, seconds=args.cpu_seconds)
        plain = extra.get("plain_fp64")
        line = {
            "metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": dist.world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["ms"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair/RBE + f64 integration/reductions",
            "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_systems_per_gpu": len(systems), "atoms_per_gpu": res["atoms_rank"],
                       "atoms_total": res["atoms_all"], "batched_step_per_launch": True, "parallelism": f"dp{dist.world} (independent systems)",
                       "l2": "inputs larger than L2 (all systems resident, >1 GB)"},
            "roofline": r_fp32, "roofline_hbm": r_hbm,
            "pipe_peaks_tflops": {"fp32": fp32_peak, "fp64": fp64_peak},
            "cpu_baseline": cpu,
            "clocks": res["clocks"],
            "gpu_launches": res["launches"],
            "kernel_ms": prof,
            "pairs_per_atom": {"total": ppa, "core": pcore, "shell_sampled": pshell},
            "device_status": res["status"],
        }
        if plain:
            line["plain_fp64"] = plain
            line["speedup_vs_plain_fp64"] = res["value"] / dist.world / plain["value"]
        if "accuracy" in extra:
            line["force_rel_rms"] = extra["accuracy"]
            line["energy_drift"] = extra["drift"]
            line["rbe_vs_ewald_curve"] = extra["rbe_curve"]
            line["served_config_energy"] = extra["saline_energy"]
        if e2e is not None:
            line["e2e"] = {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": e2e["h2d"],
                           "d2h_bytes_per_step": e2e["d2h"], "wall_s": e2e["wall_s"], "p50_latency_s": e2e["p50_s"],
                           "p99_latency_s": e2e["p99_s"], "latency_by_size": e2e["bands"],
                           "round_policy": ("every active request each round" if args.round_atoms <= 0 else
                                            f"least remaining work first, {args.round_atoms} atoms per round"),
                           "request_steps": args.request_steps,
                           "step": "one MD step of one request; bytes averaged over all request-steps"}
        s = json.dumps(line)
        print(s, flush=True)
        if args.out:
            with open(args.out, "w") as fh:
                fh.write(s + "\n")
    dist.close()


if __name__ == "__main__":
    main()
