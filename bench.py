#!/usr/bin/env python
"""Benchmark of the B200 grid ray-casting surface builder.

Default workload: the conformer ensemble (512 structures of 500-8000 atoms, 32 globules x 16
perturbations, each on its own grid), ray cast and triangulated as one batch in mixed precision.
One step = ray casting of the status ray set and the three accurate-triangulation ray sets
(hits, status runs, insideness bits, volume), vertex assembly and marching cubes of all 512
structures, in gradient mode: the derivatives of every structure's volume and area with respect
to its atoms (x, y, z, r) are part of the step.  ``value`` is structures/s with the patch sets
resident in HBM; ``e2e`` is the same step through the C-ABI with host buffers (batch layout,
patch and atom upload from pinned memory; the per-structure volumes, areas and atom derivatives
back).  The same batch in double precision and the plain
per-structure double-precision path are timed beside it (``comparison``).  The hit store and the
bit grids are larger than L2, so no extra flush is needed.

``--workload ses_100k`` runs one large structure instead: 100,000 atoms, probe 1.4 A, grid scale
4.0, perfil 70 (1049^3 nodes); its step adds cavity detection and filling and its e2e downloads
the status map and the mesh.  Multiple GPUs run independent replicas (the path has no cross-GPU
exchange).

``--impl reference`` times the CPU restatement of the reference path on a bounded slab sample of
the same workload with all host threads, and prints the same JSON line with ``impl: reference``.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "structures/s and rays/s, mixed-prec vs FP64 GPU kernel at ≤1e-5 Å hit error"

WORKLOADS = {
    # conformer ensemble: 32 globules of 500..8000 atoms, 16 perturbations (0.3 A) each, every
    # structure on its own grid, one batch
    "ensemble_512": dict(n_base=32, n_perturb=16, n_min=500, n_max=8000, sigma=0.3, seed=5, probe=1.4, scale=2.0,
                         perfil=80.0),
    # the same generator with 4 globules (profiling-size case)
    "ensemble_64": dict(n_base=4, n_perturb=16, n_min=500, n_max=8000, sigma=0.3, seed=5, probe=1.4, scale=2.0,
                        perfil=80.0),
    # single structures: atoms, generator seed, probe, scale, perfil, cavity fill threshold
    "ses_100k": dict(n=100000, seed=3, probe=1.4, scale=4.0, perfil=70.0, cav_vol=10.0),
    "ses_10k": dict(n=10000, seed=2, probe=1.4, scale=3.0, perfil=80.0, cav_vol=10.0),
    "ses_327": dict(n=327, seed=1, probe=1.4, scale=2.0, perfil=70.0, cav_vol=10.0),
}

STAGES = ("bin", "trace", "overflow", "cavity", "vertex", "mc", "cand", "isect", "fill")

# Floating-point operations per candidate of the mixed-precision intersection kernels (adds, muls
# and 2 per fused multiply-add, predicated-on thread instructions), measured with ncu
# (smsp__sass_thread_inst_executed_op_{dadd,dmul,dfma,fadd,fmul,ffma}_pred_on.sum) on the
# 64-structure conformer ensemble and divided by its candidate counts.
FLOPS_PER_CANDIDATE = {"torus": {"fp64": 312.0, "fp32": 35.0}, "sphere": {"fp64": 26.0, "fp32": 74.0}}
# Algorithmic operations per candidate: the oracle's operation model (oracle/oracle.py OP_MODEL:
# adds and multiplies of doubles, FMA = 2; square roots, divisions and the resolvent's cube roots,
# arccos and cos apart) summed over the branches the double-precision path takes, per candidate of
# each kind, on 16 structures of the 64-structure ensemble (10.0 M torus and 9.8 M sphere
# candidates; the model is frozen here, the ncu instruction counts above are reported next to it).
OPS_PER_CANDIDATE = {"torus": {"flops": 180.0, "sqrt": 5.10, "div": 4.81, "cbrt": 1.37, "acos": 0.20, "cos": 0.20},
                     "sphere": {"flops": 73.8, "sqrt": 1.0, "div": 2.0}}
# DRAM bytes (read + written) of the mixed intersection launches per candidate, from an ncu capture
# of the 64-structure ensemble (the ray set of panel 1: 283 MB for the sphere launch, 224 MB for the
# torus launch, 5 MB for the deferred ones, over its 19.9 M candidates)
ISECT_DRAM_BYTES_PER_CANDIDATE = 25.7


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.flush()
        rows = []
        for line in Path(self.out.name).read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    from nanoshaper_b200 import dist as D
    return D.env()


def make_workload(name: str):
    from nanoshaper_b200 import generator
    import nanoshaper_b200 as nb
    w = WORKLOADS[name]
    t0 = time.perf_counter()
    atoms = generator.rsa_globule(w["n"], w["seed"])
    t_gen = time.perf_counter() - t0
    nb.reset_seed()
    ds = nb.DelPhiShared(atoms, w["scale"], w["perfil"])
    cf = nb.ConfigFile()
    cf.add("Surface", "ses")
    cf.add("Probe_Radius", w["probe"])
    cf.add("Accurate_Triangulation", True)
    cf.add("Triangulation", True)
    surf = nb.surfaceFactory().create(cf, ds)
    t0 = time.perf_counter()
    surf.build()
    t_build = time.perf_counter() - t0
    return w, atoms, ds, surf, t_gen, t_build


def run_reference(args, w, ds, surf) -> dict:
    """CPU restatement of the reference path on a bounded slab sample, all host threads."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    O.build()
    threads = os.cpu_count() or 1
    g = ds.grid
    rays_total = g.nz * g.ny + (g.nz * g.ny + g.ny * g.nx + g.nz * g.nx)
    # size the slab for roughly ten seconds of work per step from a small probe run
    t_probe, r_probe = O.time_slab(g, surf.patches, threads, 0.48, 0.50)
    per_ray = t_probe / max(r_probe, 1)
    frac = min(1.0, max(0.01, 10.0 / max(per_ray * rays_total, 1e-9)))
    lo = 0.5 - frac / 2
    hi = 0.5 + frac / 2
    times = []
    rays = 0
    for _ in range(args.warmup):
        O.time_slab(g, surf.patches, threads, lo, hi)
    for _ in range(args.steps):
        dt, rays = O.time_slab(g, surf.patches, threads, lo, hi)
        times.append(dt)
    t = max(statistics.median(times), 1e-9)
    rays_per_s = rays / t
    structs = rays_per_s / rays_total
    sample = (f"ray casting (status + 3 triangulation ray sets) of the central slab "
              f"[{lo:.3f}, {hi:.3f}) of every ray set, {rays} of {rays_total} rays; cavity detection and "
              f"marching cubes not included; structures/s extrapolated from rays/s")
    return {"value": structs, "rays_per_s": rays_per_s, "cores": threads, "kind": "port", "sample": sample,
            "unit": "structures/s"}


def make_ensemble(w: dict):
    """Seeded conformer ensemble and its SES patch sets (host)."""
    from nanoshaper_b200 import generator
    import nanoshaper_b200 as nb
    t0 = time.perf_counter()
    atoms = generator.ensemble(w["n_base"], w["n_perturb"], w["n_min"], w["n_max"], w["sigma"], w["seed"])
    t_gen = time.perf_counter() - t0
    nb.reset_seed()
    surfs = []
    t0 = time.perf_counter()
    for a in atoms:
        ds = nb.DelPhiShared(a, w["scale"], w["perfil"])
        cf = nb.ConfigFile()
        cf.add("Surface", "ses")
        cf.add("Probe_Radius", w["probe"])
        cf.add("Accurate_Triangulation", True)
        cf.add("Triangulation", True)
        sf = nb.surfaceFactory().create(cf, ds)
        sf.build()
        surfs.append(sf)
    t_build = time.perf_counter() - t0
    return atoms, surfs, t_gen, t_build


def rays_of(g) -> int:
    """Rays of one structure: the status ray set and the three accurate-triangulation ray sets."""
    return g.nz * g.ny + (g.nz * g.ny + g.ny * g.nx + g.nz * g.nx)


def ensemble_cpu_baseline(surfs, threads: int, target_s: float = 10.0, steps: int = 1) -> dict:
    """Oracle ray casting (all four ray sets, whole structures, all host threads) of a sample of the
    ensemble: structures in a seeded random order until about target_s seconds; structures/s =
    sample rays/s / the ensemble's mean rays per structure."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    O.build()
    order = list(range(len(surfs)))
    np.random.default_rng(0).shuffle(order)
    rates, sample_idx, sample_rays = [], [], 0
    for _ in range(max(steps, 1)):
        t_tot, r_tot, idx = 0.0, 0, []
        for b in order:
            sf = surfs[b]
            dt, r = O.time_slab(sf.delphi.grid, sf.patches, threads, 0.0, 1.0)
            t_tot += dt
            r_tot += r
            idx.append(b)
            if t_tot >= target_s:
                break
        rates.append(r_tot / max(t_tot, 1e-9))
        sample_idx, sample_rays = idx, r_tot
    rays_per_s = statistics.median(rates)
    mean_rays = statistics.mean(rays_of(sf.delphi.grid) for sf in surfs)
    sizes = [len(surfs[b].delphi.atoms) for b in sample_idx]
    sample = (f"ray casting (status + 3 triangulation ray sets) of {len(sample_idx)} whole structures drawn at random "
              f"({min(sizes)}-{max(sizes)} atoms, {sample_rays} rays, about {target_s:.0f} s); "
              f"structures/s = rays/s / mean rays per structure of the ensemble ({mean_rays:.0f}); marching cubes "
              f"and gradients not included")
    return {"value": rays_per_s / mean_rays, "rays_per_s": rays_per_s, "cores": threads, "kind": "port",
            "sample": sample, "unit": "structures/s"}


def mixed_vs_fp64_accuracy(L, N, ctx, surfs, flags: int) -> dict:
    """Accuracy terms of the metric on a batch: the ray cast in double precision and in mixed
    precision (untimed, hits kept), compared ray by ray.

    * max_hit_error_A: largest |hit_mixed - hit_fp64| in Angstrom over every hit of every ray set
      of every structure (rays with equal hit counts; count_mismatch_rays counts the others);
    * status_mismatch_nodes: status-map nodes whose inside / outside decision differs, from the
      status rays' interval ends (the node range [a, b] of each interval, as the fill computes it),
      and how many of them lie within 1e-6 A of a double-precision interval end (near-node);
    * insideness_mismatch_bits: differing bits of the insideness grids;
    * near_node_hits: double-precision interval ends within 1e-6 A of a decision coordinate (a node
      for status rays, a rintp half-integer for triangulation rays)."""
    def run(prec):
        v = ctypes.c_double()
        N.check(L.nsg_raycast(ctx, flags | N.KEEP_HITS, prec, ctypes.byref(v)), "raycast")
        sets = []
        for s in range(4):
            tot = sum(rays_in_set(sf.delphi.grid, s) for sf in surfs)
            counts = np.zeros(tot, np.int32)
            rc = L.nsg_download_hits(ctx, s, N.ptr(counts), None, 0)
            if rc < 0:
                N.check(rc, "download hits")
            vals = np.zeros(int(counts.astype(np.int64).sum()))
            N.check(L.nsg_download_hits(ctx, s, N.ptr(counts), N.ptr(vals), len(vals)), "download hits")
            sets.append((counts, vals))
        words = sum(((sf.delphi.grid.nx + 31) // 32) * sf.delphi.grid.ny * sf.delphi.grid.nz for sf in surfs)
        bits = np.empty(words, np.uint32)
        N.check(L.nsg_download_insideness(ctx, N.ptr(bits)), "download insideness")
        return sets, bits

    r64, b64 = run(0)
    r32, b32 = run(1)
    out = {"max_hit_error_A": 0.0, "count_mismatch_rays": 0, "status_mismatch_nodes": 0,
           "status_mismatch_near_node": 0, "insideness_mismatch_bits": 0, "near_node_hits": 0, "hits_compared": 0}
    out["insideness_mismatch_bits"] = int(np.unpackbits((b64 ^ b32).view(np.uint8)).sum())
    near = 1e-6
    for s in range(4):
        c64, v64 = r64[s]
        c32, v32 = r32[s]
        ray0 = 0
        h64 = np.concatenate([[0], np.cumsum(c64.astype(np.int64))])
        h32 = np.concatenate([[0], np.cumsum(c32.astype(np.int64))])
        for sf in surfs:
            g = sf.delphi.grid
            nr = rays_in_set(g, s)
            a64, a32 = c64[ray0:ray0 + nr], c32[ray0:ray0 + nr]
            t64 = v64[h64[ray0]:h64[ray0 + nr]]
            t32 = v32[h32[ray0]:h32[ray0 + nr]]
            ray0 += nr
            eq = a64 == a32
            out["count_mismatch_rays"] += int((~eq).sum())
            vc = (0, 0, 2, 1)[s]
            ncoord = (g.nx, g.ny, g.nz)[vc]
            vmin = (g.xmin, g.ymin, g.zmin)[vc]
            delta = 0.0 if s == 0 else 1e-10 - g.hside
            pa = (vmin + 0.0 * g.side) + delta
            dirl = ((vmin + (ncoord - 1) * g.side) + delta) - pa
            m64 = np.repeat(eq, a64)
            m32 = np.repeat(eq, a32)
            if m64.any():
                d = np.abs(t64[m64] - t32[m32]) * abs(dirl)
                out["max_hit_error_A"] = max(out["max_hit_error_A"], float(d.max()))
                out["hits_compared"] += int(m64.sum())
            lim = pa + dirl * t64
            u = (lim - vmin) * g.scale
            if s == 0:
                dist = np.abs(u - np.rint(u)) * g.side
            else:
                dist = np.abs(u - np.floor(u) - 0.5) * g.side
            out["near_node_hits"] += int((dist < near).sum())
            if s == 0:
                # status decisions: node range [a, b] of every kept pair of rays with equal counts
                even = eq & (a64 > 0) & (a64 % 2 == 0)
                sel64 = np.repeat(even, a64)
                sel32 = np.repeat(even, a32)
                p64 = t64[sel64].reshape(-1, 2)
                p32 = t32[sel32].reshape(-1, 2)
                if len(p64):
                    def ranges(p):
                        keep = np.abs(p[:, 1] - p[:, 0]) >= 1e-8
                        l1 = pa + dirl * p[:, 0]
                        l2 = pa + dirl * p[:, 1]
                        a = np.clip(np.floor((l1 - vmin) * g.scale + 0.5), 0, g.nx - 1)
                        b = np.clip(np.floor((l2 - vmin) * g.scale + 0.5), 0, g.nx - 1)
                        a = a + ((vmin + a * g.side) < l1)
                        b = b - ((vmin + b * g.side) > l2)
                        return keep, a, b, l1, l2
                    k64, a_64, b_64, l1_64, l2_64 = ranges(p64)
                    k32, a_32, b_32, _, _ = ranges(p32)
                    e64 = np.where(k64 & (a_64 <= b_64), b_64 - a_64 + 1, 0)
                    e32 = np.where(k32 & (a_32 <= b_32), b_32 - a_32 + 1, 0)
                    diff = (k64 != k32) | (a_64 != a_32) | (b_64 != b_32)
                    nodes = np.where(k64 == k32, np.abs(a_64 - a_32) + np.abs(b_64 - b_32), np.abs(e64 - e32))
                    nodes = np.where(diff, np.maximum(nodes, 1), 0)
                    out["status_mismatch_nodes"] += int(nodes.sum())
                    if diff.any():
                        ul1 = (l1_64 - vmin) * g.scale
                        ul2 = (l2_64 - vmin) * g.scale
                        nr1 = np.abs(ul1 - np.rint(ul1)) * g.side < near
                        nr2 = np.abs(ul2 - np.rint(ul2)) * g.side < near
                        out["status_mismatch_near_node"] += int(nodes[diff & (nr1 | nr2)].sum())
    out["status_mismatch_not_near_node"] = out["status_mismatch_nodes"] - out["status_mismatch_near_node"]
    return out


def rays_in_set(g, s: int) -> int:
    return (g.ny * g.nz, g.ny * g.nz, g.nx * g.ny, g.nx * g.nz)[s]


def run_ensemble(args, world: int, rank: int, local: int) -> None:
    """Batched conformer ensemble: one step = ray casting (4 ray sets) + marching cubes of every
    structure of the ensemble in one batch; value = structures/s over all ranks (replicas)."""
    w = WORKLOADS[args.workload]
    if args.impl == "reference":
        if rank != 0:
            return
        atoms, surfs, t_gen, t_build = make_ensemble(w)
        threads = os.cpu_count() or 1
        cb = ensemble_cpu_baseline(surfs, threads, steps=max(args.steps, 1))
        line = {
            "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "structures/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "rays_per_s": cb["rays_per_s"],
            "config": {"workload": args.workload, "structures": len(surfs),
                       "atoms_total": int(sum(len(a) for a in atoms)), "probe": w["probe"], "scale": w["scale"],
                       "perfil": w["perfil"]},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "structures/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return

    import torch
    from nanoshaper_b200 import dist as D
    torch.cuda.set_device(local)
    pg = D.init("nccl")

    import nanoshaper_b200 as nb
    from nanoshaper_b200 import _native as N
    from nanoshaper_b200 import build as nbuild
    nbuild.build()
    L = N.lib()

    def barrier():
        D.barrier(pg)
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        return D.max_over_ranks(pg, x)

    atoms, surfs, t_gen, t_build = make_ensemble(w)
    nstruct = len(surfs)
    prec = 0 if args.precision == "fp64" else 1
    batch = nb.SurfaceBatch(surfs, device=local, precision=args.precision)
    # launch shapes of the tracer for this batch and precision (untimed; uploads the batch)
    if args.tuning:
        tuning, tune_ms = [int(x) for x in args.tuning.split(",")], None
        batch.upload()
        batch.set_tuning(tuning)
    else:
        tuning, tune_ms = batch.autotune(grad=True, reps=1)
    ctx = batch._context().handle
    atom_off, atoms_cat, patch_atoms = batch.packed_atoms()
    N.check(L.nsg_upload_atoms(ctx, N.ptr(atom_off), N.ptr(atoms_cat), N.ptr(patch_atoms)), "upload atoms")
    flags = N.STATUS | N.ACCURATE_TRIANGULATION | N.GRAD

    def step(precision: int, gv_host=None, ga_host=None):
        """Volume, area and their atom derivatives of every structure (results stay on the device
        unless host buffers are given)."""
        v = ctypes.c_double()
        N.check(L.nsg_raycast(ctx, flags, precision, ctypes.byref(v)), "raycast")
        a = ctypes.c_double()
        nv = ctypes.c_int64()
        nt = ctypes.c_int64()
        N.check(L.nsg_triangulate(ctx, ctypes.byref(a), ctypes.byref(nv), ctypes.byref(nt)), "triangulate")
        rc = L.nsg_atom_grads(ctx, gv_host, ga_host)
        if rc not in (N.NSG_OK, -8):
            N.check(rc, "atom gradients")
        return nv.value, nt.value

    def timed(precision: int, steps: int) -> float:
        # an NVTX range per timed region ("timed_fp64" / "timed_mixed") lets a profiler capture
        # exactly the timed launches (ncu --nvtx --nvtx-include "timed_mixed/")
        torch.cuda.nvtx.range_push("timed_" + ("fp64" if precision == 0 else "mixed"))
        N.check(L.nsg_event_record(ctx, 0), "event")
        for _ in range(steps):
            step(precision)
        N.check(L.nsg_event_record(ctx, 1), "event")
        torch.cuda.nvtx.range_pop()
        ms = ctypes.c_double()
        N.check(L.nsg_event_elapsed(ctx, 0, 1, ctypes.byref(ms)), "elapsed")
        return ms.value / steps

    def results():
        vol = np.zeros(nstruct)
        area = np.zeros(nstruct)
        N.check(L.nsg_batch_results(ctx, N.ptr(vol), N.ptr(area)), "batch results")
        return vol, area

    # the metric's accuracy terms (untimed): every hit of the mixed-precision ray cast against the
    # double-precision one, status and insideness decisions, near-node counts
    accuracy = mixed_vs_fp64_accuracy(L, N, ctx, surfs, N.STATUS | N.ACCURATE_TRIANGULATION)
    # double-precision batch: reference numbers for the volume / area comparison
    step(0)
    vol64, area64 = results()
    # per-stage kernel times of the measured precision from one profiled pass, with the ray sets
    # one after another so that each kernel's event interval holds that kernel alone
    step(prec)
    tun = (ctypes.c_int32 * 5)()
    N.check(L.nsg_get_tuning(ctx, tun, 5), "tuning")
    serial = (ctypes.c_int32 * 5)(*tun)
    serial[3] = 0
    N.check(L.nsg_set_tuning(ctx, serial, 5), "tuning")
    N.check(L.nsg_profile(ctx, 1), "profile")
    step(prec)
    stage_ms = np.zeros(12)
    stage_calls = np.zeros(12, np.int64)
    L.nsg_stage_times(ctx, stage_ms.ctypes.data, stage_calls.ctypes.data, 12)
    counters = np.zeros(8, np.int64)
    L.nsg_trace_counters(ctx, counters.ctypes.data, 8)
    N.check(L.nsg_profile(ctx, 0), "profile")
    N.check(L.nsg_set_tuning(ctx, tun, 5), "tuning")

    for _ in range(args.warmup):
        nv, nt = step(prec)
    st = np.zeros(8, np.int64)
    N.check(L.nsg_stats(ctx, N.ptr(st), 8), "stats")
    active_cubes = int(st[4])
    barrier()
    clk = ClockSampler(local)
    clk.start()
    launches0 = L.nsg_launch_count(ctx)
    ms_per_step = timed(prec, args.steps)
    launches = L.nsg_launch_count(ctx) - launches0
    barrier()
    clocks = clk.stop()
    ms_per_step = max_over_ranks(ms_per_step)
    vol, area = results()

    # the same batch in double precision, and the plain per-structure double-precision path
    ms_fp64_batch = max_over_ranks(timed(0, max(1, min(args.steps, 3))))
    plain = nb.Context(local)
    dev = torch.device("cuda", local)
    dpatch = []
    plain_off = [np.array([0, len(sf.patches.built_from)], np.int64) for sf in surfs]
    for sf in surfs:
        p = sf.patches
        dpatch.append([torch.from_numpy(x).to(dev) for x in (p.f64, p.i32, p.pool, p.pool_flag)])
    torch.cuda.synchronize()

    def plain_pass(count: int) -> None:
        for b in range(count):
            sf, (f64, i32, pool, flag) = surfs[b], dpatch[b]
            p = sf.patches
            N.check(L.nsg_set_grid(plain.handle, ctypes.byref(sf.delphi.grid)), "set_grid")
            N.check(L.nsg_bind_patches_device(plain.handle, p.n, f64.data_ptr(), i32.data_ptr(), len(p.pool),
                                              pool.data_ptr(), flag.data_ptr(), p.probe), "bind")
            N.check(L.nsg_upload_atoms(plain.handle, N.ptr(plain_off[b]), N.ptr(p.built_from), N.ptr(p.atoms_of)),
                    "atoms")
            v = ctypes.c_double()
            N.check(L.nsg_raycast(plain.handle, flags, 0, ctypes.byref(v)), "raycast")
            a = ctypes.c_double()
            nv_, nt_ = ctypes.c_int64(), ctypes.c_int64()
            N.check(L.nsg_triangulate(plain.handle, ctypes.byref(a), ctypes.byref(nv_), ctypes.byref(nt_)), "tri")
            rc = L.nsg_atom_grads(plain.handle, None, None)
            if rc not in (N.NSG_OK, -8):
                N.check(rc, "atom gradients")

    plain_pass(min(8, nstruct))
    torch.cuda.synchronize()
    N.check(L.nsg_event_record(plain.handle, 0), "event")
    plain_pass(nstruct)
    N.check(L.nsg_event_record(plain.handle, 1), "event")
    pms = ctypes.c_double()
    N.check(L.nsg_event_elapsed(plain.handle, 0, 1, ctypes.byref(pms)), "elapsed")
    ms_plain = max_over_ranks(pms.value)
    plain.close()
    del dpatch

    # e2e: the ensemble from pinned host memory through the public API, chunked over two contexts
    # so that each chunk's host-to-device copy overlaps the previous chunk's kernels; per-structure
    # volumes, areas and atom derivatives back to the host
    batch.close()
    from nanoshaper_b200.pipelined import PipelinedBatches
    runner = PipelinedBatches(surfs, n_chunks=8, device=local, precision=args.precision, tuning=tuning,
                              n_contexts=4)
    h2d, d2h = runner.h2d_bytes, runner.d2h_bytes
    # the host link's copy rate (pinned host to device, the largest chunk's patch records, event
    # timed): with it the step's inputs give the transfer floor of the e2e figure
    big = max(runner.chunks, key=lambda ch: ch.pin["f64"].numel()).pin["f64"]
    link_dst = torch.empty(big.numel(), dtype=torch.uint8, device=f"cuda:{local}")
    link_dst.copy_(big, non_blocking=True)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(3):
        link_dst.copy_(big, non_blocking=True)
    ev1.record()
    torch.cuda.synchronize()
    link_gbs = 3 * big.numel() / (ev0.elapsed_time(ev1) / 1000.0) / 1e9
    del link_dst
    runner.run()
    barrier()
    e2e_steps = max(2, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        vol_e2e, area_e2e = runner.run()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) / e2e_steps * 1000.0)
    runner.close()
    e2e_matches = bool(np.allclose(vol_e2e, vol, rtol=1e-12, atol=0) and np.allclose(area_e2e, area, rtol=1e-12, atol=0))

    # end to end from the atoms: grids, jitter and SES patch construction on the host threads
    # (overlapped with the device work of the chunks already built), then the same step
    from nanoshaper_b200.pipelined import AtomsPipeline
    ap = AtomsPipeline(atoms, probe=w["probe"], scale=w["scale"], perfil=w["perfil"], n_chunks=8, device=local,
                       precision=args.precision, tuning=tuning)
    ap.run()
    barrier()
    t0 = time.perf_counter()
    ap_steps = max(2, min(args.steps, 3))
    for _ in range(ap_steps):
        vol_ap, area_ap = ap.run()
    ap_ms = max_over_ranks((time.perf_counter() - t0) / ap_steps * 1000.0)
    ap_h2d, ap_d2h = ap.h2d_bytes, ap.d2h_bytes
    ap.close()
    ap_matches = bool(np.allclose(vol_ap, vol, rtol=1e-12, atol=0) and np.allclose(area_ap, area, rtol=1e-12, atol=0))

    grids_l = [sf.delphi.grid for sf in surfs]
    rays = sum(rays_of(g) for g in grids_l)
    nodes = sum(g.nx * g.ny * g.nz for g in grids_l)
    nwords = sum(((g.nx + 31) // 32) * g.ny * g.nz for g in grids_l)
    structs_per_s = D.throughput(nstruct, world, ms_per_step)
    hit_store_gb = max(sum(g.ny * g.nz for g in grids_l), sum(g.nx * g.ny for g in grids_l),
                       sum(g.nx * g.nz for g in grids_l)) * 32 * 8 / 1e9

    peaks = load_peaks()
    stage_times = {STAGES[i]: float(stage_ms[i]) for i in range(len(STAGES))}
    # The dominant kernels are the intersection kernels (the largest share of the trace stage),
    # bound by FP64 arithmetic: achieved = the algorithmic operation model (OPS_PER_CANDIDATE) x
    # candidates / their event-timed time, against the FP64 rate of this GPU measured live with FMA
    # chains; the executed-instruction count from ncu (FLOPS_PER_CANDIDATE) is reported beside it.
    n_tor = int(counters[1])
    n_sph = int(counters[0]) - n_tor
    flops_model = n_tor * OPS_PER_CANDIDATE["torus"]["flops"] + n_sph * OPS_PER_CANDIDATE["sphere"]["flops"]
    special = {k: n_tor * OPS_PER_CANDIDATE["torus"].get(k, 0.0) + n_sph * OPS_PER_CANDIDATE["sphere"].get(k, 0.0)
               for k in ("sqrt", "div", "cbrt", "acos", "cos")}
    flops64 = n_tor * FLOPS_PER_CANDIDATE["torus"]["fp64"] + n_sph * FLOPS_PER_CANDIDATE["sphere"]["fp64"]
    flops32 = n_tor * FLOPS_PER_CANDIDATE["torus"]["fp32"] + n_sph * FLOPS_PER_CANDIDATE["sphere"]["fp32"]
    isect_s = stage_times["isect"] / 1000.0
    pk64, pk32 = ctypes.c_double(), ctypes.c_double()
    pctx = nb.Context(local)
    N.check(L.nsg_fp_peak(pctx.handle, 0, ctypes.byref(pk64)), "fp64 peak")
    N.check(L.nsg_fp_peak(pctx.handle, 1, ctypes.byref(pk32)), "fp32 peak")
    pctx.close()
    ach_model = flops_model / isect_s / 1e12 if isect_s > 0 else 0.0
    ach64 = flops64 / isect_s / 1e12 if isect_s > 0 else 0.0
    ach32 = flops32 / isect_s / 1e12 if isect_s > 0 else 0.0
    # the memory-side figure of the trace stage's fill kernel (bit grids, interval sums, pairs)
    fill_bytes = 3 * 2 * 4 * nwords + 8 * rays + 16 * nv
    roofline = {"bound": "fp64", "kernel": "k_isect (ray-patch intersection, 4 ray sets)", "achieved": ach_model,
                "peak": pk64.value / 1e12, "unit": "TFLOP/s", "frac": ach_model / (pk64.value / 1e12),
                "work": "algorithmic operation model of the oracle (OPS_PER_CANDIDATE) x the step's candidates; "
                        "isect time from the profiled pass with the ray sets run one after another",
                "ops_per_step": {"flops": flops_model, **special},
                "executed": {"note": "ncu-counted FP64/FP32 instructions per candidate (FLOPS_PER_CANDIDATE)",
                             "fp64_tflops": ach64, "fp64_frac": ach64 / (pk64.value / 1e12)},
                "traffic": (n_tor + n_sph) * ISECT_DRAM_BYTES_PER_CANDIDATE,
                "traffic_note": "DRAM bytes of the step's intersection launches: ncu-measured bytes per candidate "
                                "on the 64-structure ensemble x this step's candidates",
                "peak_source": "measured live: FMA chains on this GPU (nsg_fp_peak)",
                "flops_per_step": {"fp64": flops64, "fp32": flops32},
                "fp32": {"achieved": ach32, "peak": pk32.value / 1e12, "frac": ach32 / (pk32.value / 1e12)},
                "hbm_fill": {"kernel": "k_fill", "achieved_gbs": fill_bytes / (stage_times["fill"] / 1000.0) / 1e9
                             if stage_times["fill"] > 0 else 0.0, "peak_gbs": peaks["hbm_gbs"],
                             "peak_source": peaks["source"]},
                "stage_ms": stage_times}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = ensemble_cpu_baseline(surfs, os.cpu_count() or 1)
            cpu = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
            cpu["rays_per_s"] = cb["rays_per_s"]
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "structures/s", "cores": 0, "kind": "port", "sample": f"failed: {e}"}

    def rel(a, b):
        return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))

    if rank == 0:
        line = {
            "metric": METRIC, "value": structs_per_s, "unit": "structures/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "precision": args.precision, "data": "synthetic",
            "rays_per_s": structs_per_s * rays / nstruct, "nodes_per_s": structs_per_s * nodes / nstruct,
            "config": {"workload": args.workload, "structures": nstruct,
                       "atoms_total": int(sum(len(a) for a in atoms)), "probe": w["probe"], "scale": w["scale"],
                       "perfil": w["perfil"], "rays_per_step": rays, "nodes_per_step": nodes,
                       "outputs": "volume, area, d volume / d atoms, d area / d atoms per structure",
                       "tuning": {"isect_threads": tuning[0], "isect_blocks_per_sm": tuning[1],
                                  "cand_threads": tuning[2], "raycast_ms": tune_ms},
                       "l2": "inputs larger than L2 (hit store %.1f GB, bit grids %.2f GB)" % (
                           hit_store_gb, nwords * 4 / 1e9),
                       "parallelism": f"replicas x{world}"},
            "comparison": {
                "fp64_batched_structures_per_s": world * nstruct * 1000.0 / ms_fp64_batch,
                "fp64_plain_per_structure_structures_per_s": world * nstruct * 1000.0 / ms_plain,
                "speedup_vs_fp64_plain": ms_plain / ms_per_step,
                "speedup_vs_fp64_batched": ms_fp64_batch / ms_per_step,
                "max_rel_volume_diff_vs_fp64": rel(vol, vol64), "max_rel_area_diff_vs_fp64": rel(area, area64),
                "accuracy_vs_fp64": accuracy,
            },
            "result": {"volume_sum": float(vol.sum()), "area_sum": float(area.sum()), "vertices": nv,
                       "triangles": nt, "active_cubes": active_cubes},
            "host": {"patch_build_s": t_build, "generator_s": t_gen},
            "clocks": clocks,
            "e2e": {"value": world * nstruct * 1000.0 / e2e_ms, "unit": "structures/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms,
                    "method": "8 chunks (the first half-size) on 4 contexts, one upload at a time, copies "
                              "overlapped with compute (PipelinedBatches)",
                    "h2d_link_gbs": link_gbs, "transfer_floor_ms": h2d / link_gbs / 1e6,
                    "results_match_resident_run": e2e_matches},
            "e2e_from_atoms": {"value": world * nstruct * 1000.0 / ap_ms, "unit": "structures/s", "ms_per_step": ap_ms,
                               "h2d_bytes_per_step": int(ap_h2d), "d2h_bytes_per_step": int(ap_d2h),
                               "host_threads": os.cpu_count() or 1,
                               "method": "per step: grids, jitter and SES patch construction of every structure on "
                                         "the host threads (one single-threaded build per structure), 8 chunks "
                                         "handed to two GPU contexts as they complete (AtomsPipeline)",
                               "results_match_resident_run": ap_matches},
            "gpu_launches": int(launches),
            "trace_counters": dict(zip(("candidates", "torus_candidates", "deferred_sphere", "deferred_quartic",
                                        "deferred_root"), counters[:5].tolist())),
            "roofline": roofline,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    D.close(pg)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--workload", default="ensemble_512", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default=None, choices=("fp64", "mixed"),
                    help="default: mixed for the ensembles, fp64 for single structures")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tuning", default=None,
                    help="fixed tracer launch shapes 'isect_threads,isect_blocks_per_sm,cand_threads' "
                         "instead of the autotuner (ensembles)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    if args.precision is None:
        args.precision = "mixed" if args.workload.startswith("ensemble") else "fp64"
    world, rank, local = dist_setup()
    if args.workload.startswith("ensemble"):
        return run_ensemble(args, world, rank, local)

    if args.impl == "reference":
        if rank != 0:
            return
        w, atoms, ds, surf, t_gen, t_build = make_workload(args.workload)
        cb = run_reference(args, w, ds, surf)
        g = ds.grid
        line = {
            "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "structures/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "rays_per_s": cb["rays_per_s"],
            "config": {"workload": args.workload, "atoms": w["n"], "probe": w["probe"], "scale": w["scale"],
                       "perfil": w["perfil"], "grid": [g.nx, g.ny, g.nz], "patches": surf.patches.n},
            "cpu_baseline": {"value": cb["value"], "unit": "structures/s", "cores": cb["cores"], "kind": cb["kind"],
                             "sample": cb["sample"]},
            "e2e": {"value": cb["value"], "unit": "structures/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return

    import torch
    from nanoshaper_b200 import dist as D
    torch.cuda.set_device(local)
    pg = D.init("nccl")

    import nanoshaper_b200 as nb
    from nanoshaper_b200 import _native as N
    from nanoshaper_b200 import build as nbuild
    nbuild.build()
    L = N.lib()

    w, atoms, ds, surf, t_gen, t_build = make_workload(args.workload)
    surf.device = local
    surf.precision = args.precision
    g = ds.grid
    p = surf.patches
    ctx = surf._context().handle
    prec = 0 if args.precision == "fp64" else 1
    surf.precision = args.precision
    flags = N.STATUS | N.ACCURATE_TRIANGULATION

    def barrier():
        D.barrier(pg)
        torch.cuda.synchronize()

    # device-resident inputs
    surf.upload()

    def step():
        v = ctypes.c_double()
        N.check(L.nsg_raycast(ctx, flags, prec, ctypes.byref(v)), "raycast")
        nc = ctypes.c_int()
        N.check(L.nsg_cavities(ctx, w["cav_vol"], ctypes.byref(nc)), "cavities")
        a = ctypes.c_double()
        nv = ctypes.c_int64()
        nt = ctypes.c_int64()
        N.check(L.nsg_triangulate(ctx, ctypes.byref(a), ctypes.byref(nv), ctypes.byref(nt)), "triangulate")
        return v.value, a.value, nc.value, nv.value, nt.value

    # per-stage kernel times from one profiled (untimed) pass, after a first pass that sizes the
    # context's buffers
    step()
    N.check(L.nsg_profile(ctx, 1), "profile")
    step()
    stage_ms = np.zeros(12)
    stage_calls = np.zeros(12, np.int64)
    L.nsg_stage_times(ctx, stage_ms.ctypes.data, stage_calls.ctypes.data, 12)
    counters = np.zeros(8, np.int64)
    L.nsg_trace_counters(ctx, counters.ctypes.data, 8)
    N.check(L.nsg_profile(ctx, 0), "profile")
    stats = surf.stats()

    for _ in range(args.warmup):
        step()
    barrier()
    clk = ClockSampler(local)
    clk.start()
    launches0 = L.nsg_launch_count(ctx)
    N.check(L.nsg_event_record(ctx, 0), "event")
    for _ in range(args.steps):
        vol, area, ncav, nv, nt = step()
    N.check(L.nsg_event_record(ctx, 1), "event")
    ms = ctypes.c_double()
    N.check(L.nsg_event_elapsed(ctx, 0, 1, ctypes.byref(ms)), "elapsed")
    launches = L.nsg_launch_count(ctx) - launches0
    barrier()
    clocks = clk.stop()
    ms_per_step = D.max_over_ranks(pg, ms.value / args.steps)

    rays_per_struct = g.nz * g.ny + (g.nz * g.ny + g.ny * g.nx + g.nz * g.nx)
    nodes = g.nx * g.ny * g.nz
    structs_per_s = D.throughput(1, world, ms_per_step)
    rays_per_s = structs_per_s * rays_per_struct
    nodes_per_s = structs_per_s * nodes

    # e2e through the C-ABI with pinned host buffers
    pin = {}
    for name in ("f64", "i32", "pool", "pool_flag"):
        a = getattr(p, name)
        t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
        t.numpy()[:] = a.view(np.uint8).ravel()
        pin[name] = t
    status_host = torch.empty(nodes * 4, dtype=torch.uint8, pin_memory=True)
    verts_host = torch.empty(max(nv, 1) * 24 + 4096, dtype=torch.uint8, pin_memory=True)
    keys_host = torch.empty(max(nv, 1) * 16 + 4096, dtype=torch.uint8, pin_memory=True)
    tris_host = torch.empty(max(nt, 1) * 12 + 4096, dtype=torch.uint8, pin_memory=True)
    h2d = sum(t.numel() for t in pin.values())

    def e2e_step():
        N.check(L.nsg_upload_patches(ctx, p.n, pin["f64"].data_ptr(), pin["i32"].data_ptr(), len(p.pool),
                                     pin["pool"].data_ptr(), pin["pool_flag"].data_ptr(), p.probe), "upload")
        r = step()
        N.check(L.nsg_download_status(ctx, status_host.data_ptr()), "download status")
        N.check(L.nsg_download_mesh(ctx, verts_host.data_ptr(), keys_host.data_ptr(), tris_host.data_ptr()), "mesh")
        return r

    e2e_steps = max(2, min(args.steps, 5))
    e2e_step()
    barrier()
    N.check(L.nsg_event_record(ctx, 2), "event")
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        r = e2e_step()
    N.check(L.nsg_event_record(ctx, 3), "event")
    e2e_wall = (time.perf_counter() - t0) / e2e_steps
    e_ms = ctypes.c_double()
    N.check(L.nsg_event_elapsed(ctx, 2, 3, ctypes.byref(e_ms)), "elapsed")
    e2e_ms = D.max_over_ranks(pg, max(e_ms.value / e2e_steps, e2e_wall * 1000.0))
    d2h = nodes * 4 + r[3] * (24 + 16) + r[4] * 12

    # roofline of the dominant stage (HBM: algorithmic bytes per launch / measured launch time)
    peaks = load_peaks()
    stage_times = {STAGES[i]: float(stage_ms[i]) for i in range(len(STAGES))}
    dominant = max(stage_times, key=stage_times.get)
    nwords = ((g.nx + 31) // 32) * g.ny * g.nz
    ncav_nodes = nodes  # cavity pass streams the whole status map
    alg_bytes = {
        # status rows written (4 B/node) + bit grid (cleared by three ray sets, read+write) +
        # per-ray interval-length words and pair records of the triangulation rays
        "trace": 4 * nodes + 3 * 2 * 4 * nwords + 8 * rays_per_struct + 16 * nv,
        "overflow": 4 * nodes,
        "bin": 6 * 4 * p.n,
        # union-find: status read (init, hook), labels write+read (init, hook, compress, stats,
        # label), status write (label) -- 4 B each
        "cavity": 4 * ncav_nodes * 8,
        "vertex": 8 * 2 * nv + 40 * nv,
        "mc": nwords * 4 * 8 + 40 * nv + 12 * nt,
    }
    dom_ms = stage_times[dominant] / max(int(stage_calls[STAGES.index(dominant)]), 1)
    achieved = alg_bytes[dominant] / (dom_ms / 1000.0) / 1e9
    roofline = {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": None, "peak_source": peaks["source"],
                "stage_ms": stage_times, "algorithmic_bytes": alg_bytes[dominant]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cb = run_reference(argparse.Namespace(steps=1, warmup=0), w, ds, surf)
            cpu = {"value": cb["value"], "unit": "structures/s", "cores": cb["cores"], "kind": cb["kind"],
                   "sample": cb["sample"], "rays_per_s": cb["rays_per_s"]}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "structures/s", "cores": 0, "kind": "port", "sample": f"failed: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": structs_per_s, "unit": "structures/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "precision": args.precision, "data": "synthetic",
            "rays_per_s": rays_per_s, "nodes_per_s": nodes_per_s,
            "config": {"workload": args.workload, "atoms": w["n"], "probe": w["probe"], "scale": w["scale"],
                       "perfil": w["perfil"], "grid": [g.nx, g.ny, g.nz], "patches": p.n,
                       "patch_kinds": list(p.counts), "rays_per_structure": rays_per_struct,
                       "l2": "inputs larger than L2 (status map %.1f GB)" % (nodes * 4 / 1e9),
                       "parallelism": f"replicas x{world}"},
            "result": {"volume": vol, "area": area, "cavities": ncav, "vertices": nv, "triangles": nt,
                       "overflow_rays": stats["overflow_rays"]},
            "host": {"patch_build_s": t_build, "generator_s": t_gen},
            "clocks": clocks,
            "e2e": {"value": world * 1000.0 / e2e_ms, "unit": "structures/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms},
            "gpu_launches": int(launches),
            "trace_counters": dict(zip(("candidates", "torus_candidates", "fallback_sphere", "fallback_quartic",
                                        "fallback_root"), counters[:5].tolist())),
            "roofline": roofline,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    surf.ctx.close()
    D.close(pg)


if __name__ == "__main__":
    main()
