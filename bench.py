"""Benchmark of the grid-block evaluator on the 740-function workload.

Workload (one "step"): rho, grad rho, lap rho, tau and ELF of the total
density of a seeded C12N4O4H20 molecule (740 spherical AOs, 76 doubly
occupied MOs, written as FCHK) on a 128^3 grid at 0.2 bohr centred on the
atoms (2,097,152 points), AUTO backend (AO-MO), block 128, screening 1e-12.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl kumo|reference]

value: grid points/s of the mixed-precision form with the molecule resident
and outputs left in HBM (device API), max over ranks; `fp64` holds the same
for the FP64 form.  e2e: the same metric through the host C-ABI call
(kumo_evaluate_grid, host output arrays, device-to-host copies inside the
timed region).  Under torchrun the ranks split the one grid into slabs of
whole planes (kumo_b200.shard.slab_range), each rank evaluating its slab as a
grid of its own; no collective on the data path (strong scaling).  At one GPU
the run adds the unrestricted-triplet workload (`triplet`), the
electrostatic potential (`esp`) and the serving loop (`serve`).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "chem-kumo_b200"))

WORKLOAD = "organic_740"
METRIC = "grid pts/s (ρ,∇ρ,∇²ρ,τ,ELF) mixed vs FP64 on B200 @≤1e-7 rel; serve p50/p99 ms"
L2_FLUSH_BYTES = 256 << 20


def _props(K):
    P = K.PropertyKind
    return [K.density(P.Density), K.density(P.Gradient), K.density(P.Laplacian), K.density(P.Tau), K.density(P.Elf)]


def _synth_dir() -> str:
    d = os.environ.get("KUMO_SYNTH_CACHE") or os.path.join(tempfile.gettempdir(), "kumo_b200_synth")
    os.makedirs(d, exist_ok=True)
    return d


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return p, "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"kumo_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for name, v in zip(names, r[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        loaded = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def cpu_baseline(fchk: str, grid, nblocks_sample: int, threads: int = 0):
    """Oracle restatement of the reference's CPU path on a bounded sample of the
    workload's 128-point blocks (evenly spaced over the grid), all host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    o = O.OracleMolecule.from_fchk(fchk)
    pts = grid.points()
    nb = (len(pts) + 127) // 128
    pick = np.unique(np.linspace(0, nb - 1, nblocks_sample).astype(int))
    sample = np.concatenate([pts[b * 128:(b + 1) * 128] for b in pick])
    props = [(0, 0, 0, 0), (1, 0, 0, 0), (3, 0, 0, 0), (4, 0, 0, 0), (6, 0, 0, 0)]
    o.evaluate(props, points=sample[:256], threads=threads)  # warm-up
    t0 = time.perf_counter()
    o.evaluate(props, points=sample, threads=threads)
    dt = time.perf_counter() - t0
    cores = threads if threads > 0 else O.lib().ko_max_threads()
    return {"value": len(sample) / dt, "unit": "grid pts/s", "cores": cores, "kind": "port",
            "sample": f"{len(pick)} evenly spaced 128-point blocks ({len(sample)} points) of the 128^3 grid, "
                      f"{dt:.1f} s"}


def run_reference(args, rank: int) -> None:
    """--impl reference: the CPU restatement of the reference path (oracle port),
    all host threads, each step a bounded sample of the workload."""
    if rank != 0:
        return
    import kumo_b200.synth as synth
    from kumo_b200 import Grid

    fchk = synth.workload_fchk(WORKLOAD, _synth_dir())
    rec = synth.read_fchk(fchk)
    coords = np.asarray(rec["Current cartesian coordinates"]).reshape(-1, 3)
    origin, steps, counts = synth.workload_grid(WORKLOAD, coords)
    grid = Grid(origin, steps, counts)
    vals = []
    info = None
    for i in range(args.warmup + args.steps):
        info = cpu_baseline(fchk, grid, args.ref_blocks)
        if i >= args.warmup:
            vals.append(info["value"])
    value = float(np.median(vals))
    line = {"metric": METRIC, "value": value, "unit": "grid pts/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 2097152 / value * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded FCHK)",
            "config": {"workload": "organic_740 (C12N4O4H20, 740 AOs, 76 occ MOs) rho/grad/lap/tau/ELF on 128^3 @0.2 bohr",
                       "backend": "AO_MO", "block": 128, "threshold": 1e-12},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "grid pts/s", "cores": info["cores"], "kind": "port",
                             "sample": info["sample"]},
            "e2e": {"value": value, "unit": "grid pts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def field_errors(torch, a, r, rho, kind_positive: bool):
    """Errors of one field (channels x points, device tensors) against FP64:
    `abs` = max |a - r|, `scaled` = max|a - r| / max(1, max|r|) (chem-kumo's
    tests/density_screening_test.cpp:137-150), `pointwise` = max |a - r| /
    max(1, |a|, |r|) (tests/test_support.hpp:68-76), and for fields that are
    positive wherever rho > 1e-6 (rho, tau, ELF, RDG, the spin densities)
    `rel` = max |a - r| / |r| over those points."""
    d = (a - r).abs()
    out = {"abs": float(d.max()),
           "scaled": float(d.max() / max(1.0, float(r.abs().max()))),
           "pointwise": float((d / torch.clamp(torch.maximum(a.abs(), r.abs()), min=1.0)).max())}
    if kind_positive:
        m = rho > 1e-6
        out["rel"] = float((d[:, m] / r[:, m].abs().clamp_min(1e-300)).max()) if bool(m.any()) else 0.0
    return out


def triplet_bench(K, synth, d: str, grid_n: int = 0, steps: int = 1, peaks=None):
    """Unrestricted-triplet workload: C60N20O20H100 (3,700 AOs, 381 alpha and
    379 beta electrons, seed 2), alpha, beta and spin densities, RDG and
    sign(lambda2) rho (the full AO Hessian) on its 192^3 grid at 0.17 bohr,
    screening threshold 1e-10; FP64 and mixed forms of the AO-MO (AUTO's
    choice) and AO-P backends, one warm-up and `steps` timed steps each, and
    the mixed-vs-FP64 errors per field."""
    import torch
    fchk = synth.workload_fchk("triplet_3700", d)
    m = K.Molecule.from_fchk(fchk)
    _, _, xyz = m.atoms()
    origin, st, counts = synth.workload_grid("triplet_3700", xyz)
    if grid_n:
        origin = xyz.mean(axis=0) - 0.5 * st[0, 0] * (grid_n - 1)
        counts = (grid_n,) * 3
    grid = K.Grid(origin, st, counts)
    n = grid.npoints
    P, D = K.PropertyKind, K.DensityComponent
    props = [K.density(P.Density, D.Alpha), K.density(P.Density, D.Beta), K.density(P.Density, D.Difference),
             K.density(P.ReducedGradient), K.density(P.SignLambda2Density)]
    names = ["rho_alpha", "rho_beta", "spin", "rdg", "sign_lambda2_rho"]
    positive = [True, True, False, True, False]
    stream = torch.cuda.current_stream()
    peaks = peaks or {}
    res = {"workload": f"triplet_3700 (C60N20O20H100, 3700 AOs, 381/379 electrons) alpha/beta/spin density, "
                       f"RDG, sign(lambda2)rho on {counts[0]}^3 @0.17 bohr, threshold 1e-10",
           "points": n}
    for backend in (K.Backend.AO_MO, K.Backend.AO_P):
        outs = {}
        for prec in (K.Precision.FP64, K.Precision.Mixed):
            ev = K.Evaluator(m, backend=backend, threshold=1e-10, precision=prec)
            out = torch.empty(5 * n, dtype=torch.float64, device="cuda")
            ptrs = [out.data_ptr() + 8 * i * n for i in range(5)]
            used = ev.evaluate_grid_device(grid, props, ptrs, stream.cuda_stream)  # warm-up
            assert used == int(backend)
            torch.cuda.synchronize()
            K.profile_reset()
            K.profile_enable(True)
            ts = []
            for _ in range(steps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ev.evaluate_grid_device(grid, props, ptrs, stream.cuda_stream)
                e1.record(stream)
                ts.append((e0, e1))
            torch.cuda.synchronize()
            ms = float(np.mean([a.elapsed_time(b) for a, b in ts]))
            prof = K.profile_read()
            K.profile_enable(False)
            kern = {k: {"launches": v["launches"], "ms": round(v["ms"], 3)} for k, v in prof.items() if v["launches"]}
            ck = "contract_p" if backend == K.Backend.AO_P else (
                "contract_mixed" if prec == K.Precision.Mixed else "contract_mo_f64")
            entry = {"ms_per_step": ms, "pts_per_s": n / (ms * 1e-3), "kernels": kern}
            c = prof.get(ck, {})
            if c.get("launches"):
                tf = c["flops"] / (c["ms"] * 1e-3) / 1e12
                if prec == K.Precision.Mixed:
                    peak, unit = peaks.get("bf16_tflops", 1590.0), "bf16 TFLOP/s (measured burst peak)"
                else:
                    peak, unit = 37.0, "FP64 TFLOP/s (nominal B200 FP64 peak)"
                entry["roofline"] = {"kernel": ck, "achieved_tflops": tf, "peak": peak, "peak_unit": unit,
                                     "frac": tf / peak,
                                     "algorithmic": ("2 * m_kept^2 * 128 * left panels per block and density "
                                                     "matrix (4 panels; 1 for a matrix whose components need "
                                                     "values only)"
                                                     if backend == K.Backend.AO_P else
                                                     "2 * 128 * 10 panels * m_kept * (n_alpha + n_beta) per block")}
            res[f"{backend.name}_{prec.name}"] = entry
            outs[prec] = out
        f64, mix = outs[K.Precision.FP64], outs[K.Precision.Mixed]
        rho = f64[:n] + f64[n:2 * n]
        res[f"{backend.name}_mixed_vs_fp64"] = {
            name: field_errors(torch, mix[i * n:(i + 1) * n].view(1, n), f64[i * n:(i + 1) * n].view(1, n), rho, pos)
            for i, (name, pos) in enumerate(zip(names, positive))}
        res[f"{backend.name}_mixed_over_fp64"] = (res[f"{backend.name}_FP64"]["ms_per_step"] /
                                                  res[f"{backend.name}_Mixed"]["ms_per_step"])
        del outs, f64, mix
    return res


def _serve_arrivals(K, srv, precision: int, seconds: float, rate: float, pool, seed: int):
    """Submit the serving workload's Poisson arrivals to `srv` for `seconds`;
    returns the tickets and the count of each request type."""
    P = K.PropertyKind
    rng = np.random.default_rng(seed)
    dens = [P.Density, P.Gradient, P.Laplacian, P.Tau, P.Elf, P.Lol]
    t0 = time.perf_counter()
    t_next = 0.0
    tickets, kinds = [], {"cube": 0, "plane": 0, "line": 0, "points": 0}
    while True:
        t_next += rng.exponential(1.0 / rate)
        if t_next > seconds:
            break
        m, xyz, nalpha, nmo = pool[int(rng.integers(len(pool)))]
        c = xyz.mean(axis=0)
        kind = ["cube", "plane", "line", "points"][int(rng.integers(4))]
        kinds[kind] += 1
        props = []
        for _ in range(int(rng.integers(1, 4))):
            choice = int(rng.integers(len(dens) + 2))
            if choice < len(dens):
                props.append(K.density(dens[choice]))
            elif choice == len(dens):
                props.append(K.orbital(int(min(max(1, nalpha + int(rng.integers(-2, 3))), nmo))))
            elif kind in ("line", "points"):
                props.append(K.density(P.ElectrostaticPotential))
        if not props:
            props = [K.density(P.Density)]
        now = time.perf_counter() - t0
        if t_next > now:
            time.sleep(t_next - now)
        if kind == "cube":
            e = int(rng.integers(40, 161))
            g = K.Grid(c - 0.1 * (e - 1), np.eye(3) * 0.2, (e, e, e))
            tickets.append(srv.submit_grid(m, g, props, precision=precision)[0])
        elif kind == "plane":
            g = K.Grid(c - np.array([19.9, 19.9, 0.0]), np.diag([0.2, 0.2, 1.0]), (200, 200, 1))
            tickets.append(srv.submit_grid(m, g, props, precision=precision)[0])
        elif kind == "line":
            a, b = xyz.min(0) - 3.0, xyz.max(0) + 3.0
            st = (b - a) / 999.0
            g = K.Grid(a, np.column_stack([st, [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]]), (1000, 1, 1))
            tickets.append(srv.submit_grid(m, g, props, precision=precision)[0])
        else:
            n = int(rng.integers(1, 1001))
            pts = rng.uniform(xyz.min(0) - 2.5, xyz.max(0) + 2.5, (n, 3))
            tickets.append(srv.submit_points(m, pts, props, precision=precision)[0])
    return tickets, kinds


def serve_bench(K, synth, precision: int, seconds: float, rate: float, pool, seed: int, graph_points: int = 65536,
                scratch_gb: float = 2.0, warmup_s: float = 0.0):
    """Serving loop under the serving workload: Poisson arrivals at `rate`
    requests/s for `seconds`, each request one type drawn uniformly (cube of
    40^3..160^3 points at 0.2 bohr, 200x200 plane at 0.2 bohr, 1000-point line,
    1..1000 scattered points) on a molecule drawn from the pool, with 1-3
    properties drawn from {rho, grad rho, lap rho, tau, ELF, LOL, MO homo-2 ..
    lumo+2, ESP} (ESP only on lines and point sets).  Latency runs from submit
    until the results are in the caller's arrays; the run ends when every
    request is done.

    With `warmup_s` > 0, that many seconds of the same arrivals (another seed)
    run first through a server of their own and are not counted, so that the
    stream-ordered memory pool has grown to the serving footprint (the server
    itself loads every kernel of the library when it is created).  The default
    measures a cold server."""
    kw = dict(max_active=8, graph_points=graph_points, request_scratch_bytes=scratch_gb * 2**30)
    if warmup_s > 0:
        warm = K.Server(**kw)
        wt, _ = _serve_arrivals(K, warm, precision, warmup_s, rate, pool, seed + 1000)
        for t in wt:
            warm.wait(t, 600.0)
        warm.close()
    srv = K.Server(**kw)
    t0 = time.perf_counter()
    tickets, kinds = _serve_arrivals(K, srv, precision, seconds, rate, pool, seed)
    submit_s = time.perf_counter() - t0
    for t in tickets:
        srv.wait(t, 600.0)
    s = srv.stats()
    srv.close()
    return {"requests": int(s["completed"]), "failed": int(s["failed"]), "p50_ms": s["p50_ms"],
            "p99_ms": s["p99_ms"], "mean_ms": s["mean_ms"], "pts_per_s": s["points_per_s"],
            "points": int(s["points"]), "busy_s": s["busy_s"], "graph_captures": int(s["graph_captures"]),
            "graph_replays": int(s["graph_replays"]), "direct_runs": int(s["direct_runs"]),
            "peak_hbm_gb": s["peak_bytes"] / 1e9, "budget_hbm_gb": s["budget_bytes"] / 1e9,
            "host_launch_s": s["launch_s"], "host_copy_s": s["copy_s"], "queue_ms": s["queue_ms"],
            "submit_s": submit_s, "mix": kinds, "warmup_s": warmup_s}


def esp_bench(K, synth, fchk_dir: str, oracle_pts: int = 32):
    """Electrostatic-potential workload: C30N3O3H24 cation (60 atoms, 1260 AOs),
    exact potential (tolerance 0) on its 96^3 cube at 0.24 bohr and on the
    rho = 0.001 isosurface vertices, then tolerances 1e-8 and 1e-6; unit:
    point-pair interactions."""
    import torch
    fchk = synth.workload_fchk("esp_1260", fchk_dir)
    m = K.Molecule.from_fchk(fchk)
    _, _, xyz = m.atoms()
    origin, steps, counts = synth.workload_grid("esp_1260", xyz)
    grid = K.Grid(origin, steps, counts)
    n = grid.npoints
    esp = K.density(K.PropertyKind.ElectrostaticPotential)
    ev = K.Evaluator(m)
    pairs = m.esp_pair_count()
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    ev.evaluate_grid_device(K.Grid(origin, steps, (8, 8, 8)), [esp], [out.data_ptr()], stream.cuda_stream)

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    ms_cube = timed(lambda: ev.evaluate_grid_device(grid, [esp], [out.data_ptr()], stream.cuda_stream))
    # The rho = 0.001 isosurface at the reference's default spacing (0.25 bohr):
    # device marching tetrahedra, vertices placed on the exact isosurface.
    t0 = time.perf_counter()
    mesh = K.density_isosurface(m, 1e-3, 0.25)
    surface_build_s = time.perf_counter() - t0
    surf = mesh.vertices
    dpts = torch.tensor(surf.ravel(), dtype=torch.float64, device="cuda")
    sout = torch.empty(len(surf), dtype=torch.float64, device="cuda")
    ms_surf = timed(lambda: ev.evaluate_points_device(dpts.data_ptr(), len(surf), [esp], [sout.data_ptr()],
                                                      stream.cuda_stream))
    # Opt-in mixed form (FP64 Boys values and nuclear term, FP32 Hermite
    # recursion and compensated pair sums) on the same cube and surface,
    # against FP64.
    os.environ["KUMO_ESP_MIXED"] = "1"
    evm = K.Evaluator(m, precision=K.Precision.Mixed)
    outm = torch.empty_like(out)
    soutm = torch.empty_like(sout)
    evm.evaluate_grid_device(K.Grid(origin, steps, (8, 8, 8)), [esp], [outm.data_ptr()], stream.cuda_stream)
    ms_cube_m = timed(lambda: evm.evaluate_grid_device(grid, [esp], [outm.data_ptr()], stream.cuda_stream))
    ms_surf_m = timed(lambda: evm.evaluate_points_device(dpts.data_ptr(), len(surf), [esp], [soutm.data_ptr()],
                                                         stream.cuda_stream))

    del os.environ["KUMO_ESP_MIXED"]

    def scaled(a, r):
        return float((a - r).abs().max() / max(1.0, float(r.abs().max())))

    # potential_tolerance > 0 (the reference's default 1e-8, and 1e-6): pairs
    # whose bounds sum to at most half the tolerance are dropped (set up once
    # per tolerance, untimed); max |error| against the exact values above.
    tolerance = {}
    for tol in (1e-8, 1e-6):
        evt = K.Evaluator(m, potential_tolerance=tol)
        outt, soutt = torch.empty_like(out), torch.empty_like(sout)
        evt.evaluate_grid_device(K.Grid(origin, steps, (8, 8, 8)), [esp], [outt.data_ptr()], stream.cuda_stream)
        used = m.esp_pairs_evaluated(tol)
        ms_c = timed(lambda: evt.evaluate_grid_device(grid, [esp], [outt.data_ptr()], stream.cuda_stream))
        ms_s = timed(lambda: evt.evaluate_points_device(dpts.data_ptr(), len(surf), [esp], [soutt.data_ptr()],
                                                        stream.cuda_stream))
        tolerance[f"{tol:g}"] = {"pairs_evaluated": int(used), "cube_ms": ms_c, "surface_ms": ms_s,
                                 "speedup_vs_exact_cube": ms_cube / ms_c, "speedup_vs_exact_surface": ms_surf / ms_s,
                                 "max_abs_err_vs_exact_cube": float((outt - out).abs().max()),
                                 "max_abs_err_vs_exact_surface": float((soutt - sout).abs().max())}

    mixed = {"opt_in": "KUMO_ESP_MIXED=1", "cube_ms": ms_cube_m, "cube_pair_points_per_s": n * pairs / (ms_cube_m * 1e-3),
             "surface_ms": ms_surf_m, "surface_pair_points_per_s": len(surf) * pairs / (ms_surf_m * 1e-3),
             "speedup_vs_fp64_cube": ms_cube / ms_cube_m, "speedup_vs_fp64_surface": ms_surf / ms_surf_m,
             "scaled_err_vs_fp64_cube": scaled(outm, out), "scaled_err_vs_fp64_surface": scaled(soutm, sout),
             "max_rel_err_vs_fp64_surface": float(((soutm - sout).abs() / sout.abs().clamp_min(1e-300)).max())}
    # Accuracy on a sample against the CPU oracle, and the oracle's own rate.
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    o = O.OracleESP(O.OracleMolecule.from_fchk(fchk))
    pick = np.linspace(0, len(surf) - 1, oracle_pts).astype(int)
    t0 = time.perf_counter()
    ref = o.evaluate(surf[pick])
    cpu_s = time.perf_counter() - t0
    got = sout.cpu().numpy()[pick]
    return {"workload": "esp_1260 (C30N3O3H24+, 60 atoms, 1260 AOs) exact ESP, 96^3 cube @0.24 bohr and "
                        "the vertices of its rho = 0.001 isosurface (0.25 bohr construction grid)",
            "pairs": int(pairs),
            "cube": {"points": n, "ms": ms_cube, "pair_points_per_s": n * pairs / (ms_cube * 1e-3),
                     "pts_per_s": n / (ms_cube * 1e-3)},
            "surface": {"points": len(surf), "triangles": int(len(mesh.triangles)),
                        "build_s": surface_build_s, "ms": ms_surf,
                        "pair_points_per_s": len(surf) * pairs / (ms_surf * 1e-3)},
            "scaled_err_vs_oracle": float(np.max(np.abs(got - ref)) / max(1.0, float(np.max(np.abs(ref))))),
            "mixed": mixed,
            "tolerance": tolerance,
            "cpu_oracle": {"pair_points_per_s": oracle_pts * pairs / cpu_s, "cores": O.lib().ko_max_threads(),
                           "sample": f"{oracle_pts} surface points, {cpu_s:.1f} s"}}


def serving_pool(K, synth, count: int, max_atoms: int, seed: int = 7):
    """The serving pool's molecules, built in a process pool (spawned)."""
    import concurrent.futures as cf
    import multiprocessing as mp
    specs = synth.serving_pool(count, seed, 3, max_atoms)
    t0 = time.perf_counter()
    # Largest molecules first, so that the process pool ends together; each
    # worker's BLAS gets its share of the cores (not all of them each).
    order = sorted(range(len(specs)), key=lambda i: -specs[i][1])
    workers = min(16, os.cpu_count() or 4)
    blas = {v: os.environ.get(v) for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")}
    for v in blas:
        os.environ[v] = str(max(1, (os.cpu_count() or 4) // workers))
    try:
        with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            built = list(ex.map(synth.serving_records, [specs[i] for i in order]))
    finally:
        for v, old in blas.items():
            if old is None:
                os.environ.pop(v, None)
            else:
                os.environ[v] = old
    recs = [None] * len(specs)
    for i, r in zip(order, built):
        recs[i] = r
    t1 = time.perf_counter()
    # Host-side loading (parsing the records, the orbital check) on threads.
    with cf.ThreadPoolExecutor(max_workers=workers) as ex:
        mols = list(ex.map(K.Molecule.from_records, recs))
    pool = []
    for r, m in zip(recs, mols):
        # Resident before serving: the device copy and the potential's primitive pairs.
        K.Evaluator(m).evaluate_points(np.zeros((1, 3)), [K.density(K.PropertyKind.Density),
                                                          K.density(K.PropertyKind.ElectrostaticPotential)])
        xyz = np.asarray(r["Current cartesian coordinates"], dtype=float).reshape(-1, 3)
        nmo = int(np.asarray(r["Alpha MO coefficients"]).size // int(r["Number of basis functions"]))
        pool.append((m, xyz, int(r["Number of alpha electrons"]), nmo))
    print(f"serving pool: {len(specs)} molecules built in {t1 - t0:.1f} s, loaded and made resident in "
          f"{time.perf_counter() - t1:.1f} s", file=sys.stderr)
    return pool, [n for _, n, _ in specs]


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="kumo", choices=["kumo", "reference"])
    ap.add_argument("--ref-blocks", type=int, default=2048, help="128-point blocks per reference step")
    ap.add_argument("--cpu-blocks", type=int, default=8192, help="128-point blocks of the CPU baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--grid-n", type=int, default=0, help="points per axis (default: the workload's 128)")
    ap.add_argument("--serve-seconds", type=float, default=5.0, help="arrival window of the serving run (0: skip)")
    ap.add_argument("--serve-warmup", type=float, default=0.0,
                    help="seconds of uncounted arrivals (own server, other seed) before the measured window")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="mean arrivals per second")
    ap.add_argument("--serve-pool", type=int, default=32, help="molecules in the serving pool")
    ap.add_argument("--serve-max-atoms", type=int, default=200, help="largest molecule of the serving pool")
    ap.add_argument("--serve-graph-points", type=int, default=65536, help="largest request replayed from a graph")
    ap.add_argument("--serve-scratch-gb", type=float, default=2.0, help="AO scratch per serving request")
    ap.add_argument("--serve-only", action="store_true", help="run the serving measurement only (prints its JSON)")
    ap.add_argument("--no-esp", action="store_true", help="skip the electrostatic-potential measurement")
    ap.add_argument("--esp-only", action="store_true", help="run the electrostatic-potential measurement only")
    ap.add_argument("--only", choices=["mixed", "fp64"], default=None,
                    help="time one form only (small profiling cases)")
    ap.add_argument("--no-triplet", action="store_true", help="skip the unrestricted-triplet workload")
    ap.add_argument("--triplet-only", action="store_true", help="run the unrestricted-triplet workload only")
    ap.add_argument("--triplet-grid-n", type=int, default=0, help="points per axis of the triplet grid (default 192)")
    ap.add_argument("--triplet-steps", type=int, default=1, help="timed steps of each triplet variant")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import torch.distributed as dist

    import kumo_b200 as K
    import kumo_b200.synth as synth

    torch.cuda.set_device(local)
    K.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    d = _synth_dir()
    if rank == 0:
        fchk = synth.workload_fchk(WORKLOAD, d)
    if world > 1:
        dist.barrier()
    fchk = synth.workload_fchk(WORKLOAD, d)
    m = K.Molecule.from_fchk(fchk)
    _, _, xyz = m.atoms()
    origin, steps, counts = synth.workload_grid(WORKLOAD, xyz)
    if args.grid_n:
        spacing = steps[0, 0]
        origin = xyz.mean(axis=0) - 0.5 * spacing * (args.grid_n - 1)
        counts = (args.grid_n,) * 3
    from kumo_b200 import shard
    n_total = int(np.prod(counts))
    # One grid over the ranks: each rank evaluates its slab of whole planes.
    i0, i1 = shard.slab_range(counts, rank, world)
    s_origin, s_steps, s_counts = shard.slab_grid(origin, steps, counts, i0, i1)
    grid = K.Grid(s_origin, s_steps, s_counts)
    n = grid.npoints
    props = _props(K)
    nchan = sum(K.channels(p.kind) for p in props)
    out = torch.empty(nchan * n, dtype=torch.float64, device="cuda")
    ptrs, off = [], 0
    for p in props:
        ptrs.append(out.data_ptr() + 8 * off)
        off += K.channels(p.kind) * n
    stream = torch.cuda.current_stream()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    ev = {"mixed": K.Evaluator(m, precision=K.Precision.Mixed), "fp64": K.Evaluator(m)}

    def step(name):
        used = ev[name].evaluate_grid_device(grid, props, ptrs, stream.cuda_stream)
        assert used == 2

    def timed(name, steps_):
        times = []
        for _ in range(steps_):
            flush.zero_()  # L2 flush between timed iterations (not timed)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step(name)
            e1.record(stream)
            times.append((e0, e1))
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in times]

    def max_over_ranks(x: float) -> float:
        return shard.max_over_ranks(x, dist, world, device="cuda")

    if args.esp_only:
        if rank == 0:
            print(json.dumps(esp_bench(K, synth, d)))
        return
    if args.triplet_only:
        if rank == 0:
            print(json.dumps(triplet_bench(K, synth, d, args.triplet_grid_n, args.triplet_steps, _peaks()[0])))
        return
    if args.serve_only:
        pool, _ = serving_pool(K, synth, args.serve_pool, args.serve_max_atoms)
        kw = dict(graph_points=args.serve_graph_points, scratch_gb=args.serve_scratch_gb, warmup_s=args.serve_warmup)
        res = {f: serve_bench(K, synth, int(prec), args.serve_seconds, args.serve_rate, pool, 21, **kw)
               for f, prec in (("mixed", K.Precision.Mixed), ("fp64", K.Precision.FP64))}
        if rank == 0:
            print(json.dumps({"serve_only": kw, **res}))
        return
    if args.only:
        # Small profiling case: warm-up and timed steps of one form only.
        for _ in range(args.warmup):
            step(args.only)
        t = timed(args.only, args.steps)
        if rank == 0:
            print(json.dumps({"only": args.only, "points": n, "ms_per_step": float(np.mean(t))}))
        return
    for _ in range(args.warmup):
        step("mixed")
        step("fp64")
    torch.cuda.synchronize()
    # FP64 reference output for the accuracy check of the mixed form.
    step("fp64")
    torch.cuda.synchronize()
    ref = out.clone()

    # Timed region: mixed form, with live kernel timing.
    clocks = ClockSampler(local)
    K.profile_reset()
    K.profile_enable(True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    t_mixed = timed("mixed", args.steps)
    clk = clocks.stop()
    prof = K.profile_read()
    K.profile_enable(False)
    ms_mixed = max_over_ranks(float(np.mean(t_mixed)))
    # Accuracy of the last mixed step against FP64, per field.
    acc = {}
    off = 0
    names = ["rho", "grad_rho", "lap_rho", "tau", "elf"]
    positive = [True, False, False, True, True]
    rho_ref = ref[:n].view(1, n)
    for p, name, pos in zip(props, names, positive):
        c = K.channels(p.kind)
        a, r = out[off:off + c * n].view(c, n), ref[off:off + c * n].view(c, n)
        acc[name] = field_errors(torch, a, r, rho_ref[0], pos)
        off += c * n

    if world > 1:
        dist.barrier()
    t_f64 = timed("fp64", args.steps)
    ms_f64 = max_over_ranks(float(np.mean(t_f64)))

    # End to end through the host C ABI (host outputs, D2H inside the timed region).
    # The caller's result arrays are page-locked host memory, reused across calls.
    e2e_eval = K.Evaluator(m, precision=K.Precision.Mixed)
    host_out = [torch.empty((K.channels(p.kind), n), dtype=torch.float64, pin_memory=True).numpy() for p in props]
    e2e_eval.evaluate_grid(grid, props, out=host_out)
    e2e_times = []
    for _ in range(0 if args.no_e2e else max(2, args.steps // 2)):
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        e2e_eval.evaluate_grid(grid, props, out=host_out)
        e2e_times.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(float(np.median(e2e_times)) if e2e_times else float("nan"))

    # The other workloads run at one GPU only (their own single-device
    # measurements): the serving loop first, before the potential and triplet
    # workloads leave GBs in the stream-ordered memory pool.
    serve = None
    if args.serve_seconds > 0 and world == 1:
        pool, sizes = serving_pool(K, synth, args.serve_pool, args.serve_max_atoms)
        kw = dict(graph_points=args.serve_graph_points, scratch_gb=args.serve_scratch_gb, warmup_s=args.serve_warmup)
        serve = {"config": {"arrivals": f"Poisson {args.serve_rate:g}/s for {args.serve_seconds:g} s (seeded)",
                            "pool": f"{len(pool)} synthetic molecules, atoms log-uniform in [3, {args.serve_max_atoms}]",
                            "admission": "HBM budget 150 GB (capped at 90% of free memory), 8 streams, "
                                         f"{args.serve_scratch_gb:g} GiB AO scratch per request",
                            "graphs": f"requests <= {args.serve_graph_points} points replay CUDA graphs "
                                      "from the second time their shape is met",
                            "warmup": (f"{args.serve_warmup:g} s of the same arrivals (other seed) through a "
                                       "server of their own before the measured window, not counted"
                                       if args.serve_warmup > 0 else
                                       "none (the server loads every kernel of the library when created)")},
                 "mixed": serve_bench(K, synth, int(K.Precision.Mixed), args.serve_seconds, args.serve_rate, pool,
                                      21, **kw),
                 "fp64": serve_bench(K, synth, int(K.Precision.FP64), args.serve_seconds, args.serve_rate, pool,
                                     21, **kw)}
    esp_line = None if (args.no_esp or world > 1) else esp_bench(K, synth, d)
    triplet = None if (args.no_triplet or world > 1) else triplet_bench(K, synth, d, args.triplet_grid_n,
                                                                          args.triplet_steps, _peaks()[0])

    if rank == 0:
        peaks, peak_kind = _peaks()
        # Dominant kernel of the mixed step.
        kern = max((k for k in prof if prof[k]["launches"]), key=lambda k: prof[k]["ms"])
        st = prof[kern]
        if kern.startswith("contract"):
            achieved = st["flops"] / (st["ms"] * 1e-3) / 1e12
            peak = peaks["bf16_tflops"]
            # DRAM bytes per launch: the ncu capture of contract_bulk_kernel on the
            # 48^3 case read and wrote 1.198 GB for the 437,070 AO rows the AO
            # kernel wrote (2,741 B per row); scaled by the rows written per launch.
            ao = prof.get("ao_build", {})
            rows_per_launch = ao["kept_rows"] / ao["launches"] if ao.get("launches") else 0.0
            roof = {"bound": "tensor", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": 2741.0 * rows_per_launch,
                    "traffic_source": "ncu dram__bytes_read+write of contract_bulk_kernel, 48^3 capture, "
                                      "per AO row written, scaled to this launch's rows",
                    "peak_source": f"{peak_kind} bf16_tflops (burst)",
                    "algorithmic": "2 * 128 points * 5 panels * 76 MOs per AO row of a block",
                    "issued_tflops": 6 * achieved,
                    "issued": "6 BF16 products per FP32 product (three-piece split of both operands)"}
        else:
            bytes_ = st["kept_rows"] * 5 * 128 * 4
            achieved = bytes_ / (st["ms"] * 1e-3) / 1e9
            peak = peaks["hbm_gbs"]
            roof = {"bound": "hbm", "kernel": kern, "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": None, "peak_source": f"{peak_kind} hbm_gbs",
                    "algorithmic": "kept AO rows * 5 panels * 128 points * 4 B written"}
        total_ms = sum(v["ms"] for v in prof.values())
        kernels = {k: {"launches": v["launches"], "ms": round(v["ms"], 3),
                       "share": round(v["ms"] / total_ms, 4) if total_ms else 0.0} for k, v in prof.items()
                   if v["launches"]}
        launches = sum(v["launches"] for v in prof.values())
        launches += 2 * prof["ao_build"]["launches"]  # kept-row counters of the profiler
        value = n_total / (ms_mixed * 1e-3)
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "grid pts/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_mixed,
            "higher_is_better": True,
            "scaling": "strong",
            "vs_baseline": None,
            "dtype": "mixed: f32 AO values and split-bf16 tensor-core products (f32 accumulation), "
                     "f64 exact rows, reductions and fields",
            "data": "synthetic (seeded FCHK)",
            "config": {"workload": "organic_740 (C12N4O4H20, 740 AOs, 76 occ MOs) rho/grad/lap/tau/ELF on 128^3 @0.2 bohr",
                       "points": n_total, "points_rank0": n, "backend": "AO_MO", "block": 128,
                       "threshold": 1e-12, "exact_rows": int(os.environ.get("KUMO_MIXED_EXACT_ROWS", "38")),
                       "l2": "256 MB buffer written between timed steps (untimed); AO scratch > L2",
                       "parallelism": f"slabs of whole planes x{world} (one grid, strong)"},
            "fp64": {"value": n_total / (ms_f64 * 1e-3), "ms_per_step": ms_f64},
            "mixed_over_fp64": ms_f64 / ms_mixed,
            "mixed_vs_fp64_error": acc,
            "e2e": {"value": n_total / e2e_s, "unit": "grid pts/s", "h2d_bytes_per_step": 108,
                    "d2h_bytes_per_step": nchan * n_total * 8},
            "roofline": roof,
            "kernels": kernels,
            "tile_tuning": K.tile_tuning_report().strip().splitlines(),
            "gpu_launches": launches,
            "clocks": clk,
        }
        if serve is not None:
            line["serve"] = serve
        if esp_line is not None:
            line["esp"] = esp_line
        if triplet is not None:
            line["triplet"] = triplet
        if not args.no_cpu_baseline:
            whole = K.Grid(origin, steps, counts)
            line["cpu_baseline"] = cpu_baseline(fchk, whole, args.cpu_blocks)
            line["cpu_baseline_1_thread"] = cpu_baseline(fchk, whole, max(16, args.cpu_blocks // 32), threads=1)
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
