#!/usr/bin/env python
"""Benchmark of the B200 exact-diagonalisation engine (one JSON line on rank 0).

Default workload (one GPU): Lanczos solves of the spin-1/2 J1-J2 chain, L=28
periodic, Sz=0 (D = 40,116,600), J1 = 1, J2 drawn uniformly from [0, 0.5]
(numpy default_rng seed 2802, one value per solve), lowest 2 eigenvalues, plain
FP64 (the drop-in path).  A step is one complete solve (ietl convergence rule,
100 eps).  Inputs (basis tables, couplings) are resident on the device before
the timed region; every vector is 321 MB, larger than the 126 MB L2, so no L2
flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun (N > 1) every rank solves its own stream of inputs (replicas,
weak scaling, no collective on the data path); value = all solves / max time.

`--impl reference` times the CPU restatement of the reference's algorithm
(explicit matrix built in hamiltonian_matrix's element order, row sums, ietl
vector passes) on a bounded sample of rows of the same workload with all host
threads, scaled to one solve.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from math import comb

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Lanczos solves/s (J1-J2 chain L=28, Sz=0, FP64, lowest 2 eigenvalues)"
UNIT = "solves/s"
L28 = 28
SEED_J2 = 2802
NEV = 2

# Lanczos iteration counts of the FP64 solves of the first inputs of the seed-2802
# J2 stream, as measured by this bench's own arm on B200.  The iteration count is
# a property of the input and the algorithm (the CPU restatement runs the same
# recurrence), so the reference arm, which cannot afford a full L=28 solve on the
# CPU, scales its per-iteration sample by these counts.
FP64_ITERATIONS_FALLBACK = 180  # mean of the first five inputs: 190, 142, 180, 182, 208

# DRAM bytes (read + write) of one launch of the FP64 apply on this workload,
# per apply variant, from ncu (dram__bytes_read.sum + dram__bytes_write.sum),
# summarised in profiles/hvb_kernel_l28_fp64.md; null for a variant not captured.
HV_TRAFFIC_L28_FP64 = {"blk1r4b4": 2.243246e9}


def j2_stream(n):
    return np.random.default_rng(SEED_J2).uniform(0.0, 0.5, n)


def chain_bonds(L, j2):
    """nnn chain lattice bonds in ALPS order: per cell (i,i+1) type 0, then (i,i+2) type 1."""
    out = []
    for i in range(L):
        out.append((i, (i + 1) % L, 1.0, 1.0, 0.0))
        out.append((i, (i + 2) % L, float(j2), float(j2), 0.0))
    return out


def table_upload_bytes(N, n_up, bonds):
    """Host->device bytes of the sector and coupling tables that aed_create copies: thi, tlo,
    lolist, looff, tiles (h, r), bundle block list, first tile per hi block, crossing-flip table,
    lo-neighbour table, per-step scalars."""
    nlo = (N + 1) // 2
    nhi = N - nlo
    pc = [bin(v).count("1") for v in range(1 << nlo)]
    cnt = [comb(nlo, k) for k in range(nlo + 1)]
    ks = [k for k in range(nlo + 1) if 0 <= n_up - k <= nhi]
    n_tiles = sum(comb(nhi, n_up - k) * -(-cnt[k] // 2048) for k in ks)
    n_blk = sum(-(-comb(nhi, n_up - k) // 4) * 4 for k in ks)
    lo_pairs = set()
    for b in bonds:
        s, t = sorted((b[0], b[1]))
        if s >= nhi and b[3] != 0.0:
            lo_pairs.add((N - 1 - s, N - 1 - t))
    masks = [(1 << i) | (1 << j) for i, j in lo_pairs]
    width = max((sum(1 for m in masks if pc[l & m] == 1) for l in range(1 << nlo)), default=0)
    return ((1 << nhi) * 4 + 2 * (1 << nlo) * 2 + (nlo + 2) * 4 + n_tiles * 8 + n_blk * 4 + (1 << nhi) * 4
            + nlo * (1 << nlo) * 2 + width * (1 << nlo) * 4)


def pair_offdiag_mean(N, n_up, bonds):
    """Exact mean number of off-diagonal elements per row (distinct flip pairs)."""
    pairs = {(min(b[0], b[1]), max(b[0], b[1])) for b in bonds if b[3] != 0.0}
    D = comb(N, n_up)
    anti = 2 * comb(N - 2, n_up - 1)
    return len(pairs) * anti / D


def read_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.idx)], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.15)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    smax = float(f[2])
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
            os.unlink(self.path)
        except Exception:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def barrier(pg):
    import torch

    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()


def _reduce(pg, v, op):
    if pg is None:
        return v
    import torch

    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(pg, v):
    return _reduce(pg, v, None if pg is None else pg.ReduceOp.MAX)


def sum_over_ranks(pg, v):
    return _reduce(pg, v, None if pg is None else pg.ReduceOp.SUM)


def rank_inputs(n_per_rank, world, rank):
    """This rank's J2 values: the seed-2802 stream dealt round robin over the ranks
    (replicas: every rank solves its own inputs, no data-path collective)."""
    return j2_stream(n_per_rank * world)[rank::world]


def cpu_sample(j2, iterations, threads_note="1 thread (the reference path is single-threaded)", rows=400_000):
    """Reference-algorithm restatement timed on a bounded sample of rows, scaled to one solve."""
    import oracle

    N, n_up = L28, L28 // 2
    states = oracle.basis_fast(N, n_up)
    D = states.size
    bonds = chain_bonds(L28, j2)
    r0 = D // 3
    tb, tp, tv = oracle.sample_times(N, states, bonds, r0, r0 + rows)
    scale = D / rows
    solve_s = tb * scale + iterations * (tp + tv) * scale
    return {
        "value": 1.0 / solve_s,
        "unit": UNIT,
        "cores": 1,
        "kind": "port",
        "sample": (f"rows [{r0}, {r0 + rows}) of the L=28 sector ({rows / D:.2%}): explicit-matrix row build "
                   f"({tb:.2f} s), row sums ({tp * 1e3:.1f} ms), make_step vector passes ({tv * 1e3:.1f} ms), "
                   f"scaled by D/rows, build once + {iterations} iterations; {threads_note}"),
    }


def cpu_matfree_sample(j2, iterations, rows=4_000_000):
    """Best-CPU baseline: the matrix-free restatement (no stored matrix, binary-search ranks) with
    all host threads, timed on a bounded sample of rows and scaled to one solve."""
    import oracle

    N, n_up = L28, L28 // 2
    states = oracle.basis_fast(N, n_up)
    D = states.size
    bonds = chain_bonds(L28, j2)
    x = np.random.default_rng(5).uniform(0, 1, D)
    r0 = D // 3
    oracle.hv_matfree(N, states, bonds, x, r0, r0 + rows // 8)  # warm the threads and pages
    t0 = time.perf_counter()
    oracle.hv_matfree(N, states, bonds, x, r0, r0 + rows)
    t = time.perf_counter() - t0
    solve_s = iterations * t * D / rows
    return {"value": 1.0 / solve_s, "unit": UNIT, "cores": oracle.num_threads(), "kind": "port",
            "sample": (f"matrix-free H*x (OpenMP, {oracle.num_threads()} threads) on rows [{r0}, {r0 + rows}) "
                       f"({rows / D:.1%} of the sector) in {t:.2f} s, scaled to {iterations} applies per solve; "
                       "vector passes not counted")}


def seeded_start(seed, n):
    """The engine's seeded start vector (`solve(seed=s)`: splitmix64 of the seed and the index, its top
    53 bits as a uniform double in [0, 1)) built on the host, so that the end-to-end leg starts from the
    vector the device-timed leg starts from and does the same iterations."""
    out = np.empty(n, np.float64)
    chunk = 1 << 22
    with np.errstate(over="ignore"):
        for a in range(0, n, chunk):
            i = np.arange(a, min(n, a + chunk), dtype=np.uint64)
            z = np.uint64(seed) + np.uint64(0x9E3779B97F4A7C15) * (i + np.uint64(1))
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            z ^= z >> np.uint64(31)
            out[a:a + i.size] = (z >> np.uint64(11)).astype(np.float64) * 2.0 ** -53
    return out


def compare_energies(got, ref):
    """Relative differences of eigenvalue lists against a reference run (lists of per-solve lists).
    gs: ground states only (the 1e-9 criterion).  An excited value of `got` below the reference's by
    more than 1e-9 relative is a state the reference run missed (a Ritz value cannot lie below the
    eigenvalue of its index): such solves are counted, not mixed into the maximum."""
    gs = max(abs(a[0] - b[0]) / abs(b[0]) for a, b in zip(got, ref))
    allv, missed = 0.0, 0
    for a, b in zip(got, ref):
        if any(x < y - 1e-9 * abs(y) for x, y in zip(a[1:], b[1:])):
            missed += 1
            continue
        allv = max([allv] + [abs(x - y) / abs(y) for x, y in zip(a, b)])
    return {"gs": gs, "all": allv, "ref_missed_states": missed}


def run_ours(args):
    import torch

    import alps_b200 as ed

    world, rank, local, pg = dist_setup(args)
    torch.cuda.set_device(local)
    K, W = args.steps, args.warmup
    N, n_up = L28, L28 // 2
    j2s = rank_inputs(W + K, world, rank)
    # the sector tables are resident before the timed region; each step sets
    # that step's couplings (coupling tables + diagonal, ~ms) and solves
    ham = ed.Hamiltonian(N, n_up, chain_bonds(L28, j2s[0]), precision=ed.FP64, device=local)
    D = ham.dim
    for j2 in j2s[:W]:
        ham.set_couplings(chain_bonds(L28, j2))
        ham.solve(nev=NEV, seed=1)
    stream = torch.cuda.ExternalStream(ham.stream())
    launches0 = ed.launch_count()
    clocks = ClockSampler(local)
    iters, apply_ms, evals = [], [], []
    with clocks:
        barrier(pg)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        t0 = time.perf_counter()
        for j2 in j2s[W:]:
            ham.set_couplings(chain_bonds(L28, j2))
            r = ham.solve(nev=NEV, seed=1, profile=True)
            iters.append(r["iterations"])
            apply_ms.append(r["apply_ms"])
            evals.append(r["evals"].tolist())
        e1.record(stream)
        e1.synchronize()
        wall = time.perf_counter() - t0
        barrier(pg)
    dev_s = e0.elapsed_time(e1) / 1e3
    launches = ed.launch_count() - launches0
    t_max = max_over_ranks(pg, dev_s)
    total = sum_over_ranks(pg, float(K))
    value = total / t_max
    # roofline of the dominant kernel (the apply)
    nbar = pair_offdiag_mean(N, n_up, chain_bonds(L28, 0.25))
    b_apply = D * ((1 + nbar) * 8 + 8)
    t_apply = float(np.mean(apply_ms)) / 1e3
    peak, peak_kind = read_peaks()
    achieved = b_apply / t_apply / 1e9
    xv, yv = ham.new_vector(), ham.new_vector()  # the tuned apply variant (no launch: already tuned)
    ham.fill_random(xv, 1)
    _, vused = ham.time_apply(xv, yv, 1)
    xv.free()
    yv.free()
    vname = ed.apply_variants()[vused]
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "peak_kind": peak_kind, "kernel": f"apply variant {vname} (FP64)", "apply_ms": t_apply * 1e3,
            "algorithmic_bytes_per_apply": b_apply, "traffic": HV_TRAFFIC_L28_FP64.get(vname),
            "traffic_source": "profiles/hvb_kernel_l28_fp64.md (ncu dram__bytes_read.sum + dram__bytes_write.sum, "
                              "one launch)"}
    print(f"[bench] fp64: {value:.3f} solves/s, iterations {iters}, apply {t_apply*1e3:.3f} ms "
          f"({achieved:.0f} GB/s)", file=sys.stderr)
    # end-to-end through the public API with host buffers, every step:
    # aed_create (tables H2D) + aed_solve from a pinned host start vector (H2D)
    # + eigenvalues and the alpha/beta stream (D2H) + aed_destroy
    start = torch.empty(D, dtype=torch.float64, pin_memory=True)
    start.numpy()[:] = seeded_start(1, D)  # the timed solves' start (seed 1), here from host memory
    h2d = d2h = 0
    barrier(pg)
    t0 = time.perf_counter()
    for j2 in j2s[W:]:
        bonds = chain_bonds(L28, j2)
        h = ed.Hamiltonian(N, n_up, bonds, precision=ed.FP64, device=local)
        r = h.solve(nev=NEV, start=start.numpy())
        h.close()
        h2d += D * 8 + table_upload_bytes(N, n_up, bonds) + 16
        d2h += 16 * (r["iterations"] + 1) + 32 * NEV
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(pg, time.perf_counter() - t0)
    e2e = {"value": total / e2e_s, "unit": UNIT, "h2d_bytes_per_step": h2d // K, "d2h_bytes_per_step": d2h // K,
           "path": "aed_create + aed_solve(pinned host start vector) + aed_destroy, wall clock"}
    # mixed precision on the same inputs: FP32 Lanczos basis + FP64 refinement
    mixed = None
    if not args.no_mixed:
        h32 = ed.Hamiltonian(N, n_up, chain_bonds(L28, j2s[0]), precision=ed.FP32, device=local)
        # warm-up: the FP32 basis store sized once for 256 vectors (40 GB; the FP32 phases here take 88-214
        # steps), as a long-running caller keeps it, so that no timed solve waits on a device allocation
        h32.reserve_basis(256)
        h32.solve(nev=NEV, seed=1)
        barrier(pg)
        s32 = torch.cuda.ExternalStream(h32.stream())
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        mev, mit, m32ms = [], [], []
        m0.record(s32)
        for j2 in j2s[W:]:
            h32.set_couplings(chain_bonds(L28, j2))
            r = h32.solve(nev=NEV, seed=1, profile=True)
            mev.append(r["evals"].tolist())
            mit.append((r["iterations_low"], r["iterations"]))
            m32ms.append(r["apply_ms"])
        m1.record(s32)
        m1.synchronize()
        mixed_s = max_over_ranks(pg, m0.elapsed_time(m1) / 1e3)
        rel = compare_energies(mev, evals)
        b32 = D * ((1 + nbar) * 4 + 4)
        mixed = {"solves_per_s": total / mixed_s, "speedup_vs_fp64": (total / mixed_s) / value,
                 "rel_energy_err_vs_fp64": rel, "iterations_fp32_fp64": mit,
                 "apply_ms_fp32": float(np.mean(m32ms)),
                 "hv_fp32_gbs": b32 / (float(np.mean(m32ms)) / 1e3) / 1e9}
        h32.close()
        print(f"[bench] mixed: {mixed}", file=sys.stderr)
    cpu = cpu_all = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_sample(float(j2s[W]), int(round(np.mean(iters))))
        cpu_all = cpu_matfree_sample(float(j2s[W]), int(round(np.mean(iters))))
    ham.close()
    # the other configurations, on one GPU only (their own sections, not part of `value`)
    others = None
    if rank == 0 and world == 1 and not args.no_configs:
        others = {"cfg1_chain16": chain16_result(ed), "cfg3_square6x5": square_result(ed),
                  "cfg4_batch512": batch_result(ed, args.steps_per_launch, with_cpu=not args.no_cpu)}
        print(f"[bench] configs: {json.dumps(others)[:2000]}", file=sys.stderr)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": t_max / K * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "J1-J2 chain L=28 periodic, Sz=0, D=40116600, J1=1, J2~U[0,0.5] seed 2802, "
                                   "lowest 2 eigenvalues, FP64 Lanczos (ietl rule 100 eps)",
                       "dimension": D, "nev": NEV, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (each vector 321 MB); no flush"},
            "iterations": iters, "evals": evals, "wall_s": wall,
            "roofline": roof, "cpu_baseline": cpu, "cpu_baseline_all_cores": cpu_all, "e2e": e2e, "gpu_launches": launches,
            "clocks": clocks.summary(), "mixed": mixed, "configs": others,
        }
        print(json.dumps(line))
    if pg is not None:
        pg.destroy_process_group()


def ladder_bonds(L, jl, jr):
    """ladder lattice (anisotropic2d cell, periodic legs, open rungs) in ALPS order; site = 2x + y."""
    out = []
    for x in range(L):
        for y in range(2):
            s = 2 * x + y
            out.append((s, 2 * ((x + 1) % L) + y, float(jl), float(jl), 0.0))
            if y == 0:
                out.append((s, s + 1, float(jr), float(jr), 0.0))
    return out


def square_bonds(Lx, Wy, seed):
    """square lattice (simple2d cell, periodic) in ALPS order, per-bond J ~ U[0.8, 1.2]."""
    raw = []
    for x in range(Lx):
        for y in range(Wy):
            s = x * Wy + y
            raw.append((s, x * Wy + (y + 1) % Wy))
            raw.append((s, ((x + 1) % Lx) * Wy + y))
    js = np.random.default_rng(seed).uniform(0.8, 1.2, len(raw))
    return [(a, b, float(j), float(j), 0.0) for (a, b), j in zip(raw, js)]


def batch_requests():
    """Config 4: 512 J1-J2 chains, L uniform over {12,...,22} even, J2 ~ U[0,1], seed 5124, 2 eigenvalues."""
    rng = np.random.default_rng(5124)
    Ls = rng.choice([12, 14, 16, 18, 20, 22], size=512)
    j2 = rng.uniform(0.0, 1.0, size=512)
    return [(int(L), chain_bonds(int(L), j), 2, k) for k, (L, j) in enumerate(zip(Ls, j2))]


def serve_requests(n):
    """Config 5: Poisson arrivals at 200/s (seed 2000); chain L in {14..26} even or ladder 2x{7..12},
    J_leg, J_rung ~ U[0.5, 1.5], k ~ U{1..4}."""
    rng = np.random.default_rng(2000)
    arr = np.cumsum(rng.exponential(1.0 / 200.0, n))
    out = []
    for k in range(n):
        jl, jr = rng.uniform(0.5, 1.5, 2)
        nev = int(rng.integers(1, 5))
        if rng.random() < 0.5:
            L = int(rng.choice(np.arange(14, 27, 2)))
            out.append((float(arr[k]), L, chain_bonds_jl(L, jl), nev, k))
        else:
            L = int(rng.integers(7, 13))
            out.append((float(arr[k]), 2 * L, ladder_bonds(L, jl, jr), nev, k))
    return out


def chain_bonds_jl(L, jl):
    return [(i, (i + 1) % L, float(jl), float(jl), 0.0) for i in range(L)]


def cpu_solve_estimate(N, bonds, nev, iterations, rows=200_000):
    """Seconds of the reference-algorithm restatement for one solve on one core: a full
    oracle solve when the sector is small, else a bounded row sample scaled to the sector."""
    import oracle

    D = comb(N, N // 2)
    if D <= 60000:
        t0 = time.perf_counter()
        M = oracle.Matrix(N, N // 2, bonds)
        M.lanczos(nev=nev, seed=1)
        return time.perf_counter() - t0, "full"
    states = oracle.basis_fast(N, N // 2)
    r = min(rows, D)
    tb, tp, tv = oracle.sample_times(N, states, bonds, 0, r)
    return (tb + iterations * (tp + tv)) * D / r, f"sample {r} rows"


def square_result(ed, solves=1):
    """Config 3: 6x5 square lattice, per-bond J ~ U[0.8,1.2] (seed 3005), lowest eigenvalue: FP64 and mixed
    solves (the apply variant tuned and the FP32 store grown by an untimed solve first), with the applies'
    achieved bandwidth by algorithmic bytes."""
    bonds = square_bonds(6, 5, 3005)
    out = {}
    for name, prec in (("fp64", ed.FP64), ("mixed", ed.FP32)):
        ham = ed.Hamiltonian(30, 15, bonds, precision=prec)
        ham.solve(nev=1, seed=1)
        ts, rs = [], []
        for _ in range(solves):
            t0 = time.perf_counter()
            rs.append(ham.solve(nev=1, seed=1, profile=True))
            ts.append(time.perf_counter() - t0)
        r = rs[-1]
        out[name] = {"seconds": float(np.mean(ts)), "evals": r["evals"].tolist(), "iterations": r["iterations"],
                     "iterations_low": r["iterations_low"], "apply_ms": r["apply_ms"],
                     "refined_by": r.get("refined_by")}
        ham.close()
    D = 155117520
    nbar = 60 * 2 * comb(28, 14) / D
    peak, _ = read_peaks()
    g64 = D * ((1 + nbar) * 8 + 8) / (out["fp64"]["apply_ms"] / 1e3) / 1e9
    g32 = D * ((1 + nbar) * 4 + 4) / (out["mixed"]["apply_ms"] / 1e3) / 1e9
    rel = abs(out["mixed"]["evals"][0] - out["fp64"]["evals"][0]) / abs(out["fp64"]["evals"][0])
    return {"workload": "square lattice 6x5 periodic, Sz=0, D=155117520, J_b~U[0.8,1.2] seed 3005, k=1",
            "fp64": out["fp64"], "mixed": out["mixed"],
            "fp64_solves_per_s": 1.0 / out["fp64"]["seconds"], "mixed_solves_per_s": 1.0 / out["mixed"]["seconds"],
            "speedup_mixed_vs_fp64": out["fp64"]["seconds"] / out["mixed"]["seconds"],
            "rel_energy_err_mixed_vs_fp64": rel,
            "hv_gbs": {"fp64": g64, "fp32": g32, "peak": peak, "frac_fp64": g64 / peak, "frac_fp32": g32 / peak,
                       "bytes_per_row_fp64": (1 + nbar) * 8 + 8, "bytes_per_row_fp32": (1 + nbar) * 4 + 4}}


def run_square(args):
    """Config 3 alone: one JSON line."""
    import alps_b200 as ed

    sq = square_result(ed, solves=max(1, args.steps))
    line = {"metric": "6x5 square lattice ground state: solves/s, mixed vs FP64", "value": sq["mixed_solves_per_s"],
            "unit": "solves/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": sq["workload"]}}
    line.update({k: v for k, v in sq.items() if k != "workload"})
    print(json.dumps(line))


def chain16_result(ed, reps=20):
    """Config 1: Heisenberg chain L=16 periodic, J=1, Sz=0 (D=12,870), lowest 4 eigenvalues, FP64: complete
    solves on the GPU (after one untimed solve) and the oracle's complete solve of the reference algorithm
    (explicit matrix in hamiltonian_matrix's element order, ietl Lanczos) on one host core."""
    import oracle

    bonds = [(i, (i + 1) % 16, 1.0, 1.0, 0.0) for i in range(16)]
    ham = ed.Hamiltonian(16, 8, bonds)
    ham.solve(nev=4, seed=1)
    t0 = time.perf_counter()
    for _ in range(reps):
        r = ham.solve(nev=4, seed=1)
    gpu_s = (time.perf_counter() - t0) / reps
    ham.close()
    t0 = time.perf_counter()
    M = oracle.Matrix(16, 8, bonds)
    o = M.lanczos(nev=4, seed=1)
    cpu_s = time.perf_counter() - t0
    return {"workload": "Heisenberg chain L=16 periodic, J=1, Sz=0, D=12870, lowest 4 eigenvalues, FP64",
            "gpu_solves_per_s": 1.0 / gpu_s, "gpu_iterations": r["iterations"], "evals": r["evals"].tolist(),
            "cpu_reference_port_solves_per_s": 1.0 / cpu_s, "cpu_iterations": o["iterations"],
            "cpu_cores": 1, "max_rel_diff_vs_cpu": float(np.max(np.abs(r["evals"] - o["evals"]) / np.abs(o["evals"]))),
            "speedup_gpu_vs_cpu": cpu_s / gpu_s}


def run_momentum(args):
    """Momentum sectors: every TOTAL_MOMENTUM of the Sz=0 sector of the J1-J2 chain L=28 (J2 = the first value
    of the seed-2802 stream), lowest 2 eigenvalues each, as the reference's default sparsediag path runs it
    (TRANSLATION_SYMMETRY on); the lowest value over the momenta against the plain Sz=0 FP64 solve."""
    import torch

    import alps_b200 as ed

    L = L28
    j2 = float(j2_stream(1)[0])
    bonds = chain_bonds(L, j2)
    params = {"MODEL": "spin", "LATTICE": "nnn chain lattice", "L": L, "CONSERVED_QUANTUMNUMBERS": "Sz"}
    ks = ed.lattice_momenta(params)
    trans = [ed.lattice_translations(params, k) for k in ks]
    h0 = ed.Hamiltonian(L, L // 2, bonds, translations=trans[0])  # warm-up: tables, allocator cache
    h0.solve(nev=NEV, seed=1)
    h0.close()
    sectors, apply_ms = [], []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k, tr in zip(ks, trans):
        ham = ed.Hamiltonian(L, L // 2, bonds, translations=tr)
        r = ham.solve(nev=NEV, seed=1, profile=True)
        sectors.append({"k": ed.momentum_label(k), "dim": ham.dim, "iterations": r["iterations"],
                        "evals": r["evals"].tolist()})
        apply_ms.append((ham.dim, r["apply_ms"]))
        ham.close()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    # the same scan with several sectors at once (own handle and stream each, host threads): the sectors
    # are independent, so every result must equal the one-by-one loop's.  At L=28 one sector's apply
    # already fills the GPU, so this pass is reported beside the one-by-one rate, not as the value
    from concurrent.futures import ThreadPoolExecutor

    def one(tr):
        ham = ed.Hamiltonian(L, L // 2, bonds, translations=tr)
        try:
            return ham.solve(nev=NEV, seed=1)["evals"].tolist()
        finally:
            ham.close()

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=args.sector_workers) as pool:
        conc = list(pool.map(one, trans))
    torch.cuda.synchronize()
    dt_conc = time.perf_counter() - t0
    same = all(c == s["evals"] for c, s in zip(conc, sectors))
    real = ed.Hamiltonian(L, L // 2, bonds)
    t1 = time.perf_counter()
    e0 = real.solve(nev=1, seed=1)["evals"][0]
    t_real = time.perf_counter() - t1
    real.close()
    lowest = min(s["evals"][0] for s in sectors)
    # apply roofline: per row x_i, y_i (16 B each), rep 4, norm_i 8, diag_i 8, and per flip the map entry (4),
    # n_j (8) and x_j (16); flips per row ~ the Sz sector's mean off-diagonal count
    nbar = pair_offdiag_mean(L, L // 2, bonds)
    dim0, ms0 = max(apply_ms)
    b_row = 52 + nbar * 28
    peak, peak_kind = read_peaks()
    ach = dim0 * b_row / (ms0 / 1e3) / 1e9
    line = {"metric": "momentum sectors solved per second (Sz=0, J1-J2 chain L=28, all 28 momenta, FP64, lowest 2 each)",
            "value": len(sectors) / dt, "unit": "sectors/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "c128", "data": "synthetic", "seconds_all_momenta": dt,
            "sectors_at_once": {"workers": args.sector_workers, "seconds_all_momenta": dt_conc,
                                "sectors_per_s": len(sectors) / dt_conc, "same_results_as_one_by_one": same},
            "config": {"workload": f"nnn chain L=28 periodic, J1=1, J2={j2:.6f} (seed 2802), Sz=0, TOTAL_MOMENTUM "
                                   "2 pi m / 28, m = 0..27, lowest 2 eigenvalues per sector"},
            "lowest_over_momenta": lowest, "sz0_fp64_ground_state": e0,
            "rel_diff": abs(lowest - e0) / abs(e0), "sz0_fp64_solve_s": t_real,
            "roofline": {"bound": "hbm", "kernel": "mom_hv_kernel", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "peak_kind": peak_kind, "apply_ms": ms0, "rows": dim0,
                         "algorithmic_bytes_per_row": b_row},
            "sectors": sectors}
    print(json.dumps(line))


def run_spin(args):
    """Spin-1 Heisenberg chain L=18, Sz=0 (44,152,809 states), FP64, lowest 2 eigenvalues, through the
    spin-S engine (local_S = 1); apply roofline from the sampled mean of off-diagonal terms per row."""
    import alps_b200 as ed

    L = 18
    bonds = [(i, (i + 1) % L, 1.0, 1.0, 0.0) for i in range(L)]
    ham = ed.Hamiltonian(L, L, bonds, two_s=2)
    x, y = ham.new_vector(), ham.new_vector()
    ham.fill_random(x, 1)
    ham.time_mult(x, y, 2)
    ms = ham.time_mult(x, y, 10)
    states = ham.basis(0, min(ham.dim, 200000))
    digits = np.array([(states >> np.uint64(2 * (L - 1 - i))) & np.uint64(3) for i in range(L)]).astype(int)
    a, c = digits, np.roll(digits, -1, axis=0)
    nbar = float(np.mean(np.sum((a < 2) & (c > 0), axis=0) + np.sum((a > 0) & (c < 2), axis=0)))
    b_row = 16 + nbar * 8  # x_i, y_i, and one gathered x_j per off-diagonal term
    peak, peak_kind = read_peaks()
    ach = ham.dim * b_row / (ms / 1e3) / 1e9
    t0 = time.perf_counter()
    r = ham.solve(nev=NEV, seed=1)
    dt = time.perf_counter() - t0
    line = {"metric": "spin-1 chain L=18 Sz=0 Lanczos solves/s (FP64, lowest 2)", "value": 1.0 / dt, "unit": "solves/s",
            "n_gpus": 1, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "spin-1 Heisenberg chain L=18 periodic, J=1, Sz_total=0, D=%d" % ham.dim},
            "iterations": r["iterations"], "evals": r["evals"].tolist(),
            "roofline": {"bound": "hbm", "kernel": "spin_hv_kernel", "achieved": ach, "peak": peak, "unit": "GB/s",
                         "frac": ach / peak, "peak_kind": peak_kind, "apply_ms": ms,
                         "algorithmic_bytes_per_row": b_row, "offdiag_per_row_sampled": nbar}}
    ham.close()
    print(json.dumps(line))


def batch_result(ed, steps_per_launch=8, with_cpu=True):
    """Config 4: 512 J1-J2 chains through the batched engine, mixed and FP64, and through the
    single-instance FP64 drop-in one after the other."""
    reqs = batch_requests()
    res = {}
    for name, prec in (("mixed", ed.FP32), ("fp64", ed.FP64)):
        srv = ed.Server(precision=prec, max_slots=512, steps=steps_per_launch, reserve=-1)  # pool mapped up front
        w = [srv.submit(n, n // 2, b, nev=nev, seed=sd) for n, b, nev, sd in reqs[:8]]  # warm-up
        srv.run(w)
        t0 = time.perf_counter()
        tickets = [srv.submit(n, n // 2, b, nev=nev, seed=sd) for n, b, nev, sd in reqs]
        out = srv.run(tickets)
        dt = time.perf_counter() - t0
        st = srv.stats()
        srv.close()
        res[name] = {"seconds": dt, "solves_per_s": len(reqs) / dt, "graph_launches": st["graph_launches"],
                     "evals": [out[t]["evals"].tolist() for t in tickets],
                     "converged": all(out[t]["converged"] for t in tickets)}
    # the drop-in single-instance FP64 path, instance after instance
    t0 = time.perf_counter()
    single = []
    hams = {}
    for n, b, nev, sd in reqs:
        h = hams.get(n)
        if h is None:
            h = hams[n] = ed.Hamiltonian(n, n // 2, b, precision=ed.FP64)
        else:
            h.set_couplings(b)
        single.append(h.solve(nev=nev, seed=sd)["evals"].tolist())
    t_single = time.perf_counter() - t0
    for h in hams.values():
        h.close()
    rel = compare_energies(res["mixed"]["evals"], single)
    rel64 = compare_energies(res["fp64"]["evals"], single)
    out = {"workload": "512 J1-J2 chains, L~U{12..22} even, J2~U[0,1] seed 5124, Sz=0, k=2",
           "steps_per_graph": steps_per_launch,
           "mixed_batched": {k: v for k, v in res["mixed"].items() if k != "evals"},
           "fp64_batched": {k: v for k, v in res["fp64"].items() if k != "evals"},
           "fp64_single_instance": {"seconds": t_single, "solves_per_s": len(reqs) / t_single},
           "speedup_mixed_batched_vs_fp64_single": res["mixed"]["solves_per_s"] / (len(reqs) / t_single),
           "speedup_mixed_batched_vs_fp64_batched": res["mixed"]["solves_per_s"] / res["fp64"]["solves_per_s"],
           "rel_energy_err_mixed_vs_fp64_single": rel, "rel_energy_err_fp64_batched_vs_single": rel64}
    if with_cpu:
        classes, counts = {}, {}
        for n, b, nev, sd in reqs:
            classes.setdefault(n, (b, nev))
            counts[n] = counts.get(n, 0) + 1
        tot, notes = 0.0, {}
        for n, (b, nev) in sorted(classes.items()):
            t, how = cpu_solve_estimate(n, b, nev, 120)
            tot += t * counts[n]
            notes[n] = f"{t:.3g} s ({how})"
        out["cpu_baseline"] = {"value": len(reqs) / tot, "unit": "solves/s", "cores": 1, "kind": "port",
                               "sample": "one instance per chain length, explicit-matrix Lanczos on one core "
                                         "(row sample x 120 iterations above 60000 states): " + json.dumps(notes)}
    return out


def run_batch(args):
    """Config 4 alone: one JSON line."""
    import alps_b200 as ed

    b = batch_result(ed, args.steps_per_launch, with_cpu=not args.no_cpu)
    line = {"metric": "batched Lanczos solves/s (512 J1-J2 chains, L 12..22), mixed vs plain FP64",
            "value": b["mixed_batched"]["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": b["workload"], "steps_per_graph": b["steps_per_graph"]}}
    line.update({k: v for k, v in b.items() if k not in ("workload", "steps_per_graph")})
    print(json.dumps(line))


def run_serve(args):
    """Config 5: Poisson stream of requests at 200/s through the served engine; latency from the
    scheduled arrival to the harvest of the result."""
    import alps_b200 as ed

    # the seed-2000 stream; --rate rescales its arrival times (the same requests at another offered rate)
    reqs = [(arr * 200.0 / args.rate,) + tuple(r) for arr, *r in serve_requests(args.requests)]
    prec = ed.FP32 if args.precision == "mixed" else ed.FP64
    srv = ed.Server(precision=prec, max_slots=512, steps=args.steps_per_launch, reserve=-1,  # pool mapped up front
                    max_lanes=args.lanes, lane_min_dim=args.lane_min_dim if args.lanes > 0 else -1)
    w = [srv.submit(n, n // 2, b, nev=nev, seed=sd) for _, n, b, nev, sd in reqs[:16]]
    srv.run(w)
    pending = {}
    lat = []
    large = []  # whether each finished request was one for a single-instance lane
    work = {p: {"iterations_low": 0, "iterations": 0, "refined_by": {}} for p in ("lanes", "batch")}
    min_dim = args.lane_min_dim if args.lanes > 0 else None
    i = 0
    t0 = time.perf_counter()
    while i < len(reqs) or pending:
        now = time.perf_counter() - t0
        while i < len(reqs) and reqs[i][0] <= now:
            arr, n, b, nev, sd = reqs[i]
            pending[srv.submit(n, n // 2, b, nev=nev, seed=sd)] = (arr, comb(n, n // 2))
            i += 1
        if pending:
            srv.step()
            done_t = time.perf_counter() - t0
            for t in list(pending):
                r = srv.poll(t)
                if r is not None:
                    arr, dim = pending.pop(t)
                    lat.append(done_t - arr)
                    big = min_dim is not None and dim >= min_dim
                    large.append(big)
                    w = work["lanes" if big else "batch"]
                    w["iterations_low"] += r["iterations_low"]
                    w["iterations"] += r["iterations"]
                    w["refined_by"][r["refined_by"]] = w["refined_by"].get(r["refined_by"], 0) + 1
        elif i < len(reqs):
            time.sleep(max(0.0, min(0.002, reqs[i][0] - (time.perf_counter() - t0))))
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    lat = np.array(lat)
    large = np.array(large, dtype=bool)

    def pct(a):
        return {"n": int(a.size), "p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99))} if a.size \
            else {"n": 0}

    line = {"metric": f"served Lanczos: solves/s and latency (Poisson {args.rate:g} req/s)", "value": len(reqs) / wall,
            "unit": "solves/s", "n_gpus": 1, "higher_is_better": True, "dtype": "f32+f64" if prec == ed.FP32 else "f64",
            "data": "synthetic",
            "config": {"workload": f"{len(reqs)} requests, Poisson {args.rate:g}/s seed 2000, chain L 14..26 or "
                                   "ladder 2x7..2x12, "
                                   "J_leg,J_rung~U[0.5,1.5], k~U{1..4}", "precision": args.precision,
                       "steps_per_graph": args.steps_per_launch,
                       "lanes": {"max": args.lanes, "min_dim": args.lane_min_dim if args.lanes > 0 else None}},
            "latency_s": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                          "mean": float(lat.mean()), "max": float(lat.max())},
            "latency_s_by_path": {"lanes": pct(lat[large]), "batch": pct(lat[~large])},
            "work_by_path": work,
            "offered_rate": args.rate, "graph_launches": st["graph_launches"], "wall_s": wall}
    print(json.dumps(line))


def reference_complete_solves():
    """Complete solves of the reference algorithm's restatement (explicit matrix in hamiltonian_matrix's
    element order, ietl Lanczos and T-matrix rules) on one host core, the reference path being single-threaded:
    config 1 (Heisenberg chain L=16, lowest 4) and one chain of each config-4 length up to L=20 (the first
    of the seed-5124 requests with that length, lowest 2)."""
    import oracle

    out = {}
    cases = [("cfg1_chain16_k4", 16, [(i, (i + 1) % 16, 1.0, 1.0, 0.0) for i in range(16)], 4)]
    seen = set()
    for n, b, nev, _ in batch_requests():
        if n <= 20 and n not in seen:
            seen.add(n)
            cases.append((f"cfg4_chain{n}_k{nev}", n, b, nev))
    for name, n, b, nev in sorted(cases, key=lambda c: c[1]):
        t0 = time.perf_counter()
        M = oracle.Matrix(n, n // 2, b)
        o = M.lanczos(nev=nev, seed=1)
        dt = time.perf_counter() - t0
        out[name] = {"dimension": int(M.D), "seconds": dt, "solves_per_s": 1.0 / dt, "iterations": o["iterations"],
                     "evals": o["evals"].tolist()}
    return out


def run_reference(args):
    """The reference's algorithm on the host cores (the oracle port: the reference itself needs Boost and
    LAPACK, absent here) for the default workload.  A complete L=28 solve of the reference algorithm does not
    fit the run (its explicit matrix alone is ~75 GB of map nodes), so each step is a bounded sample: the
    explicit-matrix build, the row sums and the make_step vector passes over a block of rows with all host
    threads, scaled by D / rows to the sector and by the iteration count of the FP64 solve to one solve.
    Complete solves of configs 1 and 4 ride along in their own section."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle

    K, W = args.steps, args.warmup
    j2s = j2_stream(W + K)
    threads = oracle.num_threads()
    N, n_up = L28, L28 // 2
    states = oracle.basis_fast(N, n_up)
    D = states.size
    rows = min(D // 4, 120_000 * threads)
    r0 = D // 3
    vals, walls, parts = [], [], None
    for k, j2 in enumerate(j2s):
        t0 = time.perf_counter()
        tb, tp, tv = oracle.sample_times_mt(N, states, chain_bonds(L28, float(j2)), r0, r0 + rows)
        wall = time.perf_counter() - t0
        scale = D / rows
        solve_s = tb * scale + FP64_ITERATIONS_FALLBACK * (tp + tv) * scale
        if k >= W:
            vals.append(1.0 / solve_s)
            walls.append(wall)
            parts = (tb, tp, tv)
    v = float(np.mean(vals))
    sample = (f"rows [{r0}, {r0 + rows}) of the L=28 sector ({rows / D:.2%}) per step on {threads} threads: "
              f"explicit-matrix row build ({parts[0]:.2f} s), row sums ({parts[1] * 1e3:.1f} ms), make_step vector "
              f"passes ({parts[2] * 1e3:.1f} ms), scaled by D/rows = {D / rows:.1f} and build once + "
              f"{FP64_ITERATIONS_FALLBACK} iterations (the mean FP64 iteration count of these inputs)")
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": float(np.mean(walls)) * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": "J1-J2 chain L=28 periodic, Sz=0, D=40116600, J1=1, J2~U[0,0.5] seed 2802, "
                                   "lowest 2 eigenvalues, FP64 Lanczos (ietl rule 100 eps)"},
            "value_from": "extrapolated: a step is a bounded row sample (ms_per_step is its wall time); value is "
                          "that sample scaled to one complete solve",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "complete_solves": reference_complete_solves()}
    print(json.dumps(line))


def apply_case_bonds(name):
    """Workloads of `--workload apply`: l24 / l26 / l28 (J1-J2 chain, J2 = 0.25), sq6x5 (6x5 square lattice,
    per-bond J ~ U[0.8, 1.2] seed 3005)."""
    if name in ("l24", "l26", "l28"):
        L = int(name[1:])
        return L, L // 2, chain_bonds(L, 0.25)
    if name == "sq6x5":
        return 30, 15, square_bonds(6, 5, 3005)
    raise SystemExit(f"unknown apply case {name!r}")


def run_apply(args):
    """A few applies y = H x of one workload, timed with CUDA events (the commands the ncu summaries under
    profiles/ use; plain text, not a bench line).  --case spin1_l18: spin-1 Heisenberg chain L=18, Sz=0;
    --case mom_l28: J1-J2 chain L=28 (J2 = 0.25), Sz=0, momentum index --k; --case spin1mom_l18: the
    spin-1 chain's Sz=0 momentum sector of index --k."""
    import alps_b200 as ed
    if args.case == "spin1_l18":
        L = 18
        ham = ed.Hamiltonian(L, L, [(i, (i + 1) % L, 1.0, 1.0, 0.0) for i in range(L)], two_s=2)
    elif args.case == "spin1mom_l18":
        L = 18
        params = {"MODEL": "spin", "LATTICE": "chain lattice", "L": L}
        k = ed.lattice_momenta(params)[args.k]
        ham = ed.Hamiltonian(L, L, [(i, (i + 1) % L, 1.0, 1.0, 0.0) for i in range(L)], two_s=2,
                             translations=ed.lattice_translations(params, k))
    elif args.case == "mom_l28":
        params = {"MODEL": "spin", "LATTICE": "nnn chain lattice", "L": 28}
        k = ed.lattice_momenta(params)[args.k]
        ham = ed.Hamiltonian(28, 14, chain_bonds(28, 0.25), translations=ed.lattice_translations(params, k))
    else:
        N, n_up, bonds = apply_case_bonds(args.case)
        ham = ed.Hamiltonian(N, n_up, bonds, precision=ed.FP64 if args.apply_precision == "fp64" else ed.FP32)
    x, y = ham.new_vector(), ham.new_vector()
    ham.fill_random(x, 1)
    if args.case in ("spin1_l18", "mom_l28", "spin1mom_l18"):
        ham.time_mult(x, y, 1)
        print(f"{args.case} rows={ham.dim} apply_ms={ham.time_mult(x, y, args.reps):.4f}")
        return
    names = ed.apply_variants()
    if args.sweep:
        for v, name in enumerate(names):
            try:
                m0, _ = ham.time_apply(x, y, args.reps, v, False)
                m1, _ = ham.time_apply(x, y, args.reps, v, True)
                print(f"{args.case} {args.apply_precision} variant {v} ({name}): apply_ms={m0:.4f} "
                      f"with_alpha_ms={m1:.4f}")
            except ed.AEDError as e:
                print(f"{args.case} {args.apply_precision} variant {v} ({name}): {e}")
        return
    ham.time_apply(x, y, 1, args.variant, args.alpha)
    ms, v = ham.time_apply(x, y, args.reps, args.variant, args.alpha)
    print(f"{args.case} {args.apply_precision} D={ham.dim} variant={v} ({names[v]}) alpha={int(args.alpha)} "
          f"apply_ms={ms:.4f}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-configs", action="store_true", help="skip the config-1/3/4 sections of the default line")
    ap.add_argument("--workload", default="l28",
                    choices=["l28", "square", "batch", "serve", "momentum", "spin", "apply"])
    ap.add_argument("--case", default="l28", help="apply: l24, l26, l28, sq6x5, spin1_l18, mom_l28, spin1mom_l18")
    ap.add_argument("--apply-precision", default="fp64", choices=["fp64", "fp32"], help="apply: vector precision")
    ap.add_argument("--variant", type=int, default=-1, help="apply: variant index (-1: autotuned)")
    ap.add_argument("--reps", type=int, default=3, help="apply: timed applies")
    ap.add_argument("--sweep", action="store_true", help="apply: time every variant with and without partials")
    ap.add_argument("--alpha", action="store_true", help="apply: with the Lanczos step's <x,y> partials")
    ap.add_argument("--k", type=int, default=0, help="apply mom_l28 / spin1mom_l18: momentum index")
    ap.add_argument("--sector-workers", type=int, default=4, help="momentum: sectors solved at once")
    ap.add_argument("--requests", type=int, default=2000, help="serve: number of requests (20000 = full stream)")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: offered rate, requests/s (the stream's is 200)")
    ap.add_argument("--lanes", type=int, default=2, help="serve: single-instance lanes for large requests (0: none)")
    ap.add_argument("--lane-min-dim", type=int, default=1 << 21, help="serve: smallest dimension sent to a lane")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"], help="serve: engine precision")
    ap.add_argument("--steps-per-launch", type=int, default=8)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload == "apply":
        run_apply(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "momentum":
        run_momentum(args)
    elif args.workload == "spin":
        run_spin(args)
    elif args.workload == "square":
        run_square(args)
    elif args.workload == "batch":
        run_batch(args)
    elif args.workload == "serve":
        run_serve(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
