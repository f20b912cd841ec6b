"""Run a few applies y = H x of one workload (the command the ncu summaries use).

    python -m alps_b200.profile_apply --workload l28 --precision fp64 --reps 3

Workloads: l28 (J1-J2 chain L=28, J2=0.25, D=40,116,600), sq6x5 (6x5 square
lattice with per-bond J in [0.8, 1.2], seed 3005, D=155,117,520), l24 (J1-J2
chain L=24, D=2,704,156).  Prints the mean CUDA-event time per apply.
"""

from __future__ import annotations

import argparse

import numpy as np

import alps_b200 as ed


def workload_bonds(name):
    if name in ("l28", "l24", "l26"):
        L = int(name[1:])
        bonds = []
        for i in range(L):
            bonds.append((i, (i + 1) % L, 1.0, 1.0, 0.0))
            bonds.append((i, (i + 2) % L, 0.25, 0.25, 0.0))
        return L, L // 2, bonds
    if name == "sq6x5":
        Lx, Wy = 6, 5
        raw = []
        for x in range(Lx):
            for y in range(Wy):
                s = x * Wy + y
                raw.append((s, x * Wy + (y + 1) % Wy))
                raw.append((s, ((x + 1) % Lx) * Wy + y))
        js = np.random.default_rng(3005).uniform(0.8, 1.2, len(raw))
        return Lx * Wy, Lx * Wy // 2, [(a, b, float(j), float(j), 0.0) for (a, b), j in zip(raw, js)]
    raise ValueError(name)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="l28")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--variant", type=int, default=-1, help="apply variant (-1: autotuned)")
    ap.add_argument("--alpha", action="store_true", help="with the fused step's <x,y> partials")
    ap.add_argument("--sweep", action="store_true", help="time every variant with and without partials")
    a = ap.parse_args()
    N, n_up, bonds = workload_bonds(a.workload)
    prec = ed.FP64 if a.precision == "fp64" else ed.FP32
    ham = ed.Hamiltonian(N, n_up, bonds, precision=prec)
    x, y = ham.new_vector(), ham.new_vector()
    ham.fill_random(x, 1)
    names = ed.apply_variants()
    if a.sweep:
        for v, name in enumerate(names):
            try:
                m0, _ = ham.time_apply(x, y, a.reps, v, False)
                m1, _ = ham.time_apply(x, y, a.reps, v, True)
                print(f"{a.workload} {a.precision} variant {v} ({name}): apply_ms={m0:.4f} with_alpha_ms={m1:.4f}")
            except ed.AEDError as e:
                print(f"{a.workload} {a.precision} variant {v} ({name}): {e}")
        return
    if a.warmup:
        ham.time_apply(x, y, a.warmup, a.variant, a.alpha)
    ms, v = ham.time_apply(x, y, a.reps, a.variant, a.alpha)
    print(f"{a.workload} {a.precision} D={ham.dim} variant={v} ({names[v]}) alpha={int(a.alpha)} apply_ms={ms:.4f}")


if __name__ == "__main__":
    main()
