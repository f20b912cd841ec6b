"""Run a few spin-S applies y = H x (the command the ncu summary of spin_hv_kernel uses).

    python -m alps_b200.profile_spin --reps 3

Workload: spin-1 Heisenberg chain L=18, Sz=0 (44,152,809 states), FP64.
Prints the mean CUDA-event time per apply.
"""

from __future__ import annotations

import argparse

import alps_b200 as ed


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    a = ap.parse_args()
    L = 18
    ham = ed.Hamiltonian(L, L, [(i, (i + 1) % L, 1.0, 1.0, 0.0) for i in range(L)], two_s=2)
    x, y = ham.new_vector(), ham.new_vector()
    ham.fill_random(x, 1)
    if a.warmup:
        ham.time_mult(x, y, a.warmup)
    print(f"spin-1 L={L} rows={ham.dim} apply_ms={ham.time_mult(x, y, a.reps):.4f}")


if __name__ == "__main__":
    main()
