"""Run a few momentum-sector applies y = H x (the command the ncu summary of mom_hv_kernel uses).

    python -m alps_b200.profile_momentum --reps 3

Workload: J1-J2 chain L=28 (J2 = 0.25), Sz=0, TOTAL_MOMENTUM = 0: 1,432,860
representatives, complex vectors.  Prints the mean CUDA-event time per apply.
"""

from __future__ import annotations

import argparse

import alps_b200 as ed
from alps_b200.profile_apply import workload_bonds


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--k", type=int, default=0, help="momentum index m of k = 2 pi m / 28")
    a = ap.parse_args()
    N, n_up, bonds = workload_bonds("l28")
    params = {"MODEL": "spin", "LATTICE": "nnn chain lattice", "L": N}
    k = ed.lattice_momenta(params)[a.k]
    ham = ed.Hamiltonian(N, n_up, bonds, translations=ed.lattice_translations(params, k))
    x, y = ham.new_vector(), ham.new_vector()
    ham.fill_random(x, 1)
    if a.warmup:
        ham.time_mult(x, y, a.warmup)
    ms = ham.time_mult(x, y, a.reps)
    print(f"momentum k={k[0]:.6f} rows={ham.dim} apply_ms={ms:.4f}")


if __name__ == "__main__":
    main()
