"""Blocks of the benchmark's spun-up state, for the CPU baseline.

bench.py times the float32 step on the D3Q27 256^3 spherical Riemann problem
after 150 untimed spin-up steps.  The host-side oracle cannot simulate that
box, and a coarse re-simulation (24^3) has a far sharper blast that iterates
several times more per node.  This script runs the spin-up on a GPU with the
library (the benchmark's parameters), cuts `--blocks` seeded blocks of
`--edge`^3 nodes out of the state it times, and stores them (float32, as the
GPU holds them) with the GPU's per-node iteration counts of the next step:

    python tests/golden/make_cpu_sample.py --out tests/golden/bench/sphere256_blocks.npz

bench.py's CPU baseline and its reference arm step every block once per
timed step on the oracle (zero-gradient block faces), so the host does the
same work per node as the GPU at the same stage of the run.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)


def main():
    import bench
    import lbmpond_b200 as pond
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden", "bench", "sphere256_blocks.npz"))
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--spinup", type=int, default=150)
    ap.add_argument("--blocks", type=int, default=8)
    ap.add_argument("--edge", type=int, default=14)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    n, e = args.size, args.edge
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    with pond.Solver(lattice="D3Q27", shape=(n, n, n), interp=pond.LAGR4, precision="fp32", tau=bench.TAU,
                     tol_abs=bench.TOL_ABS, tol_rel=bench.TOL_REL) as s:
        s.init("sphere", *bench.sphere_params())
        s.step(args.spinup)
        f, rho, g = s.get_state()
        s.keep_niter(True)
        s.step(1)
        niter = s.niter()
        d = s.diagnostics()
    rng = np.random.default_rng(args.seed)
    corners = rng.integers(0, n - e + 1, (args.blocks, 3))
    idx = []
    for cx, cy, cz in corners:
        z, y, x = np.meshgrid(np.arange(cz, cz + e), np.arange(cy, cy + e), np.arange(cx, cx + e), indexing="ij")
        idx.append((x + n * (y + n * z)).ravel())
    idx = np.stack(idx)  # [blocks, e^3], x fastest within a block
    np.savez_compressed(args.out, f=f[:, idx].astype(np.float32), rho=rho[idx].astype(np.float32),
                        g=g[:, idx].astype(np.float32), niter_gpu=niter[idx].astype(np.int8), corners=corners,
                        edge=e, size=n, spinup=args.spinup, tau=bench.TAU, tol=(bench.TOL_ABS, bench.TOL_REL),
                        niter_mean_domain=d["niter_mean"])
    print(f"{args.blocks} blocks of {e}^3: GPU iterations {niter[idx].mean():.3f} per node in the blocks, "
          f"{d['niter_mean']:.3f} over the domain")


if __name__ == "__main__":
    main()
