"""Generate the golden fixtures of the PonD step from the reference's own CUDA
kernels (engrab6/lbmPonD, built for sm_100a by oracle/build_ref.sh and
driven by oracle/ref_main.cu).  Needs a CUDA device and the binaries in
oracle/_ref/; writes one compressed .npz per case:

    python tests/golden/make_golden.py --out tests/golden

Each case stores the seeded input state, the number of steps, tau and the
reference's output state (float64, host layout f[Q,N], rho[N], g[4,N]).
The reference has no golden files or tests of its own; these fixtures are the
pin between it and the FP64 oracle (tests/test_golden.py).
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402  (lattice tables only)
from tests.states import perturbed_populations, smooth_state, sod_state  # noqa: E402

MAGIC = 0x504F4E44
LAT_NAME = {0: "D1Q5", 1: "D3Q27", 2: "D3Q125"}


def write_state(path, f, rho, g, shape):
    Q = f.shape[0]
    with open(path, "wb") as fp:
        np.array([MAGIC, Q], dtype=np.uint32).tofile(fp)
        np.array(shape, dtype=np.int64).tofile(fp)
        f.astype(np.float64).tofile(fp)
        rho.astype(np.float64).tofile(fp)
        g.astype(np.float64).tofile(fp)


def read_state(path, Q, shape):
    N = int(np.prod(shape))
    with open(path, "rb") as fp:
        hdr = np.fromfile(fp, dtype=np.uint32, count=2)
        assert hdr[0] == MAGIC and hdr[1] == Q
        sh = np.fromfile(fp, dtype=np.int64, count=3)
        assert tuple(sh) == tuple(shape)
        f = np.fromfile(fp, dtype=np.float64, count=Q * N).reshape(Q, N)
        rho = np.fromfile(fp, dtype=np.float64, count=N)
        g = np.fromfile(fp, dtype=np.float64, count=4 * N).reshape(4, N)
        niter_max = int(np.fromfile(fp, dtype=np.int32, count=1)[0])
        ns = int(np.fromfile(fp, dtype=np.int32, count=1)[0])
        ms = np.fromfile(fp, dtype=np.float32, count=ns)
    return f, rho, g, niter_max, ms


def acoustic(nx, T0=0.1, A=0.02, gamma=3.0):
    """init.cu:43-50 (the reference's shipped initial condition)."""
    x = np.arange(nx)
    P = 1 + A * np.sin(x * 2 * np.pi / nx)
    T = T0 * P ** ((gamma - 1) / gamma)
    rho = P / T
    u = A * np.sin(x * 2 * np.pi / nx) * T0 / np.sqrt(gamma * T0)
    z = np.zeros(nx)
    return rho, np.stack([u, z, z, T])


def cases():
    out = []
    # name, lattice, shape, tau, nsteps, (rho, g), perturb-seed or None
    out.append(("d1q5_acoustic_128", 0, (128, 1, 1), 0.9, 10, acoustic(128), None))
    out.append(("d1q5_sod_128", 0, (128, 1, 1), 0.55, 6, sod_state(128, (1.0, 0.0, 0.01), (0.125, 0.0, 0.008)), None))
    out.append(("d1q5_smooth_1024", 0, (1024, 1, 1), 0.6, 5, smooth_state((1024, 1, 1), 1, seed=11, modes=3), 11))
    out.append(("d3q27_smooth_8", 1, (8, 8, 8), 0.9, 3, smooth_state((8, 8, 8), 3, seed=12, modes=1), 12))
    rho, g = smooth_state((16, 16, 16), 3, seed=13, modes=1, du=0.03)
    out.append(("d3q27_smooth_16", 1, (16, 16, 16), 0.7, 2, (rho, g), None))
    out.append(("d3q125_smooth_8x4x4", 2, (8, 4, 4), 0.9, 2, smooth_state((8, 4, 4), 3, seed=14, modes=1, du=0.02), 14))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--refdir", default=os.path.join(ROOT, "oracle", "_ref"))
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    for name, lat, shape, tau, nsteps, (rho, g), pseed in cases():
        t = O.tables(lat)
        f = t.w[:, None] * rho[None, :]
        if pseed is not None:
            f = perturbed_populations(O, lat, rho, g, seed=pseed)
        binary = os.path.join(args.refdir, f"ref_pond_{LAT_NAME[lat]}_double_{shape[0]}x{shape[1]}x{shape[2]}")
        with tempfile.TemporaryDirectory() as td:
            fin, fout = os.path.join(td, "in.state"), os.path.join(td, "out.state")
            write_state(fin, f, rho, g, shape)
            r = subprocess.run([binary, fin, fout, str(nsteps), repr(tau)], capture_output=True, text=True)
            if r.returncode != 0:
                raise SystemExit(f"{name}: reference run failed ({r.returncode})\n{r.stdout}\n{r.stderr}")
            fo, ro, go, niter_max, ms = read_state(fout, t.Q, shape)
        np.savez_compressed(os.path.join(args.out, name + ".npz"), lattice=lat, shape=np.array(shape), tau=tau,
                            nsteps=nsteps, f_in=f, rho_in=rho, g_in=g, f_out=fo, rho_out=ro, g_out=go,
                            niter_max=niter_max, kernel_ms=ms)
        print(f"{name}: NiterMax={niter_max} kernel ms/step={ms.mean():.3f}")


if __name__ == "__main__":
    main()
