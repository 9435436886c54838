"""Generate the golden fixtures of the PonD step from the reference's own CUDA
kernels (engrab6/lbmPonD, built for sm_100a by oracle/build_ref.sh and
driven by oracle/ref_main.cu).  Needs a CUDA device and the binaries in
oracle/_ref/; writes one compressed .npz per case:

    python tests/golden/make_golden.py --out tests/golden

Each case stores the seeded input state, the number of steps, tau and the
reference's output state (float64, host layout f[Q,N], rho[N], g[4,N]).
The reference has no golden files or tests of its own; these fixtures are the
pin between it and the FP64 oracle (tests/test_golden.py).

Cases with a ``scheme`` run one of the reference's alternative interpolation
calls (steps.cu:444-463, selected by oracle/build_ref.sh's scheme argument);
cases with a ``mesh`` also pass a node mask and node positions, and with
``amr`` the reference's AMR kernels run after every step; cases with
``bc = mirror`` run the reference's disabled mirror walls, and with
``timecorr = s`` its TimeCorr(s) after every step.  ``--only`` makes a
subset (names containing any of the given words).
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


def read_niter_mean(path, Q, shape):
    """The mean per-node iteration count of the last step, appended after the
    state by oracle/ref_main.cu (None for an output without it)."""
    N = int(np.prod(shape))
    skip = 8 + 24 + 8 * (Q + 5) * N
    with open(path, "rb") as fp:
        fp.seek(skip)
        fp.read(4)
        ns = int(np.fromfile(fp, dtype=np.int32, count=1)[0])
        fp.seek(4 * ns, 1)
        tail = np.fromfile(fp, dtype=np.float64, count=1)
    return float(tail[0]) if tail.size else None


MESH_MAGIC = 0x4D455348


def write_mesh(path, mask, pos):
    with open(path, "wb") as fp:
        np.array([MESH_MAGIC], dtype=np.uint32).tofile(fp)
        np.array([mask.size], dtype=np.int64).tofile(fp)
        np.ascontiguousarray(mask, dtype=np.uint8).tofile(fp)
        np.ascontiguousarray(pos, dtype=np.float64).tofile(fp)


def read_mesh(path, N):
    with open(path, "rb") as fp:
        assert int(np.fromfile(fp, dtype=np.uint32, count=1)[0]) == MESH_MAGIC
        assert int(np.fromfile(fp, dtype=np.int64, count=1)[0]) == N
        mask = np.fromfile(fp, dtype=np.uint8, count=N)
        pos = np.fromfile(fp, dtype=np.float64, count=N)
    return mask, pos


def acoustic(nx, T0=0.1, A=0.02, gamma=3.0):
    """init.cu:43-50 (the reference's shipped initial condition)."""
    x = np.arange(nx)
    P = 1 + A * np.sin(x * 2 * np.pi / nx)
    T = T0 * P ** ((gamma - 1) / gamma)
    rho = P / T
    u = A * np.sin(x * 2 * np.pi / nx) * T0 / np.sqrt(gamma * T0)
    z = np.zeros(nx)
    return rho, np.stack([u, z, z, T])


def sparse_mask(nx, seed, density=0.7):
    """A seeded node mask with at most four inactive nodes in a row."""
    rng = np.random.default_rng(seed)
    m = (rng.random(nx) < density).astype(np.uint8)
    m[::5] = 1
    return m


def stretched(nx, amp=0.3):
    x = np.arange(nx, dtype=np.float64)
    return x + amp * np.sin(2 * np.pi * x / nx)


def scheme_cases():
    """Alternative interpolation calls and the 1D mesh: dicts with the keys of
    cases() plus scheme, and mesh = (mask, positions, amr) for mesh runs."""
    out = []

    def add(name, lat, shape, tau, nsteps, state, pseed, scheme, mesh=None, bc="periodic", timecorr=0.0):
        out.append(dict(name=name, lat=lat, shape=shape, tau=tau, nsteps=nsteps, state=state, pseed=pseed,
                        scheme=scheme, mesh=mesh, bc=bc, timecorr=timecorr))

    for scheme, seed in (("lagr2", 21), ("lagr3", 22), ("lagr5", 23)):
        add(f"d1q5_{scheme}_128", 0, (128, 1, 1), 0.7, 5, smooth_state((128, 1, 1), 1, seed=seed, modes=2), seed,
            scheme)
    add("d1q5_weno5_sod_128", 0, (128, 1, 1), 0.55, 6, sod_state(128, (1.0, 0.0, 0.01), (0.125, 0.0, 0.008)), None,
        "weno5")
    add("d3q27_lagr3_8", 1, (8, 8, 8), 0.8, 2, smooth_state((8, 8, 8), 3, seed=24, modes=1, du=0.03), 24, "lagr3")
    add("d3q27_lagr2_8", 1, (8, 8, 8), 0.8, 2, smooth_state((8, 8, 8), 3, seed=30, modes=1, du=0.03), 30, "lagr2")
    add("d3q27_lagr5_8", 1, (8, 8, 8), 0.8, 2, smooth_state((8, 8, 8), 3, seed=31, modes=1, du=0.03), 31, "lagr5")
    add("d1q5_gap2_mask_128", 0, (128, 1, 1), 0.7, 4, smooth_state((128, 1, 1), 1, seed=25, modes=2), 25, "gap2",
        (sparse_mask(128, 25), np.arange(128, dtype=np.float64), 0))
    add("d1q5_gap2_amr_sod_128", 0, (128, 1, 1), 0.6, 6, sod_state(128, (1.0, 0.0, 0.01), (0.125, 0.0, 0.008)),
        None, "gap2", ((np.arange(128) % 2 == 0).astype(np.uint8), np.arange(128, dtype=np.float64), 1))
    add("d1q5_nu3_128", 0, (128, 1, 1), 0.7, 4, smooth_state((128, 1, 1), 1, seed=26, modes=2), 26, "nu3",
        (np.ones(128, np.uint8), stretched(128), 0))
    # the reference's disabled mirror walls (propagate<N>'s outflow flag, steps.cu:1004-1013)
    add("d1q5_mirror_128", 0, (128, 1, 1), 0.7, 5, smooth_state((128, 1, 1), 1, seed=27, modes=2, du=0.03), 27,
        "lagr4", bc="mirror")
    add("d3q27_mirror_8", 1, (8, 8, 8), 0.8, 2, smooth_state((8, 8, 8), 3, seed=28, modes=1, du=0.03), 28, "lagr4",
        bc="mirror")
    add("d3q125_mirror_8x4x4", 2, (8, 4, 4), 0.9, 2, smooth_state((8, 4, 4), 3, seed=32, modes=1, du=0.02), 32,
        "lagr4", bc="mirror")
    # propagateWENO<3,5> on the 3D lattices (steps.cu:458; on D3Q125 through LBMpull's generic branch)
    # (small velocities: the smoothness row of steps.cu:783 lies elsewhere in 3D, and with larger
    # perturbations a few nodes of the float64 iteration cycle at the cap)
    add("d3q27_weno5_8", 1, (8, 8, 8), 0.8, 2, smooth_state((8, 8, 8), 3, seed=33, modes=1, du=0.01), 33, "weno5")
    add("d3q125_weno5_8x4x4", 2, (8, 4, 4), 0.9, 2, smooth_state((8, 4, 4), 3, seed=33, modes=1, du=0.01), 33,
        "weno5")
    # the reference's TimeCorr after every step (halving dt: u / 2, T / 4)
    add("d1q5_timecorr_128", 0, (128, 1, 1), 0.8, 3, smooth_state((128, 1, 1), 1, seed=29, modes=2, T0=0.4), 29,
        "lagr4", timecorr=0.5)
    return out


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


def all_cases():
    out = [dict(name=name, lat=lat, shape=shape, tau=tau, nsteps=nsteps, state=state, pseed=pseed, scheme="lagr4",
                mesh=None, bc="periodic", timecorr=0.0) for name, lat, shape, tau, nsteps, state, pseed in cases()]
    return out + scheme_cases()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--refdir", default=os.path.join(ROOT, "oracle", "_ref"))
    ap.add_argument("--only", nargs="*", default=None)
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    for c in all_cases():
        name, lat, shape, tau, nsteps, (rho, g), pseed = (c[k] for k in ("name", "lat", "shape", "tau", "nsteps",
                                                                          "state", "pseed"))
        if args.only and not any(w in name for w in args.only):
            continue
        t = O.tables(lat)
        f = t.w[:, None] * rho[None, :]
        if pseed is not None:
            f = perturbed_populations(O, lat, rho, g, seed=pseed)
        binary = os.path.join(args.refdir, f"ref_pond_{LAT_NAME[lat]}_double_{shape[0]}x{shape[1]}x{shape[2]}")
        if c["scheme"] != "lagr4":
            binary += "_" + c["scheme"]
        if c["bc"] == "mirror":
            binary += "_mirror"
        extra = {}
        with tempfile.TemporaryDirectory() as td:
            fin, fout = os.path.join(td, "in.state"), os.path.join(td, "out.state")
            write_state(fin, f, rho, g, shape)
            cmd = [binary, fin, fout, str(nsteps), repr(tau)]
            if c["mesh"] is not None:
                mask, pos, amr = c["mesh"]
                min_, mout = os.path.join(td, "in.mesh"), os.path.join(td, "out.mesh")
                write_mesh(min_, mask, pos)
                cmd += [min_, mout, str(amr)]
            env = dict(os.environ)
            env.pop("POND_REF_TIMECORR", None)
            if c["timecorr"] > 0:
                env["POND_REF_TIMECORR"] = repr(c["timecorr"])
            r = subprocess.run(cmd, capture_output=True, text=True, env=env)
            if r.returncode != 0:
                raise SystemExit(f"{name}: reference run failed ({r.returncode})\n{r.stdout}\n{r.stderr}")
            fo, ro, go, niter_max, ms = read_state(fout, t.Q, shape)
            if c["mesh"] is not None:
                mo, po = read_mesh(mout, int(np.prod(shape)))
                extra = dict(mask_in=mask, pos_in=pos, amr=amr, mask_out=mo, pos_out=po,
                             limit_lines=r.stdout.count("limit of cells division exceeded"))
        np.savez_compressed(os.path.join(args.out, name + ".npz"), lattice=lat, shape=np.array(shape), tau=tau,
                            nsteps=nsteps, f_in=f, rho_in=rho, g_in=g, f_out=fo, rho_out=ro, g_out=go,
                            niter_max=niter_max, kernel_ms=ms, scheme=c["scheme"], bc=c["bc"],
                            timecorr=c["timecorr"], **extra)
        print(f"{name}: NiterMax={niter_max} kernel ms/step={ms.mean():.3f}")


if __name__ == "__main__":
    main()
