"""Generates the golden fixtures under tests/golden from the oracle (and, for MT19937, from
libstdc++'s std::mt19937 through oracle/mt_std_check).  Run from the repository root:

    python tests/golden/make_golden.py
"""
import math
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402
from oracle import oracle_c as OC  # noqa: E402

OUT = Path(__file__).resolve().parent


def mt_fixture():
    subprocess.run(["make", "-C", str(ROOT / "oracle"), "-s"], check=True)
    seeds = np.array([5489, 0, 1, 20260, 4294967295], dtype=np.uint64)
    outs = []
    for s in seeds:
        r = subprocess.run([str(ROOT / "oracle" / "mt_std_check"), str(int(s)), "1300"], capture_output=True,
                           text=True, check=True)
        outs.append(np.array([int(v) for v in r.stdout.split()], dtype=np.uint64).astype(np.uint32))
    np.savez_compressed(OUT / "mt19937.npz", seeds=seeds, outputs=np.stack(outs))


def lattice_fixture():
    cfg = O.LVLattice()
    L, x = cfg.generator()
    V, niter, dt = O.solve_lattice_fp64(L, x, cfg.strikes, cfg.r, cfg.period, cfg.nmat, cfg.dt0)
    y0 = O.nearest_node(x)
    np.savez_compressed(OUT / "lattice_lv512.npz", quotes=V[:, y0, :], niter=niter, dt=dt, y0=y0)


def mc_fixture():
    cfg = O.LVLattice(n=128)
    L, x = cfg.generator()
    niter, dt = O.plan_niter(L, 1 / 252, cfg.dt0)
    P = O.square(O.ek(L, dt), niter)
    Cm = O.cumrows_f32(P)
    y0 = O.nearest_node(x)
    disc = math.exp(-cfg.r * 64 / 252)
    paths, sums = OC.mc_paths(Cm, y0, 777, 0, 512, 64, x=x, disc=disc)
    np.savez_compressed(OUT / "mc_small.npz", C=Cm, y0=y0, seed=777, x=x, disc=disc, paths=paths, sums=sums)


if __name__ == "__main__":
    mt_fixture()
    lattice_fixture()
    mc_fixture()
    print("written to", OUT)
