"""Profiling driver: a few evaluations of a seeded water box, for ncu.

    python -m polmdqc_b200.profile --waters 4096 --evals 3 [--fp64] [--backward 2]

Box sizes and PME grids are those of the benchmark configurations (216, 4,096
and 32,768 waters), plus a 19,683-water box (27^3 lattice, the same density and
grid spacing) whose stored pair rows (~170 MB) exceed L2 while the whole
context stays near 1 GB: the size for multi-pass ncu captures.  Set AMG_NO_GRAPH=1 to run the eager path, whose kernels
ncu can profile (it cannot see kernels inside graphs with conditional nodes).
"""
import argparse

from . import abi, systems
from .engine import Engine, Settings

BOXES = {216: (18.643, 24), 4096: (49.7, 54), 19683: (83.8, 90), 32768: (99.3, 108)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--waters", type=int, default=4096, choices=sorted(BOXES))
    ap.add_argument("--evals", type=int, default=3)
    ap.add_argument("--fp64", action="store_true")
    ap.add_argument("--bench", type=int, default=0, help="also time this many device-resident evaluations")
    ap.add_argument("--backward", type=int, default=0, help="then this many amg_backward calls (host wall time)")
    ap.add_argument("--e2e", type=int, default=0,
                    help="also time this many calls of set_coords + forward from pinned host buffers (host wall time)")
    a = ap.parse_args()
    box, grid = BOXES[a.waters]
    s = systems.water_box(a.waters, box, seed=0)
    prec = abi.PREC_FP64 if a.fp64 else abi.PREC_MIXED
    e = Engine(s, Settings(nfft=(grid,) * 3, precision=prec))
    for _ in range(a.evals):
        r = e.forward(abi.DO_ENERGY | abi.DO_GRADIENT)
    print(f"em {r.em:.6f} ep {r.ep:.6f} pcg {r.pcg_iters} {e.stats()}")
    print("phase ms (total, set-up, field, solve, forces; eager path only):", " ".join(f"{t:.3f}" for t in e.timing()))
    if a.bench:
        ms, launches = e.bench(a.bench, flush_bytes=256 << 20)
        print(f"device ms per evaluation: median {sorted(ms)[len(ms) // 2]:.3f} min {ms.min():.3f} "
              f"launches {launches}")
    if a.e2e:
        import time
        import torch  # pinned host buffers
        n = s.n
        xyz = torch.from_numpy(s.xyz.reshape(-1).copy()).pin_memory().numpy()
        dem = torch.zeros(3 * n, dtype=torch.float64).pin_memory().numpy()
        dep = torch.zeros(3 * n, dtype=torch.float64).pin_memory().numpy()
        flags = abi.DO_ENERGY | abi.DO_GRADIENT
        for _ in range(3):
            e.set_coords(xyz)
            e.forward_into(flags, dem, dep)
        t0 = time.perf_counter()
        for _ in range(a.e2e):
            e.set_coords(xyz)
            e.forward_into(flags, dem, dep)
        print(f"end-to-end ms per evaluation (host wall): {1000.0 * (time.perf_counter() - t0) / a.e2e:.3f}")
    if a.backward:
        import time
        e.backward(1.0)
        t0 = time.perf_counter()
        for _ in range(a.backward):
            e.backward(1.0)
        print(f"backward ms (host wall, synchronous): {1000.0 * (time.perf_counter() - t0) / a.backward:.3f}")
    e.close()


if __name__ == "__main__":
    main()
