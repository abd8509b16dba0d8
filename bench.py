"""Benchmark of the AMOEBA electrostatics path on B200.

Metric: full AMOEBA electrostatic E+F evaluations per second (permanent
multipoles + mutual induced dipoles to 1e-6 D RMS + polarization, real-space
Ewald with Thole damping and smooth PME), mixed precision, on the seeded
32,768-water box (98,304 atoms, 99.3 A, PME grid 108^3, order 5, alpha
0.5446, cutoff 7 A).  One step = one E+F evaluation.  The 4,096-water box
(12,288 atoms, 49.7 A, 54^3) is reported beside it.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Multi-GPU runs are independent replicas (one box per rank, seed = rank):
value = evaluations of all ranks / max-over-ranks device time.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WATERS, BOX, GRID = 32768, 99.3, 108
SMALL = (4096, 49.7, 54)          # the 4,096-water box, reported beside the headline
METRIC = "AMOEBA E+F evaluations/s (mixed precision, mutual polarization to 1e-6 D)"
UNIT = "evals/s"
FLUSH_BYTES = 256 << 20          # > 126 MB L2, written before every timed step


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "20"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
            return
        # the timed region is short: start it only once samples are flowing
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.p.poll() is None:
            self.f.flush()
            if os.path.getsize(self.f.name) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = [r.split(", ") for r in open(self.f.name).read().strip().splitlines() if r.count(",") >= 8]
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows)}


def ncu_traffic(kernel, pairs):
    """DRAM bytes (read + write) per launch of `kernel` on this workload from
    the committed ncu capture summary, or None.  The capture is of a smaller
    box (the headline box is too large for a multi-pass capture); its traffic
    is scaled to this launch by the directed pairs each processes, the unit
    the kernel's bytes grow with."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_traffic.json")) as f:
            d = json.load(f)[kernel]
        return (d["dram_bytes_read"] + d["dram_bytes_write"]) * pairs / d["directed_pairs"]
    except (OSError, KeyError, ZeroDivisionError):
        return None


def workload_config():
    return {"workload": f"{WATERS}-water AMOEBA box (water03), {3 * WATERS} atoms, {BOX} A, PME {GRID}^3 order 5, "
                        "alpha 0.5446, cutoff 7 A, mutual polarization 1e-6 D",
            "atoms": 3 * WATERS, "pme_grid": [GRID] * 3, "cutoff_A": 7.0, "poleps_D": 1e-6,
            "precision": "mixed (FP32 pairs/grids, FP64 PCG reductions, accumulators, correction sweep)",
            "l2": f"flushed before every timed step ({FLUSH_BYTES >> 20} MiB write)"}


def cpu_baseline_oracle(seed=0, system=None):
    """FP64 CPU restatement (OpenMP, all host cores) on one full evaluation of
    the same box at the metric's convergence (1e-6 D): a bounded sample of
    the workload."""
    from oracle import oracle
    from polmdqc_b200 import abi, systems
    from polmdqc_b200.engine import Settings
    s = system if system is not None else systems.water_box(WATERS, BOX, seed=seed)
    st = Settings(nfft=(GRID,) * 3, precision=abi.PREC_FP64)
    oracle.forward(systems.water_box(27, 9.32, seed=1), Settings(nfft=(16,) * 3, cutoff=4.6))  # load + warm
    t = time.perf_counter()
    o = oracle.forward(s, st, flags=abi.DO_ENERGY | abi.DO_GRADIENT)
    dt = time.perf_counter() - t
    return {"value": 1.0 / dt, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": f"1 full E+F evaluation of the {WATERS}-water box, FP64, PCG to 1e-6 D ({o.pcg_iters} "
                      f"iterations), OpenMP on {os.cpu_count()} threads ({dt:.2f} s)"}


def reference_own_mode(s, device, reps):
    """The reference's own CPU code on the same box, in the one electrostatics
    mode it computes: non-Ewald permanent multipoles within a 7 A cutoff
    (empole_a, src/md/empole.cpp:96-357) through energy<CalcMode::Gradient>()
    (src/md/energy.cpp:31), run by oracle/_ref/ref_time (the reference built
    from its sources) on every host core.  This library runs the same mode on
    the same coordinates (the Tinker file's 6 decimals), FP64 and mixed,
    device-resident with L2 flushed; em is compared with the reference's."""
    from polmdqc_b200 import abi, systems
    from polmdqc_b200.engine import Engine, Settings
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_time")
    prm = os.path.join(ROOT, "oracle", "_ref", "params", "water03.prm")
    if not (os.path.exists(exe) and os.path.exists(prm)):
        return {"unavailable": "oracle/_ref (the reference built from its sources) is not present"}
    with tempfile.TemporaryDirectory() as d:
        xyz, key = os.path.join(d, "box.xyz"), os.path.join(d, "box.key")
        systems.write_tinker(s, xyz, key, prm, ["multipoleterm only", "mpole-cutoff 7.0"])
        p = subprocess.run([exe, "--reps", "1", xyz, "-k", key], capture_output=True, text=True, timeout=900, cwd=d)
        if p.returncode != 0:
            return {"unavailable": f"ref_time exited {p.returncode}: {p.stderr.strip()[-200:]}"}
        ref = json.loads(p.stdout.strip().splitlines()[-1])
    s6 = dataclasses.replace(s, xyz=np.round(s.xyz, 6))
    flags = abi.DO_ENERGY | abi.DO_GRADIENT
    cpu_s = min(ref["call_s"])
    out = {"what": "the reference's only electrostatics mode (non-Ewald permanent multipoles, cutoff 7 A, "
                   "energy<Gradient>) on the same box: the reference's own code (oracle/_ref/ref_time) on the "
                   "host cores beside this library in the same mode on the GPU",
           "reference_cpu": {"seconds_per_call": cpu_s, "evals_per_s": 1.0 / cpu_s, "threads": ref["nthread"],
                             "em": ref["em"], "kind": "reference"}}
    for name, prec in (("fp64", abi.PREC_FP64), ("mixed", abi.PREC_MIXED)):
        e = Engine(s6, Settings(use_ewald=False, poltyp=abi.POL_NONE, cutoff=7.0, precision=prec, device=device))
        try:
            g = e.forward(flags)
            e.bench(3, flags, FLUSH_BYTES)
            ms, _ = e.bench(reps, flags, FLUSH_BYTES)
        finally:
            e.close()
        t = float(np.median(ms))
        out["gpu_" + name] = {"ms_per_eval": t, "evals_per_s": 1000.0 / t, "em": g.em,
                              "em_rel_diff_vs_reference": abs(g.em - ref["em"]) / abs(ref["em"]),
                              "dem_abs_sum_rel_diff": abs(float(np.abs(g.dem).sum()) - ref["dem_abs_sum"])
                              / ref["dem_abs_sum"],
                              "speedup_vs_reference_cpu": cpu_s * 1000.0 / t}
    return out


def error_vs_oracle(s, g):
    """Errors of a GPU result g against the FP64 oracle on the same box with
    the PCG converged to 1e-9 D."""
    from oracle import oracle
    from polmdqc_b200 import abi
    from polmdqc_b200.engine import Settings
    from polmdqc_b200.prm import DEBYE
    o = oracle.forward(s, Settings(nfft=(GRID,) * 3, precision=abi.PREC_FP64), tol=1e-9,
                       flags=abi.DO_ENERGY | abi.DO_GRADIENT | abi.DO_DIPOLES)
    du = np.concatenate([g.uind - o.uind, g.uinp - o.uinp])
    return {"em_rel": abs(g.em - o.em) / abs(o.em), "ep_rel": abs(g.ep - o.ep) / abs(o.ep),
            "force_rms_kcal_mol_A": float(np.sqrt(np.mean((g.dem + g.dep - o.dem - o.dep) ** 2))),
            "force_max_kcal_mol_A": float(np.abs(g.dem + g.dep - o.dem - o.dep).max()),
            "dipole_rms_D": DEBYE * float(np.sqrt(np.mean(np.sum(du * du, axis=1)))),
            "pcg_eps_D": g.pcg_eps,
            "reference": "FP64 CPU oracle on the same box, PCG converged to 1e-9 D"}


def reduce_max(x, dist, device):
    """Maximum over the ranks of a float (x itself without a process group):
    the slowest rank's time, as the replica timing rule asks."""
    if not dist:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world, steps, seconds):
    """Whole-job rate of independent replicas: every rank's evaluations over
    the slowest rank's time."""
    return world * steps / seconds


def run_reference(args):
    """CPU reference arm: the oracle port of the full path (the reference
    itself implements only non-Ewald multipoles, src/md/empole.cpp:53-64)."""
    rank = int(os.environ.get("RANK", 0))
    if rank != 0:
        return 0
    steps = max(1, min(args.steps, 2))
    vals = []
    base = None
    for k in range(steps):
        base = cpu_baseline_oracle(seed=k)
        vals.append(base["value"])
    v = statistics.mean(vals)
    base["value"] = v
    base["sample"] += f"; {steps} step(s) (steps capped at 2 to bound the run)"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
            "warmup": 0, "ms_per_step": 1000.0 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded water box)", "config": workload_config(),
            "cpu_baseline": base, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def ion_solution_timings(device, reps):
    """8,000 waters + 22 Na+ + 22 Cl- (amoebabio18), 62.1 A, PME 72^3: mixed
    and FP64 forward (device time, L2 flushed) and forward + adjoint (host
    wall clock per pair of synchronous calls)."""
    from polmdqc_b200 import abi, systems
    from polmdqc_b200.engine import Engine, Settings
    s = systems.ion_solution(seed=0)
    flags = abi.DO_ENERGY | abi.DO_GRADIENT
    out = {"config": "8000 waters + 22 Na+ + 22 Cl- (amoebabio18), 24,044 atoms, 62.1 A, PME 72^3 order 5, "
                     "cutoff 7 A, mutual polarization 1e-6 D"}
    for name, prec in (("mixed", abi.PREC_MIXED), ("fp64", abi.PREC_FP64)):
        e = Engine(s, Settings(nfft=(72, 72, 72), precision=prec, device=device))
        try:
            e.bench(3, flags, FLUSH_BYTES)
            ms, _ = e.bench(reps, flags, FLUSH_BYTES)
            e.forward(flags)
            e.backward(1.0)
            t0 = time.perf_counter()
            for _ in range(reps):
                e.forward(flags)
                e.backward(1.0)
            fb = 1000.0 * (time.perf_counter() - t0) / reps
            out[name] = {"forward_ms": float(np.median(ms)), "forward_plus_adjoint_ms": fb}
        finally:
            e.close()
    out["mixed_over_fp64_forward"] = out["fp64"]["forward_ms"] / out["mixed"]["forward_ms"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    from polmdqc_b200 import abi, systems
    from polmdqc_b200.engine import Engine, Settings

    rank, world = int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    def max_over_ranks(x):
        return reduce_max(x, dist, "cuda")

    s = systems.water_box(WATERS, BOX, seed=rank)
    st = Settings(nfft=(GRID,) * 3, precision=abi.PREC_MIXED, device=local)
    eng = Engine(s, st)
    flags = abi.DO_ENERGY | abi.DO_GRADIENT
    eng.bench(max(args.warmup, 3), flags, FLUSH_BYTES)           # warm-up (untimed)
    barrier()
    clocks = Clocks(local) if rank == 0 else None
    ms, launches = eng.bench(args.steps, flags, FLUSH_BYTES)      # timed: device-resident
    barrier()
    clk = clocks.stop() if clocks else None
    dev_s = max_over_ranks(float(np.sum(ms)) / 1000.0)
    value = replica_rate(world, args.steps, dev_s)

    # end to end through the C ABI: host coordinates (pinned) in, gradients out
    n = s.n
    xyz = torch.from_numpy(s.xyz.reshape(-1).copy()).pin_memory().numpy()
    dem = torch.zeros(3 * n, dtype=torch.float64).pin_memory().numpy()
    dep = torch.zeros(3 * n, dtype=torch.float64).pin_memory().numpy()
    for _ in range(2):
        eng.set_coords(xyz)
        eng.forward_into(flags, dem, dep)
    barrier()
    t0 = time.perf_counter()
    iters = []
    for _ in range(args.steps):
        eng.set_coords(xyz)
        em, ep, it, eps = eng.forward_into(flags, dem, dep)
        iters.append(it)
    barrier()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": world * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 8 * 3 * n + 8 * 6,
           "d2h_bytes_per_step": 8 * 2 * 3 * n + 8 * (8 + 8 + 4) + 4 * 2}

    # dominant kernel of ours: the PCG's stored-coefficient T.u (HBM-bound once
    # L2 is flushed), timed live with CUDA events on the library's stream
    tu_ms, tu_bytes, tu_pairs = eng.time_tu_kernel(reps=20, flush_bytes=FLUSH_BYTES)

    # the same workload in plain FP64 on the GPU: speed and the mixed path's error
    st64 = Settings(nfft=(GRID,) * 3, precision=abi.PREC_FP64, device=local)
    e64 = Engine(s, st64)
    ms64, _ = e64.bench(max(3, args.steps // 2), flags, FLUSH_BYTES)
    r64 = e64.forward(flags)
    rmx = eng.forward(flags | abi.DO_DIPOLES)
    e64.close()
    fp64_value = world * len(ms64) / max_over_ranks(float(np.sum(ms64)) / 1000.0)
    err = {"em_rel": abs(rmx.em - r64.em) / abs(r64.em), "ep_rel": abs(rmx.ep - r64.ep) / abs(r64.ep),
           "force_rms_kcal_mol_A": float(np.sqrt(np.mean((rmx.dem + rmx.dep - r64.dem - r64.dep) ** 2))),
           "pcg_eps_D": rmx.pcg_eps, "reference": "FP64 GPU path"}

    # the 4,096-water box, mixed and FP64, device-resident (reported beside the headline)
    small = {}
    sw, sl, sg = SMALL
    s_small = systems.water_box(sw, sl, seed=rank)
    for name, prec in (("mixed", abi.PREC_MIXED), ("fp64", abi.PREC_FP64)):
        e = Engine(s_small, Settings(nfft=(sg,) * 3, precision=prec, device=local))
        try:
            e.bench(3, flags, FLUSH_BYTES)
            mss, _ = e.bench(max(3, args.steps // 2), flags, FLUSH_BYTES)
        finally:
            e.close()
        small[name] = world * len(mss) / max_over_ranks(float(np.sum(mss)) / 1000.0)
    small = {"config": f"{sw} waters, {3 * sw} atoms, {sl} A, PME {sg}^3", "unit": UNIT, "mixed": small["mixed"],
             "fp64": small["fp64"], "mixed_over_fp64": small["mixed"] / small["fp64"]}

    # the adjoint (amg_backward after a forward): wall time of the synchronous
    # call, gradients copied to the host, on the bench box
    eng.forward(flags)
    for _ in range(2):
        eng.backward(1.0)
    nb = max(3, min(20, args.steps // 5))
    barrier()
    t0 = time.perf_counter()
    for _ in range(nb):
        eng.backward(1.0)
    barrier()
    adjoint_ms = max_over_ranks(1000.0 * (time.perf_counter() - t0) / nb)
    ions = ion_solution_timings(local, nb) if world == 1 else None

    if rank == 0:
        peaks, src = load_peaks()
        achieved = tu_bytes / (tu_ms * 1e-3) / 1e9
        roofline = {"kernel": "k_tu_stored (PCG real-space T.u, stored pair coefficients)", "bound": "hbm",
                    "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": achieved / peaks["hbm_gbs"], "traffic": ncu_traffic("k_tu_stored", tu_pairs),
                    "bytes_per_launch": tu_bytes, "directed_pairs": tu_pairs, "avg_launch_ms": tu_ms,
                    "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({src}); L2 flushed before each timed launch"}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1000.0 * dev_s / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (mixed)", "data": "synthetic (seeded water box)",
                "config": workload_config(), "e2e": e2e, "gpu_launches": launches, "clocks": clk,
                "pcg_iterations": int(statistics.median(iters)), "em": em, "ep": ep,
                "ns_per_day": {"dt_1fs": value * 86400 * 1e-6, "dt_2fs": value * 86400 * 2e-6},
                "roofline": roofline, "fp64_gpu_value": fp64_value, "mixed_over_fp64": value / fp64_value,
                "mixed_error_vs_fp64": err,
                "adjoint_ms": {"value": adjoint_ms, "calls": nb,
                               "what": "amg_backward after one forward (d/d coordinates, local multipoles, "
                                       "polarizabilities, Thole factors), synchronous, host wall clock"}}
        line["config_4096_waters"] = small
        from polmdqc_b200.engine import fma_peak
        line["fma_peak_gflops"] = {"fp32": fma_peak(local, False), "fp64": fma_peak(local, True),
                                   "what": "amg_fma_peak: independent FMA chains on every SM, 2 flops per FMA"}
        if ions:
            line["ion_solution"] = ions
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_oracle(seed=0, system=s)
            line["mixed_error_vs_oracle"] = error_vs_oracle(s, rmx)
            line["reference_own_mode"] = reference_own_mode(s, local, max(3, args.steps // 2))
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
