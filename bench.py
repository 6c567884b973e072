"""Throughput of the B200 nonbonded + PME path on the TIP3P water box.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Workload: 7,850 rigid TIP3P waters (23,550 atoms) at 33.4 nm^-3, cutoff
0.9 nm, reach 1.0 nm, PME order 4 on a 64^3 grid (0.1 nm), SETTLE, NVT at
300 K (Bussi, 0.1 ps), dt 2 fs, mixed precision: the MD step of the device
path (neighbor build when the test of validity asks, pair kernel, excluded
correction, PME with cuFFT, leap-frog + SETTLE + thermostat) as a CUDA
graph.  One bench step = `--md-steps` MD steps (1,000 by default, 2 ps:
the interval at which a run usually writes a frame; replays of the step
graph, then one read of the run's status); the L2 is flushed between bench
steps (a 256 MiB write).  Metric:
ns/day; with N GPUs, N independent replicas (the single box does not
shard): `value` is their aggregate and `per_replica_ns_day` each box's.

The reference arm (--impl reference) times the OpenMP CPU port of MDIR's
host algorithm for the same workload on the host cores, with MDIR's CPU
neighbor matrix at a reach of r_c + 0.15 nm."""

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

DT_PS = 0.002
# DRAM bytes read + written by one nb_pairs launch on the 23,550-atom box at
# the tuned reaches (ncu dram__bytes_read.sum + dram__bytes_write.sum; the
# counters need a profiler replay, so the figure is from a capture, not this run)
PAIRS_TRAFFIC_BYTES = 6.93e6
# MDIR's CPU neighbor matrix: the cutoff plus a 0.15 nm skin
CPU_SKIN_NM = 0.15
METRIC = "ns/day water box (TIP3P 23,550 atoms, PME, SETTLE, NVT, 2 fs)"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--md-steps", type=int, default=1000,
                   help="MD steps per bench step (2 ps; a trajectory frame's usual interval)")
    p.add_argument("--unroll", type=int, default=10, help="MD steps per graph")
    p.add_argument("--waters", type=int, default=7850)
    p.add_argument("--reach", type=float, default=1.2, help="reach of the outer lists (nm)")
    p.add_argument("--pruned", type=float, default=1.0, help="reach of the pruned inner lists (nm); 0: one list")
    p.add_argument("--equilibrate", type=int, default=5000, help="untimed MD steps before warm-up")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-tune", action="store_true", help="keep --reach/--pruned instead of the autotuner's choice")
    p.add_argument("--pair-sms", type=int, default=0, help="span of the pair grid with --no-tune (0: all SMs)")
    p.add_argument("--pair-blocks", type=int, default=0,
                   help="blocks of the pair kernel an SM with --no-tune (0: the library's default)")
    p.add_argument("--pme-fft", default="own", choices=["own", "cufft"],
                   help="the PME transforms: the library's three kernels, or cuFFT")
    p.add_argument("--only", choices=["adjoint", "batch", "precision"], help="run one leg alone (profiling)")
    p.add_argument("--adjoint-frames", type=int, default=64)
    p.add_argument("--frame-lanes", type=int, default=4,
                   help="contexts that evaluate the gradient leg's frames side by side")
    p.add_argument("--batch-frames", type=int, default=256)
    p.add_argument("--no-adjoint", action="store_true", help="skip the force-matching gradient leg")
    p.add_argument("--no-batch", action="store_true", help="skip the batch-of-frames leg")
    p.add_argument("--no-precision", action="store_true", help="skip the 1.07M-atom precision leg")
    return p.parse_args()


def workload(args):
    from mdir_b200 import systems
    s = systems.tip3p(waters=args.waters)
    s["reach"] = args.reach
    s["pruned"] = args.pruned
    v = systems.maxwell_velocities(s, 300.0, seed=2)
    return s, v


def config(args, s):
    """The workload (the same for both arms); each arm's own list reaches
    are tuning and go in its `tuning` key."""
    return {"workload": f"tip3p-{len(s['charges'])}", "atoms": len(s["charges"]),
            "box_nm": round(float(s["box"][0]), 4), "cutoff_nm": s["cutoff"],
            "pme_grid": list(s["grid"]), "pme_order": s["order"], "dt_ps": DT_PS,
            "md_steps_per_step": args.md_steps, "graph_steps": args.unroll, "ensemble": "NVT Bussi 300 K",
            "l2": "flushed between timed steps (256 MiB write); each step replays md_steps MD steps",
            "parallelism": f"replicas x{args.gpus}"}


class Clocks:
    """nvidia-smi samples during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.thread.join(timeout=2)
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) >= 9 for k in range(4)
                          if r[5 + k].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "samples": len(sm), "reasons": reasons}


def count_pairs(x, box, rc, excluded_pairs):
    """Unordered non-excluded pairs with r < r_c (minimum image), counted on
    the device in chunks: the work units of the pair kernel's roofline."""
    import torch
    X = x.to(torch.float64)
    L = torch.tensor(box, dtype=torch.float64, device=X.device)
    n = X.shape[0]
    total = 0
    chunk = 1024
    for a in range(0, n, chunk):
        d = X[a:a + chunk, None, :] - X[None, :, :]
        d -= L * torch.round(d / L)
        r2 = (d * d).sum(-1)
        i = torch.arange(a, min(a + chunk, n), device=X.device)[:, None]
        j = torch.arange(n, device=X.device)[None, :]
        total += int(((r2 < rc * rc) & (j > i)).sum())
    ex = np.asarray(excluded_pairs).reshape(-1, 2)
    if len(ex):
        xe = X.cpu().numpy()
        d = xe[ex[:, 0]] - xe[ex[:, 1]]
        d -= np.asarray(box) * np.round(d / np.asarray(box))
        total -= int((np.sum(d * d, 1) < rc * rc).sum())
    return total


def ns_per_day(md_steps, seconds):
    return md_steps / seconds * DT_PS * 86400.0 / 1000.0


def cpu_system(s):
    """The workload as the CPU port runs it: one neighbor matrix at MDIR's
    CPU reach r_c + 0.15 nm (no dual list)."""
    c = dict(s)
    c["reach"] = s["cutoff"] + CPU_SKIN_NM
    return c


def cpu_description():
    from oracle.cpu_port import reference_fft
    fft = ("MDIR's runtime/mdrt_fft.c + pocketfft built from the reference's sources" if reference_fft()
           else "numpy's pocketfft (MDIR's mdrt_fft.c not built)")
    return (f"f32 neighbor matrix at r_c + {CPU_SKIN_NM} nm (cells of half the reach), f32 row loop with MDIR's "
            f"D90 erfc, f64 excluded pairs, i64 PME spreading, {fft}; one matrix rebuild every 10 steps")


def cpu_baseline(s, x, steps=3):
    from oracle.cpu_port import time_md_steps
    c = cpu_system(s)
    sec, threads, tb, tf = time_md_steps(c, x, steps)
    return {"value": round(ns_per_day(1, sec), 4), "unit": "ns/day", "cores": threads, "kind": "port",
            "sample": f"{steps} force evaluations of the {len(s['charges'])}-atom box after a warm-up, "
                      f"{cpu_description()} amortised: {tf * 1e3:.1f} ms/eval, {tb * 1e3:.1f} ms/build",
            "tuning": {"reach_nm": c["reach"], "pruned_reach_nm": 0.0}}


def adjoint_leg(args, dev, flush, world=1, frames=64, reps=5, warmup=3):
    """Frames/s of the force-matching gradient of the differentiation form:
    a loss (1/K) sum |F - F_ref|^2 over `frames` jittered copies of the box
    (8 oxygen LJ types, N(0, 0.005 nm)), differentiated in the 8 sigma, 8
    epsilon and all charges through mdir_b200.torch.forces (forward, loss,
    adjoint backward), against the plain per-frame forward plus central
    differences, 2 forwards per parameter (timed forward x (2P + 1)).
    With N ranks each takes its own `frames` (weak scaling) and the
    gradients are summed over the ranks (one f64 all-reduce per batch)."""
    import torch
    from mdir_b200 import FrameEvaluator, systems
    from mdir_b200 import torch as mtorch
    from mdir_b200.ranks import max_over_ranks, sum_gradients
    s, X, target = systems.force_matching(frames=frames, waters=args.waters)
    n = X.shape[1]
    ev = FrameEvaluator(s, device=dev.index, lanes=args.frame_lanes)
    Xd = torch.tensor(X, device=dev)
    # target forces: the device forward at the perturbed parameters (untimed)
    ev.set_parameters(target["sigma"], target["epsilon"], target["charges"])
    F_ref = ev.forces(Xd).clone()
    sig = torch.tensor(s["type_sigma"], device=dev, requires_grad=True)
    eps = torch.tensor(s["type_epsilon"], device=dev, requires_grad=True)
    q = torch.tensor(s["charges"], device=dev, requires_grad=True)
    hX = torch.tensor(X).pin_memory()
    host_grad = torch.empty(n + 2 * len(s["type_sigma"]), dtype=torch.float64).pin_memory()

    def step(x):
        for t in (sig, eps, q):
            t.grad = None
        F = mtorch.forces(ev, sig, eps, q, x)
        loss = ((F - F_ref) ** 2).sum() / frames
        loss.backward()
        sum_gradients(sig.grad, eps.grad, q.grad)
        return loss

    stream = torch.cuda.current_stream(dev)
    for _ in range(warmup):
        step(Xd)
    torch.cuda.synchronize(dev)
    builds0 = ev.builds
    ms = []
    for _ in range(reps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step(Xd)
        b.record(stream)
        torch.cuda.synchronize(dev)
        ms.append(a.elapsed_time(b))
    dev_ms = max_over_ranks(statistics.median(ms), dev)
    # end to end: the frames from pinned host memory into the evaluator's
    # input buffer, the gradients back (warm-up passes first: the library
    # keeps the launches of buffers it has seen as graphs)
    e2e = []
    Xe = torch.empty_like(Xd)
    for i in range(warmup + reps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        Xe.copy_(hX, non_blocking=True)
        step(Xe)
        host_grad[:n].copy_(q.grad, non_blocking=True)
        host_grad[n:n + len(sig)].copy_(sig.grad, non_blocking=True)
        host_grad[n + len(sig):].copy_(eps.grad, non_blocking=True)
        torch.cuda.synchronize(dev)
        if i >= warmup:
            e2e.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(statistics.median(e2e), dev)
    # the plain forward of one frame with the same lists, for the differences
    Fb = torch.empty_like(Xd)
    fw = []
    for _ in range(reps):
        flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        ev.forces(Xd, out=Fb)
        b.record(stream)
        torch.cuda.synchronize(dev)
        fw.append(a.elapsed_time(b) / frames)
    fwd_ms = statistics.median(fw)
    n_lj = 2 * 8
    p_all = n_lj + n
    adj_fps = frames * world / (dev_ms / 1e3)
    fd_all = 1.0 / (fwd_ms / 1e3 * (2 * p_all + 1))
    fd_lj = 1.0 / (fwd_ms / 1e3 * (2 * n_lj + 1))
    return {"metric": "force-matching gradient frames/s (8 sigma + 8 epsilon + all charges)",
            "frames": frames, "atoms": n, "parameters": p_all,
            "value": round(adj_fps, 1), "unit": "frames/s", "ms_per_batch": round(dev_ms, 3),
            "e2e": {"value": round(frames * world / e2e_s, 1), "unit": "frames/s",
                    "h2d_bytes_per_step": int(X.nbytes), "d2h_bytes_per_step": int(host_grad.numel() * 8)},
            "forward_ms_per_frame": round(fwd_ms, 4),
            "fd_frames_per_s": round(fd_all, 4), "fd_frames_per_s_lj_only": round(fd_lj, 2),
            "speedup_vs_fd": round(adj_fps / fd_all, 1), "speedup_vs_fd_lj_only": round(adj_fps / fd_lj, 2),
            "builds_in_timed": int(ev.builds - builds0), "frame_lanes": ev.lanes,
            "gradient_error": "adjoint vs FP64 central differences (h = 1e-5) <= 1e-4 per element "
                              "(tests/test_gpu_adjoint.py, 23,550 atoms)",
            "targets": "device forward at parameters x (1 +- 2%)",
            "l2": "flushed before each timed batch (256 MiB write)"}


def batch_leg(args, dev, flush, world=1, rank=0, frames=256, reps=5, warmup=3):
    """Frames/s of the batching form: `frames` solvated frames of 1,000 to
    8,000 atoms (multiples of 3, each its own cubic cell at water density
    and its own PME grid, one LJ type table of 8 types), forces and
    per-frame energies of all of them by one launch of each kernel.  Timed:
    the build plus the evaluation (new frames need a build), and the
    evaluation alone replayed as a CUDA graph; an e2e figure uploads the
    positions from pinned host memory and reads the energies back.  With N
    ranks the frames are shared by bin-packing on atom counts and the
    per-frame energies all-gathered."""
    import torch
    from mdir_b200 import systems
    from mdir_b200.batch import BatchEvaluator, shard
    from mdir_b200.ranks import gather_frame_values, max_over_ranks
    allf = systems.batch_frames(count=frames)
    mine = shard([len(f["charges"]) for f in allf], world)[rank] if world > 1 else list(range(frames))
    fr = [allf[k] for k in mine]
    ev = BatchEvaluator(fr, device=dev.index)
    stream = torch.cuda.current_stream(dev)
    ev.build()
    choice = ev.autotune()
    for _ in range(warmup):
        ev.build()
        ev.force(energy=True, graph=True)
    torch.cuda.synchronize(dev)

    def timed(fn):
        ms = []
        for _ in range(reps):
            flush.zero_()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            torch.cuda.synchronize(dev)
            ms.append(a.elapsed_time(b))
        return max_over_ranks(statistics.median(ms), dev)

    def build_and_force():
        ev.build()
        ev.force(energy=True, graph=True)

    full_ms = timed(build_and_force)
    force_ms = timed(lambda: ev.force(energy=True, graph=True))
    hx = torch.tensor(ev.packed["positions"]).pin_memory()
    e2e = []
    for _ in range(reps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        ev.x.copy_(hx, non_blocking=True)
        ev.build()
        ev.force(energy=True, graph=True)
        e = ev.energies()
        e2e.append(time.perf_counter() - t0)
    e2e_s = max_over_ranks(statistics.median(e2e), dev)
    gather_frame_values(frames, mine, e["potential"])
    atoms = int(ev.n)
    return {"metric": "batched frames/s (forces + per-frame energies, build included)",
            "frames": frames, "atoms_this_rank": atoms, "value": round(frames / (full_ms / 1e3), 1),
            "unit": "frames/s", "ms_per_batch": round(full_ms, 3),
            "force_only": {"value": round(frames / (force_ms / 1e3), 1), "unit": "frames/s",
                           "ms_per_batch": round(force_ms, 3), "graph": True},
            "e2e": {"value": round(frames / e2e_s, 1), "unit": "frames/s",
                    "h2d_bytes_per_step": int(hx.numel() * 8), "d2h_bytes_per_step": int(len(fr) * 16 * 8)},
            "autotuned": choice, "grid_shapes": len({tuple(g) for g in ev.packed["grids"].tolist()}),
            "scaling": "strong (frames shared by bin-packing)" if world > 1 else "n/a",
            "l2": "flushed before each timed batch (256 MiB write)"}


def precision_leg(args, dev, flush, reach=1.6, pruned=1.05, thermalize=1000, nve=10000, every=500, timed=200):
    """The precision form on the large water box (356,700 TIP3P waters,
    1.07M atoms, 224^3 grid) in the deterministic mode (FP32 pairs, 64-bit
    fixed-point forces and grid, FP64 energies): ns/day of the NVT step,
    bitwise determinism of two 20-step runs from one state, and the NVE
    drift of the total energy (potential and kinetic energy at the same
    time) after a thermalisation.  The RMS force error against FP64 is the
    tests' (the oracle does not run here)."""
    import torch
    from mdir_b200 import NonbondedTerm, systems
    from mdir_b200.md import Integrator
    s = systems.tip3p(waters=356700)
    n = len(s["charges"])
    t = NonbondedTerm(n, device=dev.index)
    t.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
    t.set_exclusions(pairs=s["excluded_pairs"])
    t.set_interaction(s["cutoff"], reach, s["beta"])
    t.set_pruned_reach(pruned)
    t.set_pme(s["grid"], s["order"])
    t.set_deterministic(True)
    md = Integrator(t, s["masses"], s["waters"])
    x = torch.tensor(s["positions"], dtype=torch.float64, device=dev)
    v = torch.tensor(systems.maxwell_velocities(s, 300.0, seed=2), device=dev)
    box = s["box"]
    md.build(x, box)
    md.thermostat(300.0, 0.02, seed=11)
    md.run(x, v, box, DT_PS, thermalize, unroll=10)
    md.thermostat(300.0, 0.1, seed=12)
    stream = torch.cuda.current_stream(dev)
    flush.zero_()
    torch.cuda.synchronize(dev)
    th0 = md.thermo()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    md.run(x, v, box, DT_PS, timed, unroll=10)
    b.record(stream)
    torch.cuda.synchronize(dev)
    ms = a.elapsed_time(b)
    th1 = md.thermo()
    timed_counts = {k: int(th1[k] - th0[k]) for k in ("builds", "prunes", "regrows", "redone")}
    # two runs of 20 NVE steps from one state
    md.thermostat(300.0, 0.0, seed=13)
    x0, v0 = x.clone(), v.clone()
    md.build(x, box)
    md.run(x, v, box, DT_PS, 20, unroll=10)
    x1, v1 = x.clone(), v.clone()
    x.copy_(x0)
    v.copy_(v0)
    md.build(x, box)
    md.run(x, v, box, DT_PS, 20, unroll=10)
    same = bool(torch.equal(x, x1) and torch.equal(v, v1))
    # NVE
    samples = []
    for _ in range(nve // every):
        md.run(x, v, box, DT_PS, every - 1, unroll=0 if (every - 1) % 10 else 10)
        samples.append(md.total_energy(x, v, box, DT_PS))
    E = np.array(samples)
    tt = np.arange(len(E)) * every * DT_PS
    slope = float(np.polyfit(tt, E[:, 0], 1)[0]) if len(E) > 1 else 0.0  # kJ/mol/ps
    kin = float(E[:, 2].mean())
    return {"workload": "tip3p-1070100 (356,700 waters, 224^3 grid), deterministic mode",
            "reach_nm": reach, "pruned_reach_nm": pruned,
            "ns_per_day": round(ns_per_day(timed, ms / 1e3), 2), "ms_per_step": round(ms / timed, 4),
            "timed_steps": timed, "in_timed": timed_counts,
            "bitwise_deterministic_two_runs": same, "status": t.status(),
            "nve": {"steps": nve, "dt_ps": DT_PS, "drift_kj_mol_ns": round(slope * 1000.0, 3),
                    "drift_per_atom_kj_mol_ns": round(slope * 1000.0 / n, 6),
                    "drift_relative_to_kinetic_per_ns": round(slope * 1000.0 / kin, 6),
                    "total_std_kj_mol": round(float(E[:, 0].std()), 3),
                    "temperature_K": round(2.0 * kin / (md.thermo()["ndof"] * 0.0083144626181532), 1)},
            "force_error": "RMS relative force error vs FP64 at most 1e-5 on this box (split frames) and on the "
                           "23,550-atom box (tests/test_gpu_precision.py, tests/test_gpu_headline.py)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    s, v = workload(args)
    from oracle.cpu_port import CpuPort
    c = cpu_system(s)
    cp = CpuPort(c)
    x = s["positions"].copy()
    cp.build(x)
    for _ in range(max(args.warmup, 1)):
        cp.force(x)
    times = []
    for k in range(args.steps):
        t0 = time.perf_counter()
        if k % 10 == 0:
            cp.build(x)
        cp.force(x)
        times.append(time.perf_counter() - t0)
    sec = sum(times) / len(times)
    value = ns_per_day(1, sec)
    out = {"impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "ns/day",
           "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(sec * 1e3, 3), "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 pairs / f64 PME", "data": "synthetic",
           "config": config(args, s), "tuning": {"reach_nm": c["reach"], "pruned_reach_nm": 0.0},
           "cpu_baseline": {"value": round(value, 4), "unit": "ns/day", "cores": cp.threads, "kind": "port",
                            "sample": f"{args.steps} MD-step force evaluations of the {len(s['charges'])}-atom "
                                      f"box, {cpu_description()}; MDIR's CPU path is MLIR-generated and "
                                      "cannot be built here, so this is the OpenMP port of its algorithm"},
           "e2e": {"value": round(value, 4), "unit": "ns/day", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    import mdir_b200 as mdir
    from mdir_b200 import _lib
    from mdir_b200.md import Integrator
    from mdir_b200.term import NonbondedTerm, _dp, _hp, _stream

    if args.only:
        # one leg alone (profiling): its object as the JSON line
        flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
        if args.only == "adjoint":
            out = adjoint_leg(args, dev, flush, world, frames=args.adjoint_frames)
        elif args.only == "batch":
            out = batch_leg(args, dev, flush, world, rank, frames=args.batch_frames)
        else:
            out = precision_leg(args, dev, flush)
        if rank == 0:
            print(json.dumps({args.only: out}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    s, v0 = workload(args)
    n = len(s["charges"])

    def make_md(tuned=None):
        """The term and its integrator at the workload's reaches, or at the
        tuner's choice (a context of its own, its buffers sized for it)."""
        t_ = NonbondedTerm(n, device=local)
        t_.set_particles(s["charges"], s["types"], s["sigma"], s["epsilon"])
        t_.set_exclusions(pairs=s["excluded_pairs"])
        t_.set_interaction(s["cutoff"], s["reach"], s["beta"])
        t_.set_pruned_reach(s["pruned"])
        t_.set_pme(s["grid"], s["order"])
        t_.set_tuning(pme_fft=args.pme_fft)
        if tuned:
            t_.set_tuning(pair_sms=tuned["pair_sms"], pair_blocks_per_sm=tuned["pair_blocks_per_sm"],
                          staging_depth=tuned["staging_depth"], fused_prune=tuned["fused_prune"])
        else:
            if args.no_tune and args.pair_sms:
                t_.set_tuning(pair_sms=args.pair_sms)
            if args.no_tune and args.pair_blocks:
                t_.set_tuning(pair_blocks_per_sm=args.pair_blocks)
        m_ = Integrator(t_, s["masses"], s["waters"])
        m_.thermostat(300.0, 0.1, seed=1 + rank)
        return t_, m_

    # ---- device-resident leg -------------------------------------------------
    term, md = make_md()
    x = torch.tensor(s["positions"], dtype=torch.float64, device=dev)
    v = torch.tensor(v0, dtype=torch.float64, device=dev)
    box = s["box"]
    md.build(x, box)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    # untimed equilibration: the lattice start relaxes and heats; a strong
    # thermostat brings it to 300 K before the timed steps
    md.thermostat(300.0, 0.02, seed=7 + rank)
    md.run(x, v, box, DT_PS, args.equilibrate, unroll=args.unroll)
    md.thermostat(300.0, 0.1, seed=1 + rank)
    tuned = None
    if not args.no_tune:
        # the reaches and the span of the pair grid (untimed; the state is put back)
        tuned = md.tune(x, v, box, DT_PS)
        s["reach"], s["pruned"] = tuned["reach"], tuned["pruned_reach"]
        # the timed steps on a context made for the choice (the trials left
        # the lists with the room of the largest reach tried)
        md.close()
        term.close()
        term, md = make_md(tuned)
        md.build(x, box)
    for _ in range(args.warmup):
        md.run(x, v, box, DT_PS, args.md_steps, unroll=args.unroll)
    torch.cuda.synchronize(dev)
    th0 = md.thermo()
    clocks = Clocks(local)
    clocks.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for k in range(args.steps):
        flush.zero_()
        ev[k][0].record(stream)
        md.run(x, v, box, DT_PS, args.md_steps, unroll=args.unroll)
        ev[k][1].record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(ms))
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    th1 = md.thermo()
    builds = th1["builds"] - th0["builds"]
    prunes = th1["prunes"] - th0["prunes"]
    regrows = th1["regrows"] - th0["regrows"]
    stops = th1["redone"] - th0["redone"]
    ms_per_step = total_ms / args.steps
    value = ns_per_day(args.md_steps * args.steps * world, total_ms / 1e3)
    status = term.status(clear=True)
    temp = md.temperature()

    # ---- end to end through the public API, host buffers ---------------------
    # The equilibrated state of the device run goes to pinned host buffers;
    # each e2e step uploads it, runs md_steps through the public API and
    # reads the new positions and velocities back into the same buffers, so
    # that the steps chain through host memory like a checkpoint-restart
    # loop.  Each upload is a new state to the library: it tests the drift
    # from the lists' build on the device (mdrtMdRefresh) and keeps them when
    # they serve it, as they do for the state the last step read back.
    system = mdir.System.from_dict(s)
    system.pruned_distance = s["pruned"]
    hx = x.detach().cpu().pin_memory()
    hv = v.detach().cpu().pin_memory()
    st = mdir.InitialState(hx.numpy(), hv.numpy(), s["box"])
    integ, ens, exe, sch = mdir.Integrator(), mdir.Ensemble(), mdir.Execution(), mdir.Schedule()
    integ.timestep = DT_PS
    ens.kind, ens.temperature, ens.tau_t = mdir.EnsembleKind.NVT, 300.0, 0.1
    exe.device, exe.graph_steps = local, args.unroll
    exe.pair_sms = tuned["pair_sms"] if tuned else args.pair_sms
    exe.pair_blocks_per_sm = tuned["pair_blocks_per_sm"] if tuned else args.pair_blocks
    exe.fused_prune = tuned["fused_prune"] if tuned else 0
    exe.staging_depth = tuned["staging_depth"] if tuned else 1
    exe.pme_fft = args.pme_fft
    sim = mdir.Simulation(mdir.compile(system, st, integ, ens, exe, sch))

    def e2e_step():
        sim.set_state(hx, hv, non_blocking=True)
        sim.run(args.md_steps)
        hx.copy_(sim.x, non_blocking=True)
        hv.copy_(sim.v, non_blocking=True)
        torch.cuda.synchronize(dev)

    # warm-up: the first runs of a new context capture its step graph and may
    # grow its lists once ahead of need (a growth captures the graph again,
    # a few hundred ms once; 10 runs of 1,000 steps let the lists settle)
    for _ in range(max(10, args.warmup)):
        e2e_step()
    e_steps = max(3, args.steps)
    step_sec = []
    e2e_clocks = Clocks(local)
    e2e_clocks.start()
    time.sleep(0.3)
    t0 = time.perf_counter()
    for _ in range(e_steps):
        t1 = time.perf_counter()
        e2e_step()
        step_sec.append(time.perf_counter() - t1)
    e2e_sec = (time.perf_counter() - t0)
    e2e_clk = e2e_clocks.stop()
    if world > 1:
        t = torch.tensor([e2e_sec], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_sec = float(t.item())
    e2e = ns_per_day(args.md_steps * e_steps * world, e2e_sec)

    # ---- roofline of the dominant kernel (pair kernel), timed live ------------
    # on the whole GPU at its faster block count (the kernel alone), and at
    # the span the step uses (beside PME) for reference
    def stage_times():
        t_ = np.zeros(8)
        _lib.check(_lib.lib().mdrtNbTimeKernels(term._h, _dp(x), _hp(np.asarray(box, dtype=np.float64)), 200,
                                                _stream(), _hp(t_)), "mdrtNbTimeKernels")
        return t_
    step_shape = (term.pair_sms, term.pair_blocks_per_sm)
    step_times = stage_times()
    alone = []
    for blocks in (4, 3):
        term.set_tuning(pair_sms=0, pair_blocks_per_sm=blocks)
        alone.append((stage_times(), blocks))
    times, alone_blocks = min(alone, key=lambda tb: tb[0][1])
    term.set_tuning(pair_sms=step_shape[0], pair_blocks_per_sm=step_shape[1])
    pairs = count_pairs(x, box, s["cutoff"], s["excluded_pairs"])
    flop_per_pair = 50
    props = torch.cuda.get_device_properties(dev)
    sm_max = clk["sm_max_mhz"] or 1965.0
    peak_fp32 = props.multi_processor_count * 128 * 2 * sm_max * 1e6 / 1e12
    achieved = pairs * flop_per_pair / (times[1] * 1e-3) / 1e12
    roofline = {"bound": "fp32", "kernel": "nb_pairs", "achieved": round(achieved, 3),
                "peak": round(peak_fp32, 2), "unit": "TFLOP/s", "frac": round(achieved / peak_fp32, 4),
                "traffic": PAIRS_TRAFFIC_BYTES if args.waters == 7850 else None,
                "pairs_within_cutoff": pairs, "flop_per_pair": flop_per_pair,
                "pairs_per_s": round(pairs / (times[1] * 1e-3), 0),
                "launch_ms": round(times[1], 5),
                "launch_shape": {"sms": props.multi_processor_count, "blocks_per_sm": alone_blocks},
                "step_shape": {"sms": step_shape[0] or props.multi_processor_count,
                               "blocks_per_sm": step_shape[1], "launch_ms": round(step_times[1], 5)},
                "peak_note": "nominal FP32 = SMs x 128 x 2 x max SM clock (no measured FP32 peak exists)",
                "stage_ms": {"gather": round(times[0], 5), "pairs": round(times[1], 5),
                             "excluded": round(times[2], 5), "pme": round(times[3], 5),
                             "finish": round(times[4], 5)}}

    line = {"metric": METRIC, "value": round(value, 2), "unit": "ns/day", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 pairs / f64 sums (mixed)", "data": "synthetic (seeded TIP3P box, random orientations)",
            "config": config(args, s), "clocks": clk,
            "e2e": {"value": round(e2e, 2), "unit": "ns/day", "h2d_bytes_per_step": 2 * n * 3 * 8,
                    "d2h_bytes_per_step": 2 * n * 3 * 8 + 4, "steps": e_steps,
                    "median_step_ms": round(float(np.median(step_sec)) * 1e3, 3),
                    "max_step_ms": round(float(np.max(step_sec)) * 1e3, 3), "clocks": e2e_clk},
            "roofline": roofline,
            # this library's kernels per MD step: the gated pruning, spread,
            # spectrum scaling, pairs, update (cuFFT's own kernels not
            # counted), the noise once a graph of `unroll` steps, and 20 per
            # build (with the frames, the places and the references)
            "gpu_launches": int(args.steps * args.md_steps * 5 + args.steps * args.md_steps // max(1, args.unroll)
                                + builds * 20),
            "tuned": tuned,
            "tuning": {"reach_nm": s["reach"], "pruned_reach_nm": s["pruned"]},
            "per_replica_ns_day": round(value / world, 2),
            "builds": int(builds), "prunes": int(prunes), "regrows": int(regrows), "regrows_total": th1["regrows"],
            "stale_stops": int(stops),
            "temperature_K": round(temp, 1), "status": status}
    if not args.no_adjoint:
        line["adjoint"] = adjoint_leg(args, dev, flush, world)
    if not args.no_batch:
        line["batch"] = batch_leg(args, dev, flush, world, rank)
    if not args.no_precision and world == 1:
        line["precision"] = precision_leg(args, dev, flush, s["reach"], s["pruned"])
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(s, s["positions"])
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
