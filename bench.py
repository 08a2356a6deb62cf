"""Benchmark: the AM-CFD transient melt-pool solve on B200.

Workload (one line per run): the 45-degree diagonal scan on a 400 x 200 x 100
non-uniform grid (8 M interior cells; P = 300 W, r = 60 um, v = 0.8 m/s,
dt = 5e-6 s, <= 20 SIMPLE outer iterations per step, tolerance 1e-5),
synthetic deck from am-cfd_b200/amcfd_decks.py.  A "step" is one time step of
the solver (updateLaser + iterativeLoopSolve + updateSolutions).

Window: --start-step S untimed steps carry the run into the steady melt pool
(the momentum box has stopped growing), then W warm-up steps, then the K timed
steps S+W+1 .. S+W+K.  Every figure on the line (the FP64 comparator, e2e and
the reference arm) is taken on that same window of the same deck.

value  = simulated milliseconds per wall second over the K timed steps (device
         time between CUDA events on the solver stream, max over ranks, all
         ranks' replicas counted); cell-iters/s alongside.
e2e    = the same metric through the C ABI (Solver.step() + the asynchronous
         read of the FP64 temperature field into pinned host memory every step,
         the clock stopped after the last copy landed) on a fresh solver over the
         same window.
fp64_redblack_* = the plain FP64 solve on the same production path (red-black
         order, graphs, device-driven outer loop), same window and tolerance.
Each rank (one per GPU) runs an independent replica of the single-domain case
("replicas only": the case does not shard).

--impl reference times the reference's own CPU solver (oracle/_ref, OpenMP on
all physical cores) on the same deck and the same window.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "am-cfd_b200"), os.path.join(ROOT, "oracle")]

METRIC = "sim-ms/wall-s"
# Algorithmic words per interior cell per outer iteration, by kernel family
# (energy path; the contract total is 92 words per cell per outer iteration).
# In red-black order the line factorisation runs inside the first sweep of each
# colour, so its 2 words belong to the sweep family.
WORDS = {"energy_assemble": 40, "factor": 2, "energy_sweeps": 40, "h2t_meltpool": 10}
WORDS_REDBLACK = {"energy_assemble": 40, "factor": 0, "energy_sweeps": 42, "h2t_meltpool": 10}
# DRAM bytes per interior cell per launch (ncu dram__bytes_read.sum +
# dram__bytes_write.sum, one capture of each kernel on the 400x200x100 deck,
# FP32 bulk); the line reports them scaled by the cell count.
# The red-black sweep family is one pipelined launch of the 8 passes per iteration
# ("pipe"), or with --pass-launch the average over the 8 per-pass launches (the first
# sweep of each colour also forms and stores the factorisation).
TRAFFIC_PER_CELL = {"energy_assemble:fp32:redblack": 87.0, "energy_sweeps:fp32:redblack": 21.2,
                    "energy_sweeps:fp32:redblack:pipe": 174.3,
                    "h2t_meltpool:fp32:redblack": 24.2, "energy_assemble:fp32dc:redblack": 146.2,
                    "energy_sweeps:fp32dc:redblack": 21.2}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            m = json.load(f)
        return float(m["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None
        self.skip = 0

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.f = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits", "-lms", "100"],
                                     stdout=self.f, stderr=subprocess.DEVNULL)
        # the timed region can be shorter than nvidia-smi's start-up: begin it only
        # once the sampler has written its first line (at most a few seconds)
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 5.0 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)
        with open(self.path) as f:
            self.skip = sum(1 for _ in f)  # samples taken before the timed region

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        with open(self.path) as f:
            lines = f.readlines()
        os.unlink(self.path)
        return parse_clock_samples(lines, self.skip)


def parse_clock_samples(lines, skip: int = 0):
    """Summary of nvidia-smi samples (rows of Clocks.Q, no header, no units): the
    median and maximum SM clock and the throttle reasons seen, over the rows after
    the first `skip` (those taken before the timed region; all rows when that
    leaves none); None without a parsable row."""
    sm, mx, reasons = [], 0.0, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    lines = lines[skip:] if len(lines) > skip else lines
    for line in lines:
        parts = [p.strip() for p in line.split(",")]
        if len(parts) < 9:
            continue
        try:
            sm.append(float(parts[1]))
            mx = max(mx, float(parts[2]))
        except ValueError:
            continue
        for n, v in zip(names, parts[5:9]):
            if v.lower() == "active":
                reasons.add(n)
    if not sm:
        return None
    sm.sort()
    return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons),
            "samples": len(sm)}


FEATURES = {
    "none": "",
    "species": "species equation (initial 1.0, D=5e-9 m^2/s, kp=0.3, urfc=0.7)",
    "powder": "powder bed: 2 layers of 10 cells, 40 um, powder at 90 % density, k=5 W/m/K",
    "moving": "moving mesh (middle x and y zones follow the beam) with G/R every step",
    "freesurf": "energy-balance free surface (timed separately: it runs before outputs)",
}


def make_deck(tmp: str, steps: int, config: str, feature: str = "none"):
    import amcfd_decks as D
    deck = {"config1": D.config1, "config0": D.config0, "config4": D.config4}[config](steps=steps)
    if feature == "species":
        deck.species = (1.0, 5e-9, 0.3, 0.7)
    elif feature == "powder":
        deck.powder = (2, 10, 40e-6, 0.9 * deck.material.dens, 1e-6, 500.0, 0.0, 5.0)
    elif feature == "moving":
        deck.moving_mesh = (2, 2)
        deck.solidification = True
    elif feature == "freesurf":
        deck.free_surface = (-1e5, 1e5, 1.8, 30, 1e-6, 40, 1e-18, 0.5)
    return deck, deck.write(tmp)


def physical_cores() -> int:
    """Physical cores of this host (logical CPUs when the count is unknown)."""
    try:
        import psutil
        n = psutil.cpu_count(logical=False)
        if n:
            return int(n)
    except Exception:
        pass
    return os.cpu_count() or 1


def reference_arm(skip: int, steps: int, config: str, threads: int, feature: str = "none"):
    """The reference CPU solver (oracle/_ref/amcfd_ref_dump --time, OpenMP) on the same
    deck: skip + steps time steps, the last `steps` of them timed."""
    import oracle_py
    exe = oracle_py.REF_DUMP
    if not os.path.exists(exe):
        return None, "reference binary oracle/_ref/amcfd_ref_dump not built"
    with tempfile.TemporaryDirectory() as tmp:
        deck, path = make_deck(tmp, skip + steps, config, feature)
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="spread", OMP_PLACES="cores")
        out = subprocess.run([exe, path, "--time", "--steps", str(skip + steps)], env=env,
                             capture_output=True, text=True, timeout=3600)
        if out.returncode != 0:
            return None, f"reference run failed: {out.stderr[-300:]}"
        js = json.loads(out.stdout.strip().splitlines()[-1])
    st = js["step_seconds"][skip:]
    it = js["step_iters"][skip:]
    secs = sum(st)
    ncell = js["interior_cells"]
    sim_ms = 1e3 * deck.dt * len(st)
    return {"value": sim_ms / secs, "cell_iters_per_s": ncell * sum(it) / secs, "seconds": secs,
            "steps": len(st), "outer_iters": sum(it), "threads": js["threads"],
            "ms_per_step": 1e3 * secs / max(len(st), 1)}, None


CONFIG_DESC = {
    "config1": ("diagonal 45-degree single track, 400x200x100 non-uniform cells (8.0 M), P=300 W, "
                "r=60 um, v=0.8 m/s, dt=5e-6 s, <=20 outer iterations/step, tolerance 1e-5"),
    "config0": "single track +x, 120x60x40 cells, P=200 W, dt=1e-5 s, <=20 outer iterations/step",
    "config4": ("2 layers x 5 tracks bidirectional raster (hatch 100 um, 1 ms dwell, 90-degree rotation), "
                "600x300x120 non-uniform cells (21.6 M), P=200 W, v=1.0 m/s, dt=1e-5 s, <=20 outer "
                "iterations/step, tolerance 1e-5"),
}
# untimed steps before the warm-up, by deck: config 1's momentum box stops growing
# by then; config 4's toolpath opens with a 1 ms (100-step) dwell with the beam off
START_STEP = {"config1": 60, "config0": 20, "config4": 130}


SWEEP_DESC = ("process-parameter sweep: 64 single-track instances, grids 60x30x20 .. 240x120x60 cells "
              "(domain scaled from the 120x60x40 deck), P ~ U[100,400] W, v ~ U[0.5,1.5] m/s, "
              "r ~ U[40,80] um (seeded), dt=1e-5 s, <=20 outer iterations/step, tolerance 1e-5")


def sweep_reference(decks, paths, skip: int, steps: int, cores: int):
    """The reference solver on the sweep: one process per instance (as the reference
    runs), OMP_NUM_THREADS=1, `cores` processes at a time; skip + steps steps each,
    the last `steps` timed; returns the aggregate over instances."""
    import oracle_py
    from concurrent.futures import ThreadPoolExecutor
    exe = oracle_py.REF_DUMP
    if not os.path.exists(exe):
        return None, "reference binary oracle/_ref/amcfd_ref_dump not built"

    def one(path):
        env = dict(os.environ, OMP_NUM_THREADS="1")
        out = subprocess.run([exe, path, "--time", "--steps", str(skip + steps)], env=env,
                             capture_output=True, text=True, timeout=3600)
        if out.returncode != 0:
            raise RuntimeError(out.stderr[-300:])
        return json.loads(out.stdout.strip().splitlines()[-1])

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=cores) as ex:
        res = list(ex.map(one, paths))
    wall = time.perf_counter() - t0
    # every process ran skip + steps steps; the timed share of the wall clock is the
    # timed steps' share of the summed step times
    tot = sum(sum(js["step_seconds"]) for js in res)
    timed = sum(sum(js["step_seconds"][skip:]) for js in res)
    wall_timed = wall * timed / max(tot, 1e-30)
    sim_ms = sum(1e3 * d.dt * steps for d in decks)
    cells_iters = sum(js["interior_cells"] * sum(js["step_iters"][skip:]) for js in res)
    return {"value": sim_ms / wall_timed, "cell_iters_per_s": cells_iters / wall_timed, "seconds": wall_timed,
            "processes": cores}, None


def sweep_main(args):
    """The config-2 sweep: every rank solves its longest-processing-time shard of the
    64 instances; each instance is a context with its own stream and step graph, a
    pool of host threads keeps them in flight (amcfd_run_batch).  value = simulated
    ms of all instances / wall s of the slowest rank."""
    import amcfd_decks as D
    import amcfd_sweep as SW
    warmup = max(3, args.warmup)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cores = physical_cores()
    tmp = tempfile.mkdtemp(prefix=f"amcfd_sweep{rank}_")
    decks = D.config2(steps=warmup + args.steps + 1)
    paths = [dk.write(os.path.join(tmp, dk.name)) for dk in decks]
    cfg = {"workload": SWEEP_DESC, "deck": "config2", "instances": len(decks),
           "window": f"steps {warmup + 1}-{warmup + args.steps} of every instance after {warmup} warm-up steps",
           "timing": "host wall clock around the batch (device synchronised before and after); every "
                     "instance runs on its own stream"}
    if args.impl == "reference":
        if rank != 0:
            return
        r, why = sweep_reference(decks, paths, warmup, args.steps, cores)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": r["value"], "unit": METRIC,
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": warmup,
                          "ms_per_step": 1e3 * r["seconds"] / args.steps, "higher_is_better": True,
                          "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic decks",
                          "config": dict(cfg, solver="reference build (oracle/_ref), one process per instance"),
                          "cell_iters_per_s": r["cell_iters_per_s"],
                          "cpu_baseline": {"value": r["value"], "unit": METRIC, "cores": r["processes"],
                                           "kind": "reference", "sample": cfg["window"]},
                          "e2e": {"value": r["value"], "unit": METRIC, "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        shutil.rmtree(tmp, ignore_errors=True)
        return
    import torch
    import amcfd
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    prec = {"fp32": amcfd.PREC_FP32, "fp32dc": amcfd.PREC_FP32_DC, "fp64": amcfd.PREC_FP64}[args.precision]
    costs = [SW.instance_cost(amcfd.Deck(p).dims, args.steps) for p in paths]
    mine = SW.shard(costs, world)[rank]
    dk = [amcfd.Deck(paths[q]) for q in mine]
    solvers = [amcfd.Solver(d, order=amcfd.ORDER_REDBLACK, precision=prec, device=local, use_graphs=1,
                            autotune=1) for d in dk]
    amcfd.run_batch(solvers, warmup)
    it0 = [s.report.itertot for s in solvers]

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    clocks = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    l0 = sum(s.launches for s in solvers)
    t0 = time.perf_counter()
    reps, _ = amcfd.run_batch(solvers, args.steps)
    torch.cuda.synchronize()
    secs = time.perf_counter() - t0
    ck = clocks.stop()
    launches = sum(s.launches for s in solvers) - l0
    cells_iters = sum((d.dims[0] - 2) * (d.dims[1] - 2) * (d.dims[2] - 2) * (r["itertot"] - i)
                      for d, r, i in zip(dk, reps, it0))
    sim_ms = sum(1e3 * decks[q].dt * args.steps for q in mine)
    tot = torch.tensor([secs, sim_ms, cells_iters, launches], dtype=torch.float64, device=f"cuda:{local}")
    if world > 1:
        mx = tot[:1].clone()
        torch.distributed.all_reduce(mx, op=torch.distributed.ReduceOp.MAX)
        sm_ = tot[1:].clone()
        torch.distributed.all_reduce(sm_, op=torch.distributed.ReduceOp.SUM)
        secs, (sim_ms, cells_iters, launches) = float(mx.item()), sm_.tolist()
    for s in solvers:
        s.close()
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": sim_ms / secs, "unit": METRIC, "n_gpus": world,
                          "steps": args.steps, "warmup": warmup, "ms_per_step": 1e3 * secs / args.steps,
                          "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
                          "dtype": {amcfd.PREC_FP32: "f32", amcfd.PREC_FP32_DC: "f64 (energy line solves f32 "
                                    "on the correction)", amcfd.PREC_FP64: "f64"}[prec],
                          "data": "synthetic decks",
                          "config": dict(cfg, precision=args.precision, order="redblack", graphs=1,
                                         parallelism=f"instance shards over {world} GPU(s)"),
                          "cell_iters_per_s": cells_iters / secs, "gpu_launches": int(launches),
                          "clocks": ck,
                          "e2e": {"value": sim_ms / secs, "unit": METRIC, "h2d_bytes_per_step": 52 * len(decks),
                                  "d2h_bytes_per_step": 512 * len(decks),
                                  "note": "the batch call is the public API; per step every instance copies "
                                          "its laser block in and its status block out"}}))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    shutil.rmtree(tmp, ignore_errors=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--start-step", type=int, default=None,
                    help="untimed steps before the warm-up (default: per deck, into the steady melt pool)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp32dc", "fp64"],
                    help="fp32: FP32 bulk with FP64 reductions; fp32dc: FP64 fields with the energy line "
                         "solves in FP32 on the correction (defect correction); fp64: plain FP64")
    ap.add_argument("--order", default="redblack", choices=["redblack", "exact"])
    ap.add_argument("--config", default="config1", choices=sorted(CONFIG_DESC))
    ap.add_argument("--graphs", type=int, default=1, choices=[0, 1],
                    help="replay each outer iteration from a CUDA graph")
    ap.add_argument("--host-loop", action="store_true",
                    help="with graphs, one graph per outer iteration and the convergence test on the "
                         "host (default: one graph per step, iterations chained on the device)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-threads", type=int, default=0,
                    help="OpenMP threads of the reference CPU solver (0: every physical core)")
    ap.add_argument("--no-compare", action="store_true", help="skip the plain FP64 comparison run")
    ap.add_argument("--no-small-box", action="store_true",
                    help="momentum boxes of every size on the grid path (no one-CTA path)")
    ap.add_argument("--small-box", action="store_true",
                    help="the one-CTA momentum chain whenever the box fits its shared memory")
    ap.add_argument("--serial-launch", action="store_true",
                    help="no programmatic dependent launch; the box line solve as a launch per colour pass")
    ap.add_argument("--pass-launch", action="store_true",
                    help="the whole-domain red-black line sweeps as a launch per pass (not pipelined)")
    ap.add_argument("--mom-cluster", type=int, default=0, choices=[0, 1, 2, 4, 8, 16],
                    help="CTAs of the cluster momentum solve (1: none, 0: the library default)")
    ap.add_argument("--profile-window", action="store_true",
                    help="bracket the timed steps with cudaProfilerStart/Stop, so that "
                         "ncu --profile-from-start off captures those launches only")
    ap.add_argument("--feature", default="none", choices=sorted(FEATURES),
                    help="solve the deck with one of the optional models switched on")
    ap.add_argument("--workload", default="track", choices=["track", "sweep"],
                    help="track: one melt-pool instance per GPU (--config); sweep: the 64-instance "
                         "process-parameter sweep, sharded over the GPUs")
    args = ap.parse_args()
    if args.workload == "sweep":
        return sweep_main(args)
    warmup = max(3, args.warmup)
    start = START_STEP[args.config] if args.start_step is None else max(0, args.start_step)
    skip = start + warmup  # steps before the timed window
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    cores = args.ref_threads if args.ref_threads > 0 else physical_cores()
    window = f"steps {skip + 1}-{skip + args.steps} (after {start} untimed steps and {warmup} warm-up steps)"
    cfg_desc = {"workload": CONFIG_DESC[args.config], "deck": args.config, "window": window,
                "l2": "working set 1.2-6.4 GB > 126 MB L2 (no flush needed)"}
    if args.feature != "none":
        cfg_desc["feature"] = FEATURES[args.feature]

    if args.impl == "reference":
        if rank != 0:
            return
        r, why = reference_arm(skip, args.steps, args.config, cores, args.feature)
        if r is None:
            print(json.dumps({"impl": "reference", "unavailable": why}))
            return
        line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": METRIC,
                "n_gpus": args.gpus, "steps": r["steps"], "warmup": warmup,
                "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic deck",
                "config": dict(cfg_desc, solver="reference OpenMP build (oracle/_ref)"),
                "cell_iters_per_s": r["cell_iters_per_s"], "outer_iters": r["outer_iters"],
                "cpu_baseline": {"value": r["value"], "unit": METRIC, "cores": r["threads"],
                                 "kind": "reference", "logical_cpus": os.cpu_count(),
                                 "sample": f"the timed window ({window}) of the same deck, "
                                           f"OpenMP on {r['threads']} of {physical_cores()} physical cores"},
                "e2e": {"value": r["value"], "unit": METRIC, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import numpy as np
    import torch
    import amcfd

    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = local
    torch.cuda.set_device(dev)
    prec = {"fp32": amcfd.PREC_FP32, "fp32dc": amcfd.PREC_FP32_DC, "fp64": amcfd.PREC_FP64}[args.precision]
    order = amcfd.ORDER_REDBLACK if args.order == "redblack" else amcfd.ORDER_EXACT
    tmp = tempfile.mkdtemp(prefix=f"amcfd_bench{rank}_")
    total_steps = skip + 2 * args.steps + 2
    deck, path = make_deck(tmp, total_steps, args.config, args.feature)
    d = amcfd.Deck(path)
    ni, nj, nk = d.dims
    ncell = (ni - 2) * (nj - 2) * (nk - 2)

    tune = {}

    def solver(p=prec):
        # the production path tunes its launch shapes at creation; later solvers of the
        # same precision are pinned to the first one's assembly and sweep shapes (the
        # pipelined sweep's stride, which changes no bits, is tuned again)
        kw = dict(autotune=1 if order == amcfd.ORDER_REDBLACK else 0)
        if p in tune:
            kw.update(asm_kseg=tune[p]["asm_kseg"], sweep_warps=tune[p]["sweep_warps"])
        small = 0 if args.no_small_box else (1 if args.small_box else None)
        sv = amcfd.Solver(d, order=order, precision=p, device=dev, use_graphs=args.graphs,
                          host_loop=1 if args.host_loop else 0, mom_cluster=args.mom_cluster,
                          small_box=small, serial_launch=1 if args.serial_launch else 0,
                          pass_launch=1 if args.pass_launch else 0, **kw)
        tune.setdefault(p, sv.tuning())
        return sv

    s = solver()
    s.run_steps(skip)

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def allmax(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{dev}")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    # the timed steps run the production path (no per-phase events: with graphs,
    # one graph per step and the outer iterations chained on the device)
    clocks = Clocks(dev)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    l0 = s.launches
    it0 = s.report.itertot
    if args.profile_window:
        torch.cuda.cudart().cudaProfilerStart()
    rep, ms = s.run_steps(args.steps)
    if args.profile_window:
        torch.cuda.synchronize()
        torch.cuda.cudart().cudaProfilerStop()
    launches = s.launches - l0
    iters = rep["itertot"] - it0
    torch.cuda.synchronize()
    barrier()
    ck = clocks.stop()
    ms = allmax(ms)
    # the per-phase split: the next steps, with CUDA events around each phase
    # (the host drives those iterations), per outer iteration
    s.profile(True)
    s.run_steps(args.steps)
    prof = s.timing()
    s.profile(False)
    torch.cuda.synchronize()
    s.close()
    value = world * 1e3 * deck.dt * args.steps / (ms / 1e3)
    cips = world * ncell * iters / (ms / 1e3)

    # end to end on a fresh solver over the same window: per step, laser block in,
    # report + temperature field out (pinned).  Each step's field is packed on the
    # device at once and copied to the host while the next step computes; the clock
    # stops after the last copy landed.
    se = solver()
    se.run_steps(skip)
    host = torch.empty(ni * nj * nk, dtype=torch.float64, pin_memory=True)
    se.get_into_async("temp", host.data_ptr())  # warm-up: the copy stream is made on first use
    se.wait_reads()
    boxes = []
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r = se.step()
        se.get_into_async("temp", host.data_ptr())
        boxes.append(r["momentum_cells"])
    se.wait_reads()
    t1 = time.perf_counter()
    barrier()
    se.close()
    e2e_s = allmax(t1 - t0)
    e2e = {"value": world * 1e3 * deck.dt * args.steps / e2e_s, "unit": METRIC,
           "h2d_bytes_per_step": 52, "d2h_bytes_per_step": int(ni * nj * nk * 8 + 512)}

    # roofline of the dominant kernel family
    peak, peak_kind = _peaks()
    words = WORDS_REDBLACK if args.order == "redblack" else WORDS
    # bytes per word of each family: FP32 bulk, FP64, or defect correction (FP64 fields,
    # FP32 coefficients and correction in the line sweeps)
    wsize = {f: (4 if prec == amcfd.PREC_FP32 or (prec == amcfd.PREC_FP32_DC and f in ("energy_sweeps", "factor"))
                 else 8) for f in words}
    fam = max(words, key=lambda k: prof[k])
    w = wsize[fam]
    # the sweep family is 8 (red-black) or 1 (exact order) launches per iteration
    piters = prof["outer_iters"]  # outer iterations of the profiling steps
    nlaunch = prof["sweep_launches"] if fam == "energy_sweeps" else piters
    avg_ms = prof[fam] / max(nlaunch, 1)
    alg_bytes = words[fam] * ncell * w * piters / max(nlaunch, 1)
    achieved = alg_bytes / (avg_ms / 1e3) / 1e9
    pipe = ":pipe" if fam == "energy_sweeps" and args.order == "redblack" and nlaunch <= piters else ""
    tr = TRAFFIC_PER_CELL.get(f"{fam}:{args.precision}:{args.order}{pipe}")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind, "kernel": fam,
                "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_ms,
                "traffic": tr * ncell if tr else None,
                "iteration_frac": (sum(words[f] * wsize[f] for f in words) * ncell * iters / (ms / 1e3) / 1e9) / peak}

    extra = {"momentum_box_cells": {"mean": float(np.mean(boxes)), "min": int(min(boxes)),
                                    "max": int(max(boxes))},
             "tuning": tune[prec]}
    if args.feature == "freesurf":
        # one free-surface update (bisection + projection) on a fresh state; the call
        # returns after its kernels and the read-back of the monitor values
        sf = solver()
        sf.run_steps(2)
        sf.free_surface()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fs = sf.free_surface()
        extra["free_surface_ms"] = 1e3 * (time.perf_counter() - t0)
        extra["free_surface"] = fs
        sf.close()
    if not args.no_compare and rank == 0 and prec != amcfd.PREC_FP64:
        # the plain FP64 solve on the same production path and the same window
        s64 = solver(amcfd.PREC_FP64)
        s64.run_steps(skip)
        i64 = s64.report.itertot
        r64, ms64 = s64.run_steps(args.steps)
        v64 = 1e3 * deck.dt * args.steps / (ms64 / 1e3)
        extra["fp64_redblack_sim_ms_per_wall_s"] = v64
        extra["fp64_redblack_cell_iters_per_s"] = ncell * (r64["itertot"] - i64) / (ms64 / 1e3)
        extra["fp64_redblack_outer_iters"] = r64["itertot"] - i64
        extra["speedup_vs_fp64_redblack"] = (value / world) / v64
        s64.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # a bounded sample: the first steps of the same deck (the reference arm,
        # a separate run, times the full window)
        r, why = reference_arm(0, 3, args.config, cores, args.feature)
        if r is not None:
            cpu = {"value": r["value"], "unit": METRIC, "cores": r["threads"], "kind": "reference",
                   "logical_cpus": os.cpu_count(),
                   "sample": f"steps 1-{r['steps']} of the same deck, OpenMP build of the reference "
                             f"on {r['threads']} physical cores",
                   "cell_iters_per_s": r["cell_iters_per_s"]}
        else:
            cpu = {"value": None, "unit": METRIC, "cores": cores, "kind": "reference",
                   "sample": why}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
                "steps": args.steps, "warmup": warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": {amcfd.PREC_FP32: "f32", amcfd.PREC_FP32_DC: "f64 (energy line solves f32 on the correction)",
                          amcfd.PREC_FP64: "f64"}[prec], "data": "synthetic deck",
                "config": dict(cfg_desc, precision=args.precision, order=args.order, graphs=args.graphs,
                               outer_loop="host" if args.host_loop or not args.graphs else "device",
                               momentum=("grid" if args.no_small_box else "one-CTA below its capacity, else grid"
                                         if args.small_box else "cooperative box solve"
                                         " (one-CTA chain only where that is unavailable)")
                               + (", serial launches" if args.serial_launch else ""),
                               sweeps="a launch per pass" if args.pass_launch or args.serial_launch
                               else "the 8 passes of a solve in one pipelined launch",
                               parallelism=f"replicas{world}"),
                "cell_iters_per_s": cips, "outer_iters": iters, "gpu_launches": launches,
                "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": ck,
                "phase_ms": {k: v for k, v in prof.items() if k not in ("outer_iters", "sweep_launches")},
                "phase_outer_iters": prof["outer_iters"]}
        line.update(extra)
        print(json.dumps(line))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    shutil.rmtree(tmp, ignore_errors=True)


if __name__ == "__main__":
    main()
