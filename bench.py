"""Throughput of the WaterSim FLIP/MAC substep on B200.

Workload (the 128^3 planet of the headline metric): 128^3 MAC grid, unit
cells, sea-level radius 52 and ocean depth 8 (core radius 44), seeded
value-noise terrain (seed 20260114), targetParticles 2,000,000 (the
reference's fill knob; ~24 per water cell with this terrain), FLIP
with pic 0.05, red-black SOR (omega 1.7) to a 1e-5 relative residual checked
every 10 iterations, speed clamp 3.2 m/s, full planet gravity, thermal cycle
off, and the seeded Gaussian stir kick (sigma 4 cells, 2 m/s peak) every 50
substeps. One bench step = one substep of dt = 0.01 (the reference's
step(1/60) runs two such substeps).

Learned warm start (the metric's comparison): after the plain solver's
timed run, the same planet keeps running while every solve stores its
(input, converged pressure) pair (2000 pairs), the 3-level U-Net is trained
on them with Adam (lr 1e-3, batch 4), its output scale is calibrated on
eight fresh systems (1, 1/2 or 1/4 of the predicted correction, whichever
leaves SOR the fewest iterations), and the same substep is timed again with
every solve starting from the network's prediction. Both arms solve to
the same 1e-5 relative residual. `value` is the learned arm's substeps/s;
the plain arm's figure, SOR iterations of both, the residual left by the
prediction and the training and inference times are reported beside it.

Arms
  default            the CUDA library through the C ABI (watersim-v1_b200)
  --impl reference   the reference's CPU algorithm: the C restatement of
                     js/solver.js in oracle/ (no JavaScript engine exists on
                     the machine), reference order (lexicographic SOR),
                     single-threaded like solver.js, same workload.

Multi-GPU: the substep does not shard, so N GPUs run N independent replicas
(weak scaling); value = substeps completed by all ranks / max-rank time.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "watersim-v1_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

WORKLOADS = {
    "planet128": dict(name="planet128", n=128, R=52.0, depth=8.0, seed=20260114, particles=2000000,
                      levels=3, pairs=2000),
    # the large planet: 256^3, radius 110, ocean 12 deep, ~16M particles; its
    # warm start is the 4-level U-Net (16/32/64/128) trained on 1000 pairs
    "planet256": dict(name="planet256", n=256, R=110.0, depth=12.0, seed=20260114, particles=16000000,
                      levels=4, pairs=1000),
    # the 64^3 planet with the thermal cycle on: radius 26, ocean 5 deep, 220k particles; whole
    # 60 Hz frames (two substeps each, SOR to 1e-5, vorticity 0.05) make one bench step
    "planet64": dict(name="planet64", n=64, R=26.0, depth=5.0, seed=20260114, particles=220000),
}
# the thermal cycle of the frame workloads: sun at three ocean radii on a 23.4-degree
# axial tilt, sunActivity 0.6, evapIntensity 0.05, vorticity confinement 0.05
THERMAL = dict(thermalOn=1, vorticity=0.05, sunActivity=0.6, evapIntensity=0.05)
FRAME_PASSES = ("HEAT", "EVAPORATION", "VAPOR_COLLISIONS", "PHASE", "ICE_CONTACTS", "PUSH_SURFACE")
WORKLOAD = WORKLOADS["planet128"]
PARAMS = dict(pic=0.05, omega=1.7, maxSpeed=3.2, cfl=3.0, viscosity=5e-4, thermalOn=0,
              sorTol=1e-5, sorCheckEvery=10, sorMaxIters=5000, pressureIters=40)
DT = 0.01
STIR_EVERY, STIR_SIGMA, STIR_PEAK = 50, 4.0, 2.0
METRIC = "substeps/s @128^3/2M particles: learned warm-start vs plain SOR at equal \u2016\u2207\u00b7u\u2016"
METRIC_PLAIN = "substeps/s @128^3/2M particles (plain red-black SOR to 1e-5 relative divergence residual)"
# the fields the JS drop-in's _pull reads back after every step (and uploads once)
E2E_FIELDS = ("px", "py", "pz", "pvx", "pvy", "pvz", "pT", "pflag", "pLight", "pDepth")
U8_FIELDS = ("pflag", "pcool", "pDepth")


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.rows, self.proc = index, [], None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 7 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 7 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 7 for i in range(4)
                          if r[4 + i].lower() in ("active", "1")})
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


def reduce_max(value, device):
    """Max of a per-rank float over all ranks (the device-time rule for N > 1)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def make_solver(device, rank=0):
    """The bench planet through the library's own terrain generator and fill.
    Replicas (rank > 0) draw their stir kicks from their own seed."""
    from fluid_solver import FluidSolver
    W = WORKLOAD
    coreR = W["R"] - W["depth"]
    fs = FluidSolver(nx=W["n"], ny=W["n"], nz=W["n"], dx=1.0, coreR=coreR, terrainSeed=W["seed"],
                     targetParticles=float(W["particles"]), capacity=W["particles"] + 8192, device=device)
    fs.generateTerrain(W["seed"], W["R"])
    fs.resetWater(W["depth"])
    fs.set_params(**PARAMS)
    fs.set_scalars(gRamp=1.5)
    if rank > 0:
        fs.set_scalars(stirS=(0x2545f491 + 7919 * rank) & 0xffffffff)
    return fs


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local_rank)
    fs = make_solver(local_rank, rank)
    nP = fs.scalars.nP
    stream = torch.cuda.ExternalStream(fs.stream())
    count = [0]

    def one_step():
        if count[0] % STIR_EVERY == 0:
            fs.stir_gaussian(STIR_SIGMA, STIR_PEAK)
        fs._substep(DT)
        count[0] += 1

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed_region():
        """K substeps with inputs in HBM, device-timed on the library stream,
        max over ranks; nvidia-smi clocks sampled during the region."""
        barrier()
        clk = Clocks(local_rank)
        clk.start()
        time.sleep(0.5)                  # first samples land before the timed region
        l0 = fs.launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            one_step()                   # asynchronous: no host sync inside the timed region
        e1.record(stream)
        e1.synchronize()
        barrier()
        clocks = clk.stop()
        launches = fs.launch_count() - l0
        ms = e0.elapsed_time(e1)
        if world > 1:
            ms = reduce_max(ms, "cuda")
        return ms, clocks, launches

    def from_start():
        """Back to the state both arms start from (the captured substep graph
        survives: the restored terrain is the same)."""
        fs.restore(start)
        count[0] = count0

    def iterations():
        """SOR iterations of each timed substep: the same K substeps replayed
        from the start state, read back one by one."""
        from_start()
        its = []
        for _ in range(args.steps):
            one_step()
            its.append(fs.scalars.sorIters)
        return its

    for _ in range(args.warmup):
        one_step()
    # Both arms are timed over the same K substeps from one saved state.
    start, count0 = fs.snapshot(), count[0]
    # ---- plain SOR arm
    from_start()
    ms, clocks, launches = timed_region()
    iters0 = iterations()
    plain = {"substeps_per_s": args.steps * world / (ms / 1000.0), "ms_per_step": ms / args.steps,
             "sor_iterations": sum(iters0) / len(iters0), "clocks": clocks}
    ms_plain = ms
    # ---- learned warm-start arm
    learned = None
    if not args.no_learned:
        learned = learned_arm(fs, one_step, args, world)
        from_start()
        one_step()                       # captures the substep graph with the prediction in it
        from_start()
        ms, clocks, launches = timed_region()
        iters1 = iterations()
        learned["sor_iterations"] = sum(iters1) / len(iters1)
        learned["substeps_per_s"] = args.steps * world / (ms / 1000.0)
        learned["ms_per_step"] = ms / args.steps
        learned["same_start_as_plain"] = True
        qsave = fs.download("q")
        learned["inference_ms"] = fs.unet_time(0, 10)   # applies the prediction repeatedly: restore q after
        fs.upload("q", qsave)
    value = args.steps * world / (ms / 1000.0)
    # ---- end to end through the public API with pinned host buffers
    host = {k: torch.empty(nP, dtype=torch.uint8 if k in U8_FIELDS else torch.float32).pin_memory().numpy()
            for k in E2E_FIELDS}
    fs.download_state(host, nP)
    e2e_steps = max(1, min(args.steps, 20))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        fs.upload_state(host, nP)        # this step's particle state from pinned host buffers
        one_step()
        fs.download_state(host, nP)      # and the stepped state back into them
    barrier()
    e2e_s = time.perf_counter() - t0
    if world > 1:
        e2e_s = reduce_max(e2e_s, "cuda")
    bytes_io = sum(host[k].nbytes for k in E2E_FIELDS)
    # ---- roofline of the dominant kernel, timed live on the library stream
    roof = roofline(fs, ms_plain / args.steps, iters0)
    surface = surface_timing(fs, cpu=(rank == 0 and not args.no_cpu_baseline))
    render = render_timing(fs, cpu=(rank == 0 and not args.no_cpu_baseline))
    metaballs = metaball_timing(fs, cpu=(rank == 0 and not args.no_cpu_baseline))
    fp64 = fp64_errors(fs) if (rank == 0 and not args.no_cpu_baseline) else None
    balls = ball_timing(fs, one_step)
    out = None
    if rank == 0:
        cfg_learned = {}
        if learned:
            cfg_learned = {"plain_substeps_per_s": plain["substeps_per_s"],
                           "learned_vs_plain": learned["substeps_per_s"] / plain["substeps_per_s"],
                           "warm_start": learned, "plain": plain}
        out = {"metric": METRIC if learned else METRIC_PLAIN, "value": value, "unit": "substeps/s", "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic seeded planet (value-noise terrain, jittered lattice fill)",
               "config": workload_config(nP, world),
               "details": {"arm": "learned warm start" if learned else "plain SOR",
                           "sor": "red-black to 1e-5 (check every %d), mean iterations %.1f"
                                  % (PARAMS["sorCheckEvery"], (learned or plain)["sor_iterations"]),
                           "fluid_cells": fs.scalars.nFluid,
                           "sor_path": SOR_PATHS.get(fs.scalars.sorPath, "unknown"),
                           "particle_substeps_per_s": value * nP,
                           "surface_mesh": surface,
                           "render_particles": render,
                           "metaballs": metaballs,
                           "fp64_field_errors": fp64,
                           "balls": balls,
                           **cfg_learned},
               "e2e": {"value": e2e_steps * world / e2e_s, "unit": "substeps/s",
                       "h2d_bytes_per_step": bytes_io, "d2h_bytes_per_step": bytes_io},
               "gpu_launches": int(launches),
               "roofline": roof,
               "clocks": clocks}
    return out, fs


SOR_PATHS = {0: "none", 1: "grid-wide persistent (colour lists)", 2: "cluster-resident (DSMEM, colour lists)",
             3: "temporal-blocked (every SM, shared-memory regions)",
             4: "owned bricks in global memory (every SM, a grid barrier per half-sweep)"}
SOR_KERNELS = {1: "k_sor_persistent", 2: "k_sor_cluster", 3: "k_sor_tb", 4: "k_sor_tb"}


def workload_config(nP, world):
    """The workload both arms run (identical dict on both arms' lines)."""
    W = WORKLOAD
    n = W["n"]
    return {"workload": "%s: %d^3 MAC grid, R=%g, depth %g, %d particles" % (W["name"], n, W["R"], W["depth"], nP),
            "particles": nP, "parallelism": "replicas x%d" % world,
            "l2": ("state (~%d MB) larger than L2 (126 MB)" if not state_fits_l2(n, nP)
                   else "state (~%d MB) fits in L2 (126 MB): a 256 MB buffer is written between timed steps")
                  % state_mb(n, nP)}


L2_BYTES = 126 * 1000 * 1000


def state_fits_l2(n, nP):
    return state_mb(n, nP) * 1e6 < L2_BYTES


def state_mb(n, nP):
    F = 3 * (n + 1) * n * n
    return int((nP * 55 + F * 21 + n ** 3 * 16) / 1e6)


def learned_arm(fs, one_step, args, world=1):
    """Record (input, converged q) pairs from the plain solves, train the
    U-Net on them, and measure what its prediction leaves for SOR on fresh
    pressure systems. Leaves the warm start enabled."""
    fs.unet_init(7, WORKLOAD.get("levels", 3))
    fs.unet_collect(args.pairs)
    t0 = time.perf_counter()
    for _ in range(args.pairs):
        one_step()
    fs.synchronize()
    collect_s = time.perf_counter() - t0
    fs.unet_collect(0)
    t0 = time.perf_counter()
    if world > 1:
        # one network for all replicas: gradients summed over the ranks each step
        import dp_train
        dp_train.agree_gain(fs)
        loss0 = dp_train.train_data_parallel(fs, 10, 4, 1e-3, 1)
        loss1 = dp_train.train_data_parallel(fs, args.train_steps, 4, 1e-3, 2)
    else:
        loss0 = fs.unet_train(10, 4, 1e-3, 1)
        loss1 = fs.unet_train(args.train_steps, 4, 1e-3, 2)
    fs.synchronize()
    train_s = time.perf_counter() - t0
    # fresh pressure systems: iterations from the previous q and from the
    # prediction (check every iteration), and the residual each start leaves.
    # The prediction's output scale is calibrated here: each system is solved
    # from q_prev + a * (the prediction's correction) for a in SCALES, and the
    # scale with the fewest iterations over the systems (ties: the larger) is
    # kept for the timed arm. a = 1 is the network as trained.
    keep = (fs.sorCheckEvery,)
    fs.sorCheckEvery = 1
    g0 = fs.unet_info()["gain"]
    SCALES = (1.0, 0.5, 0.25)
    rows, by_scale = [], {a: [] for a in SCALES}
    for k in range(8):
        for st in ("CLEAR_RASTER", "MARK_FLUID", "P2G", "FORCES"):
            fs.stage(st, DT)
        qprev = fs.download("q")
        res = {}
        for a in SCALES:
            fs.upload("q", qprev)
            fs.unet_set_gain(g0 * a)
            res[a] = fs.unet_probe()
            fs.stage("PRESSURE", DT)
            by_scale[a].append(fs.scalars.sorIters)
        fs.upload("q", qprev)
        fs.stage("PRESSURE", DT)
        it_p = fs.scalars.sorIters
        rows.append((it_p, res))
        for st in ("PROJECT", "EXTRAPOLATE", "G2P_ADVECT"):
            fs.stage(st, DT)
    fs.sorCheckEvery = keep[0]
    mean = {a: sum(v) / len(v) for a, v in by_scale.items()}
    best = min(SCALES, key=lambda a: (mean[a], -a))
    fs.unet_set_gain(g0 * best)
    fs.unet_enable(True)
    n = len(rows)
    info = fs.unet_info()
    return {"levels": WORKLOAD.get("levels", 3), "pairs": info["pairs_stored"], "pairs_requested": args.pairs,
            "collect_s": collect_s, "train_steps": args.train_steps + 10, "batch": 4 * world,
            "training": "data-parallel over %d ranks (gradients all-reduced)" % world if world > 1 else "one GPU",
            "lr": 1e-3, "train_s": train_s, "loss_first": loss0, "loss_last": loss1,
            "train_ms_per_sample": fs.unet_time(1, 3),
            "output_scale": best,
            "probe_iterations_by_scale": {str(a): mean[a] for a in SCALES},
            "probe_iterations_plain": sum(r[0] for r in rows) / n,
            "probe_iterations_learned": mean[best],
            "probe_iterations_learned_unscaled": mean[1.0],
            "probe_relres_previous_q": sum(r[1][1.0][0] for r in rows) / n,
            "probe_relres_predicted": sum(r[1][best][1] for r in rows) / n}


def active_bricks(fs):
    """4^3 bricks within one brick of a particle's cell (the substep's work
    list, less the bricks kept for one substep after they empty)."""
    import numpy as np
    n = fs.nx
    nb = (n + 3) // 4
    nP = fs.scalars.nP
    ijk = [np.clip(np.floor(fs.download(k, nP) / fs.dx).astype(np.int64), 0, n - 1) // 4 for k in ("px", "py", "pz")]
    seed = np.zeros((nb, nb, nb), bool)
    seed[ijk[2], ijk[1], ijk[0]] = True
    act = np.zeros_like(seed)
    p = np.pad(seed, 1)
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                act |= p[dz:dz + nb, dy:dy + nb, dx:dx + nb]
    return int(act.sum())


def roofline(fs, ms_step, iters):
    """Dominant kernel by measured time share per substep; achieved =
    algorithmic bytes per launch / live launch time (CUDA events on the
    library's stream, ws_time_kernel)."""
    peak, kind = _peaks()
    n = fs.nx
    N = n ** 3
    F = 3 * (n + 1) * n * n
    s = fs.scalars
    nP, nF = s.nP, s.nFluid
    it = max(1, int(round(sum(iters) / max(1, len(iters)))))
    keep = fs.pressureIters
    fs.pressureIters = it
    us_sor = fs.time_kernel(6, 5)                 # whole solve of `it` iterations
    fs.pressureIters = keep
    # the face passes as the substep runs them: over the active-brick list of
    # the last substep (ids 8-11); their bytes count the faces of those bricks
    us_f1 = fs.time_kernel(8, 5)
    us_f2 = fs.time_kernel(9, 5)
    us_pr = fs.time_kernel(10, 5)
    us_ex = fs.time_kernel(11, 5)
    Fa = 192.0 * active_bricks(fs)
    # P2G as the substep runs it by default: particle index order, runs of up
    # to four consecutive particles per atomic (id 1); the cell-ordered variant (id 12: counting
    # sort, prefix sum, scatter of particle ids, shared-memory sums per brick,
    # every brick visited) beside it
    us_p2g = fs.time_kernel(1, 5)
    us_p2g_cell = fs.time_kernel(12, 5)
    us_g2p = fs.time_kernel(2, 5)
    step_us = ms_step * 1000
    # algorithmic bytes per launch (each input read once, each output written once):
    #  SOR solve     13 B per fluid cell per iteration (q read, rhs, stencil byte, q write)
    #  P2G           25 B per particle in + 8 B per face accumulator
    #  G2P+advect    52 B per particle + 8 B per face (u and uO)
    #  faces pass 1  8 B acc + 9 B out per face; forces 12 B per face; project 8 B per face;
    #                extrapolation 5 B per face (flag + value), all over the active bricks' faces
    # the path the timed solve took (its own diagnostics, read after it ran)
    sor_name = SOR_KERNELS.get(fs.scalars.sorPath, "k_sor_tb")
    cand = {sor_name: (us_sor, 13.0 * nF * it),
            "k_p2g_runs": (us_p2g, 25.0 * nP + 8.0 * F),
            "k_g2p_advect": (us_g2p, 52.0 * nP + 8.0 * F),
            "k_faces_bricks<normalize_bc>": (us_f1, 17.0 * Fa),
            "k_faces_bricks<forces>": (us_f2, 12.0 * Fa),
            "k_faces_bricks<project>": (us_pr, 8.0 * Fa),
            "k_faces_bricks<extrapolate>": (us_ex, 5.0 * Fa)}
    name = max(cand, key=lambda k: cand[k][0])
    us, nbytes = cand[name]
    achieved = nbytes / (us * 1e-6) / 1e9
    # DRAM bytes (read + write) per launch from one ncu capture of each kernel
    # on this 128^3 planet: the temporal-blocked solve loads its system into
    # shared memory once and iterates from there (halo exchanges hit L2), so
    # its traffic hardly depends on the iteration count
    captured = {"k_sor_tb": (17864496.0, "ncu dram__bytes_read.sum + dram__bytes_write.sum of one 60-iteration "
                                         "solve of this planet (bench.py --profile 3); the system is read once, "
                                         "the iterations run from shared memory and L2"),
                "k_g2p_advect": (65502208.0, "ncu dram__bytes_read.sum + dram__bytes_write.sum, one capture at 128^3")}
    traffic, note = captured.get(name, (None, None)) if WORKLOAD["name"] == "planet128" else (None, None)
    return {"kernel": name, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": kind, "traffic": traffic, "traffic_note": note,
            "bytes_per_launch": nbytes, "us_per_launch": us, "time_share": us / step_us,
            "others": {k: {"us_per_launch": v[0], "time_share": v[0] / step_us,
                           "GB_s": v[1] / (v[0] * 1e-6) / 1e9} for k, v in cand.items()},
            "p2g_cell_order_us": us_p2g_cell}


def surface_timing(fs, cpu=True):
    """MarchingTetrahedra.build of the splatted density (iso = the solver's
    iso): device time through ws_surface_mesh (5 calls, the last timed alone
    after warm-up), and the oracle's single-threaded CPU build of the same
    field for comparison."""
    import ctypes as C
    fs.stage("SPLAT")
    iso = fs.scalars.iso
    n, vol = C.c_int64(), C.c_double()
    for _ in range(2):
        fs._check(fs._L.ws_surface_mesh(fs._h, float(iso), C.byref(n), C.byref(vol)))
    t0 = time.perf_counter()
    for _ in range(5):
        fs._check(fs._L.ws_surface_mesh(fs._h, float(iso), C.byref(n), C.byref(vol)))
    gpu_ms = (time.perf_counter() - t0) / 5 * 1000
    out = {"iso": iso, "vertices": n.value, "volume": vol.value, "gpu_ms_per_build": gpu_ms}
    if cpu:
        from oracle.oracle import mt_mesh_field
        dens = fs.download("dens")
        t0 = time.perf_counter()
        mt_mesh_field(dens, fs.nx, fs.ny, fs.nz, 1.0, iso)
        out["cpu_oracle_ms_per_build"] = (time.perf_counter() - t0) * 1000
    return out


def ball_timing(fs, one_step, steps=50):
    """The ball coupling's cost: substeps/s of the same planet with eight
    balls (addBall; four light floaters at the sea surface, four heavy
    sinkers) against the same number of substeps without, each run of n
    substeps timed on the host between two stream synchronisations. Runs
    last: the balls move particles."""
    import numpy as np

    def timed(n):
        fs.synchronize()
        t0 = time.perf_counter()
        for _ in range(n):
            one_step()
        fs.synchronize()
        return (time.perf_counter() - t0) / n * 1000

    base = timed(steps)
    iters_base = fs.scalars.sorIters
    s = fs.scalars
    c = fs.nx * fs.dx / 2
    r = np.random.default_rng(9)
    for i in range(8):
        v = r.normal(size=3)
        v /= np.linalg.norm(v)
        R = s.oceanR if i < 4 else s.oceanR - 3.0
        fs.add_ball(*(c + v * R), 2.0, 500.0 if i < 4 else 2500.0)
    for _ in range(3):
        one_step()
    with_balls = timed(steps)
    iters_balls = fs.scalars.sorIters
    b = fs.balls
    fs.set_balls(np.zeros((0, 9)))
    return {"balls": 8, "ms_per_substep_without": base, "ms_per_substep_with": with_balls,
            "overhead_ms": with_balls - base, "sor_iterations_last_without": iters_base,
            "sor_iterations_last_with": iters_balls, "submerged": [round(float(x), 3) for x in b[:, 8]]}


def metaball_timing(fs, cpu=True):
    """Metaballs.build(solver, 0.5) of the stepped particles (the app's
    default tension and detail): device time per ws_metaball_mesh call (field
    splat, float rounding, marching-tets volume and emission; 5 calls after 2
    warm-up), and the oracle's single-threaded field + mesh on the same
    particles."""
    import ctypes as C
    n, vol = C.c_int64(), C.c_double()
    for _ in range(2):
        fs._check(fs._L.ws_metaball_mesh(fs._h, 0.5, float("nan"), C.byref(n), C.byref(vol)))
    t0 = time.perf_counter()
    for _ in range(5):
        fs._check(fs._L.ws_metaball_mesh(fs._h, 0.5, float("nan"), C.byref(n), C.byref(vol)))
    out = {"tension": 0.5, "vertices": n.value, "volume": vol.value,
           "gpu_ms_per_build": (time.perf_counter() - t0) / 5 * 1000}
    if cpu:
        from oracle.oracle import metaball_field, mt_mesh_field
        nP = fs.scalars.nP
        f = {k: fs.download(k, nP) for k in ("px", "py", "pz", "pflag")}
        t0 = time.perf_counter()
        field, m, mdx, iso, _ = metaball_field(f["px"], f["py"], f["pz"], f["pflag"], fs.nx, fs.dx,
                                               fs.scalars.spacing, 0.5)
        mt_mesh_field(field, m, m, m, mdx, iso)
        out["cpu_oracle_ms_per_build"] = (time.perf_counter() - t0) * 1000
    return out


def render_timing(fs, cpu=True):
    """WaterScene.updateParticles of the stepped particles (beads mode, lit
    planet, camera two box widths out, so every class draws and the sort
    spreads over all 64 buckets): time per ws_render_particles call (4 kernels
    + the 20-byte count read-back, 5 calls after 2 warm-up), its algorithmic
    bytes (26 read per particle: position, flag, temperature, exposure, depth,
    spin phase; 36 written per drawn point) over that time against the
    measured HBM peak, and the oracle's single-threaded CPU pass on the same
    particles."""
    from fluid_solver import render_opts
    W = fs.nx * fs.dx
    opts = render_opts(beadsMode=1, cam=(0.5 * W, 0.5 * W, -2.0 * W), sunDir=(0.6, 0.0, 0.8))
    for _ in range(2):
        counts, pts = fs.render_particles(opts, download=False)
    t0 = time.perf_counter()
    for _ in range(5):
        counts, pts = fs.render_particles(opts, download=False)
    ms = (time.perf_counter() - t0) / 5 * 1000
    nP = fs.scalars.nP
    algo = 26 * nP + 36 * pts
    peak, kind = _peaks()
    out = {"particles": nP, "points": pts, "counts": counts, "gpu_ms_per_call": ms,
           "algorithmic_bytes": algo, "achieved_gbs": algo / (ms * 1e6), "frac_of_hbm": algo / (ms * 1e6) / peak,
           "peak_source": kind}
    if cpu:
        from oracle.render_oracle import render_particles
        f = {k: fs.download(k, nP) for k in ("px", "py", "pz", "pflag", "pT", "pLight", "pDepth", "pPh",
                                             "pWx", "pWy", "pWz")}
        center = (0.5 * W, 0.5 * fs.ny * fs.dx, 0.5 * fs.nz * fs.dx)
        t0 = time.perf_counter()
        render_particles(opts, center, fs.scalars.spacing, fs._p.spinOn, f)
        out["cpu_oracle_ms_per_call"] = (time.perf_counter() - t0) * 1000
    return out


def oracle_from_device(fs, fp64=False):
    """An oracle holding the device's current planet: terrain, particles, q and
    scalars (fp64: the FP64-storage flavour)."""
    from oracle.oracle import Oracle
    s = fs.scalars
    nP = s.nP
    t = fs.terrain()
    W = WORKLOAD
    coreR = W["R"] - W["depth"]
    o = Oracle(fs.nx, fs.ny, fs.nz, 1.0, coreR=coreR, terrainSeed=W["seed"], targetParticles=s.targetParticles,
               fp64=fp64)
    depthW = W["depth"]
    Rlo = max(coreR * 0.55, W["R"] - 1.8889 * depthW)
    o.load_terrain({"n": t["n"], "dv": 0.5, "solid": t["solid"], "R": t["R"], "Rsl": W["R"],
                    "Rlo": Rlo, "Rhi": W["R"] + 0.7778 * depthW, "landFrac": t["landFrac"]})
    o.alloc_particles(nP + 8192)
    for k in ("px", "py", "pz", "pvx", "pvy", "pvz", "pT", "pAir", "pflag", "pcool"):
        o.arr(k)[:nP] = fs.download(k)
    o.arr("q")[:] = fs.q
    o.set_scalars(nP=nP, oceanR=s.oceanR, spacing=s.spacing, particleVolume=s.particleVolume,
                  gRamp=1.5, dtLast=DT, umax=s.umax)
    o.L.or_build_planet_gravity(o.h)
    return o


def fp64_errors(fs):
    """Error of each field of one substep against the FP64 oracle of the same
    substep: the device state is copied into the FP64-storage oracle (device
    order: red-black SOR, Jacobi viscosity and extrapolation), both take one
    substep of DT from it (warm start off), and each field's relative error is
    reported as max |gpu - fp64| / max |fp64| and as the L2 ratio."""
    import numpy as np
    try:
        warm = fs.unet_info()["enabled"]
    except Exception:                     # no network on this handle (plain arm only)
        warm = 0
    if warm:
        fs.unet_enable(0)
    o = oracle_from_device(fs, fp64=True)
    o.set(**{k: v for k, v in PARAMS.items()}, sorRedBlack=1, viscJacobi=1, extrapJacobi=1)
    t0 = time.perf_counter()
    o.substep(DT)
    cpu_s = time.perf_counter() - t0
    fs._substep(DT)
    fs.synchronize()
    nP = fs.scalars.nP
    out = {"oracle": "FP64 storage and arithmetic, device order", "substep_dt": DT,
           "sor_iterations": {"gpu": fs.scalars.sorIters, "fp64": o.scalars.sorIters}, "fp64_cpu_s": cpu_s}

    def err(a, b):
        a = np.asarray(a, np.float64)
        b = np.asarray(b, np.float64)
        den = np.max(np.abs(b))
        return {"linf_rel": float(np.max(np.abs(a - b)) / den) if den > 0 else 0.0,
                "l2_rel": float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))}
    out["q"] = err(fs.q, o.q)
    for k in ("u", "v", "w"):
        out[k] = err(fs.download(k), o.arr(k))
    for k in ("pvx", "pvy", "pvz"):
        out[k] = err(fs.download(k, nP), o.arr(k)[:nP])
    W = fs.nx * fs.dx
    out["positions_max_abs_over_width"] = float(max(
        np.max(np.abs(fs.download(k, nP).astype(np.float64) - o.arr(k)[:nP])) for k in ("px", "py", "pz")) / W)
    out["cell_types_differing"] = int(np.count_nonzero(fs.cellType != o.cellType))
    if warm:
        fs.unet_enable(1)
    return out


def cpu_baseline(fs, seconds=20.0):
    """The oracle (CPU restatement, reference order) on this exact planet, one
    core, a bounded sample of whole substeps."""
    s = fs.scalars
    nP = s.nP
    W = WORKLOAD
    o = oracle_from_device(fs)
    o.set(**{k: v for k, v in PARAMS.items()}, sorRedBlack=0, viscJacobi=0, extrapJacobi=0)
    done, t0 = 0, time.perf_counter()
    while True:
        o.substep(DT)
        done += 1
        el = time.perf_counter() - t0
        if el >= seconds or done >= 20:
            break
    return {"value": done / el, "unit": "substeps/s", "cores": 1, "kind": "port",
            "sample": ("%d whole substep(s) of the %d^3 planet (%d particles) in %.1f s, oracle "
                       "(C restatement of js/solver.js, lexicographic SOR) on 1 host core" % (done, W["n"], nP, el))}


def frames_metric(n, nP):
    return ("substeps/s @%d^3/%dk particles, thermal cycle on (whole 60 Hz frames, plain SOR to 1e-5)"
            % (n, nP // 1000))


def run_reference(args, rank, world, frames=False):
    """Reference arm: the CPU algorithm of js/solver.js (oracle port), one
    core, on the same workload, --steps timed steps after --warmup untimed
    ones (substeps, or whole frames with the thermal cycle on)."""
    if rank != 0:
        return None
    from oracle.oracle import make_planet
    W = WORKLOAD
    o = make_planet(W["n"], R=W["R"], depth=W["depth"], seed=W["seed"], particles=W["particles"])
    o.set(**PARAMS, sorRedBlack=0, viscJacobi=0, extrapJacobi=0)
    o.set_scalars(gRamp=1.5)
    nP = o.nP
    if frames:
        c = W["n"] / 2
        R = o.scalars.oceanR * 3
        tilt = math.radians(23.4)
        o.set(**THERMAL, sunPos=[c + R * math.cos(tilt), c + R * math.sin(tilt), c])
    count = [0]

    def one():
        if frames:
            o.step(1 / 60)
            return o.scalars.substepsLast
        if count[0] % STIR_EVERY == 0:
            o.stir_gaussian(STIR_SIGMA, STIR_PEAK)
        o.substep(DT)
        count[0] += 1
        return 1
    for _ in range(args.warmup):
        one()
    t0 = time.perf_counter()
    subs = sum(one() for _ in range(args.steps))
    el = time.perf_counter() - t0
    v = subs / el
    unit = "whole frame(s)" if frames else "whole substep(s)"
    sample = ("%d %s of the %d^3 planet (%d particles) after %d warm-up; C restatement of js/solver.js "
              "(reference order), 1 core: the reference's step is single-threaded; no JavaScript engine on the "
              "host" % (args.steps, unit, W["n"], nP, args.warmup))
    metric = frames_metric(W["n"], nP) if frames else (METRIC_PLAIN if args.no_learned else METRIC)
    return {"metric": metric, "value": v, "unit": "substeps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64 arithmetic / f32 storage",
            "data": "synthetic seeded planet (value-noise terrain, jittered lattice fill)", "impl": "reference",
            "config": workload_config(nP, world),
            "cpu_baseline": {"value": v, "unit": "substeps/s", "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "substeps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def thermal_on(fs):
    """The thermal cycle of the frame workloads on this solver."""
    c = fs.nx / 2
    R = fs.scalars.oceanR * 3
    tilt = math.radians(23.4)
    fs.set_params(**THERMAL, sunPos=[c + R * math.cos(tilt), c + R * math.sin(tilt), c])


def run_frames(args, rank, world, local_rank):
    """Whole 60 Hz frames (step(1/60): substeps, contacts, phases, rescue,
    and on tick frames the heat tick, evaporation and vapour contacts) with
    the thermal cycle on. One bench step = one frame; value = substeps/s.
    Frames are timed with CUDA events on the solver's stream (max over
    ranks); each frame pass is then timed alone once."""
    import torch
    torch.cuda.set_device(local_rank)
    fs = make_solver(local_rank, rank)
    thermal_on(fs)
    for _ in range(args.warmup):
        fs.step(1 / 60)
    fs.synchronize()
    st = torch.cuda.ExternalStream(fs.stream())
    clocks = Clocks(local_rank)
    clocks.start()
    time.sleep(0.5)
    ms, subs, evap = [], 0, []
    launches = 0
    # a state that fits in L2 is evicted between timed frames by writing a
    # buffer twice the L2 size on the solver's stream, outside the events
    flush = (torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device="cuda")
             if state_fits_l2(WORKLOAD["n"], fs.scalars.nP) else None)
    for _ in range(args.steps):
        if flush is not None:
            with torch.cuda.stream(st):
                flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = fs.launch_count()
        e0.record(st)
        fs.step(1 / 60)                  # synchronous: returns after the frame's counters are read
        e1.record(st)
        launches += fs.launch_count() - l0
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        subs += fs.scalars.substepsLast
        evap.append(fs.scalars.evapCount)
    clk = clocks.stop()
    total = sum(ms)
    if world > 1:
        total = reduce_max(total, "cuda")
    passes = {}
    for name in FRAME_PASSES:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fs.stage(name, 1 / 25)
        e1.record(st)
        e1.synchronize()
        passes[name] = round(e0.elapsed_time(e1), 3)
    s = fs.scalars
    srt = sorted(ms)
    out = None
    if rank == 0:
        out = {"metric": frames_metric(WORKLOAD["n"], s.nP),
               "value": subs * world / (total / 1000), "unit": "substeps/s", "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
               "data": "synthetic seeded planet (value-noise terrain, jittered lattice fill)",
               "config": workload_config(s.nP, world),
               "details": {"frames_per_s": args.steps * world / (total / 1000),
                           "substeps_per_frame": subs / args.steps,
                           "frame_ms": {"min": srt[0], "median": srt[len(srt) // 2], "max": srt[-1]},
                           "evaporations_last_tick": evap[-1], "vapor": s.vaporCount,
                           "sor_iterations_last": s.sorIters, "sor_path": SOR_PATHS.get(s.sorPath, "unknown"),
                           "pass_ms": passes},
               "gpu_launches": int(launches), "clocks": clk}
    return out, fs


def run_profile(args, local_rank):
    """A few substeps of the workload for capturing one kernel under a
    profiler with few launches before it (no timing). With --learned-profile
    two (input, converged q) pairs are recorded, one Adam step taken and the
    warm start turned on, so the network's convolutions run every substep."""
    import torch
    torch.cuda.set_device(local_rank)
    fs = make_solver(local_rank)
    if WORKLOAD["name"] == "planet64":
        thermal_on(fs)
    if args.learned_profile:
        fs.unet_init(7, WORKLOAD.get("levels", 3))
        fs.unet_collect(2)
        fs._substep(DT)
        fs._substep(DT)
        fs.unet_collect(0)
        fs.unet_train(1, 1, 1e-3, 1)
        fs.unet_enable(1)
    for _ in range(args.profile):
        fs._substep(DT)
    fs.synchronize()
    s = fs.scalars
    print(json.dumps({"profile_substeps": args.profile, "workload": WORKLOAD["name"], "learned": bool(args.learned_profile),
                      "sor_iterations": s.sorIters, "fluid_cells": s.nFluid,
                      "sor_path": SOR_PATHS.get(s.sorPath, "unknown")}))
    fs.close()


def run_render(args, local_rank):
    """ws_render_particles (WaterScene.updateParticles, js/scene.js:1595-1922)
    on seeded particles shaped like the 128^3 planet's: 1,856,640 particles
    over a 128^3 box in cell order, liquid only (or all six flag classes with
    --render-mix), the lit-planet scene in beads mode with the camera two box
    widths out. Time per call (four kernels, count read-back, synchronisation)
    and the algorithmic bytes per second (26 read per particle, 36 written
    per drawn point)."""
    import numpy as np
    import torch
    from fluid_solver import FluidSolver, render_opts
    torch.cuda.set_device(local_rank)
    n, W = 1856640, 128.0
    r = np.random.default_rng(3)
    px, py, pz = (r.uniform(0, W, n).astype(np.float32) for _ in range(3))
    o = np.lexsort((px, py, pz))
    flags = r.integers(0, 6, n) if args.render_mix else np.zeros(n)
    parts = {"px": px[o], "py": py[o], "pz": pz[o], "pflag": flags.astype(np.uint8),
             "pT": r.uniform(0, 1, n).astype(np.float32), "pLight": r.uniform(0, 1, n).astype(np.float32),
             "pDepth": r.integers(0, 5, n).astype(np.uint8), "pPh": r.uniform(-3, 3, n).astype(np.float32)}
    fs = FluidSolver(nx=128, ny=128, nz=128, dx=1.0, coreR=40, targetParticles=1000, capacity=n + 64,
                     device=local_rank)
    fs.set_scalars(nP=n)
    fs.upload_state(parts, count=n)
    opts = render_opts(beadsMode=1, cam=(0.5 * W, 0.5 * W, -2.0 * W), sunDir=(0.6, 0.0, 0.8))
    for _ in range(max(3, args.warmup)):
        fs.render_particles(opts, download=False)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        counts, pts = fs.render_particles(opts, download=False)
    ms = (time.perf_counter() - t0) / args.steps * 1000
    algo = 26 * n + 36 * pts
    print(json.dumps({"render_particles": n, "points": pts, "counts": counts, "mix": bool(args.render_mix),
                      "ms_per_call": ms, "algorithmic_bytes": algo, "achieved_gbs": algo / (ms * 1e6)}))
    fs.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="plain SOR arm only")
    ap.add_argument("--pairs", type=int, default=None,
                    help="training pairs recorded from plain solves (default: 2000 at 128^3, 1000 at 256^3)")
    ap.add_argument("--train-steps", type=int, default=1000, help="Adam steps of batch 4")
    ap.add_argument("--levels", type=int, default=None, choices=[3, 4],
                    help="U-Net depth (default: 3 at 128^3, 4 at 256^3)")
    ap.add_argument("--workload", default="planet128", choices=sorted(WORKLOADS),
                    help="planet64 runs whole thermal-cycle frames; planet256 the plain and learned arms at 256^3")
    ap.add_argument("--frames", action="store_true", help="whole frames with the thermal cycle on (any workload)")
    ap.add_argument("--profile", type=int, default=0, help="run this many substeps for a profiler capture and exit")
    ap.add_argument("--learned-profile", action="store_true", help="--profile with the learned warm start on")
    ap.add_argument("--render", action="store_true", help="time ws_render_particles alone and exit")
    ap.add_argument("--render-mix", action="store_true", help="--render with all six flag classes")
    args = ap.parse_args()
    global WORKLOAD, METRIC, METRIC_PLAIN
    WORKLOAD = WORKLOADS[args.workload]
    if args.pairs is None:
        args.pairs = WORKLOAD.get("pairs", 2000)
    if args.levels is not None:
        WORKLOAD = dict(WORKLOAD, levels=args.levels)
    if args.workload == "planet64":
        args.no_learned = True
    if args.workload != "planet128":
        METRIC_PLAIN = ("substeps/s @%d^3/%dM particles (plain red-black SOR to 1e-5 relative divergence residual)"
                        % (WORKLOAD["n"], WORKLOAD["particles"] // 1000000))
        METRIC = ("substeps/s @%d^3/%dM particles: learned warm-start (%d-level U-Net) vs plain SOR at equal "
                  "\u2016\u2207\u00b7u\u2016" % (WORKLOAD["n"], WORKLOAD["particles"] // 1000000, WORKLOAD.get("levels", 3)))
    frames = args.frames or args.workload == "planet64"
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        out = run_reference(args, rank, world, frames)
        if out is not None:
            print(json.dumps(out))
        return
    if args.profile:
        return run_profile(args, local_rank)
    if args.render:
        return run_render(args, local_rank)
    import torch
    import datetime
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    out, fs = (run_frames if frames else run_ours)(args, rank, world, local_rank)
    if rank == 0:
        if not args.no_cpu_baseline and not frames:
            out["cpu_baseline"] = cpu_baseline(fs, args.cpu_seconds)
        print(json.dumps(out))
    fs.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
