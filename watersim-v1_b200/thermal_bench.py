"""Whole frames of the bench planet with the thermal cycle on: sun at three
ocean radii on a 23.4-degree tilt, sunActivity 0.6, evapIntensity 0.05,
vorticity 0.05; 60 Hz frames (`step(1/60)`: substeps, contacts, phases,
rescue, and on tick frames the heat tick, evaporation and vapour contacts).

    python watersim-v1_b200/thermal_bench.py [--workload planet256] [--frames 30] [--warmup 3]

Frames are timed with CUDA events on the solver's stream; SM clocks and
throttle reasons are sampled during the timed frames. Then each frame pass is
timed alone (one call, events around it). Prints one JSON line.
"""
import argparse
import json
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.dirname(HERE))
import bench  # noqa: E402  (the benchmark planets and their knobs)

PASSES = ("HEAT", "EVAPORATION", "VAPOR_COLLISIONS", "PHASE", "ICE_CONTACTS", "PUSH_SURFACE")
TILT = math.radians(23.4)


def main():
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="planet256", choices=sorted(bench.WORKLOADS))
    ap.add_argument("--frames", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    a = ap.parse_args()
    bench.WORKLOAD = bench.WORKLOADS[a.workload]
    fs = bench.make_solver(0)
    c = fs.nx / 2
    R = fs.scalars.oceanR * 3
    fs.set_params(thermalOn=1, vorticity=0.05, sunActivity=0.6, evapIntensity=0.05,
                  sunPos=[c + R * math.cos(TILT), c + R * math.sin(TILT), c])
    for _ in range(a.warmup):
        fs.step(1 / 60)
    fs.synchronize()
    st = torch.cuda.ExternalStream(fs.stream())
    clocks = bench.Clocks(0)
    clocks.start()
    ms, subs, evap = [], 0, []
    for _ in range(a.frames):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fs.step(1 / 60)
        e1.record(st)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
        subs += fs.scalars.substepsLast
        evap.append(fs.scalars.evapCount)
    clk = clocks.stop()
    total_s = sum(ms) / 1000
    passes = {}
    for name in PASSES:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fs.stage(name, 1 / 25)
        e1.record(st)
        e1.synchronize()
        passes[name] = round(e0.elapsed_time(e1), 3)
    s = fs.scalars
    srt = sorted(ms)
    print(json.dumps({
        "workload": a.workload, "particles": s.nP, "frames": a.frames,
        "frames_per_s": a.frames / total_s, "substeps_per_s": subs / total_s,
        "substeps_per_frame": subs / a.frames,
        "frame_ms": {"min": srt[0], "median": srt[len(srt) // 2], "max": srt[-1]},
        "evaporations_last_tick": evap[-1], "vapor": s.vaporCount, "sor_iterations_last": s.sorIters,
        "pass_ms": passes, "clocks": clk}))


if __name__ == "__main__":
    main()
