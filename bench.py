#!/usr/bin/env python
"""Throughput of the batched 3DMM video fit (fitted frames/s) on B200.

Workload "cap53k_video": the seeded synthetic morphable model with the shapes of the
reference's full-size model (53,490 vertices, 106,466 triangles, 79 expression components),
a batch of video frames (AR(1) expressions, random-walk head pose, face boxes 120-600 px in
1080p) rescaled to the reference's 256x256 crop, fitted per frame as
VideoFitter::fit_to_video_frame does after its landmark initialisation: light fit, then the
log-barrier Gauss-Newton shape fit (pose + 79 expressions) capped at 20 outer iterations.

One step = one fit of the whole batch. ``value`` times ``tdi_batch_fit`` with every input
resident in device memory; ``e2e`` times ``tdi_fit_frames`` from pinned host buffers
(host->device copy of the frames and states, the fit, and the read-back of states and reports).
Inputs (256 MB of target crops for 1,024 frames) exceed the 126 MB L2 between steps.

``--impl reference`` times the CPU restatement of the same path (oracle/, OpenMP over frames,
all host threads) on a bounded sample of the same frames: 3DI cannot be built here (it needs
OpenCV) and has no CPU path of its own.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "cap53k_video"
MAX_ITERS = 20
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12
METRIC = "fitted frames/s (batched video fit, 53,490-vertex model, 256x256 crop)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=1024, help="frames per GPU per step")
    ap.add_argument("--cpu-frames", type=int, default=8, help="frames of the CPU sample")
    ap.add_argument("--profile-kernel", default="vertex",
                    help="kernel timed live for the roofline (the largest share of the step)")
    ap.add_argument("--plain-frames", type=int, default=16, help="frames of the unbatched (plain) run")
    ap.add_argument("--normal-eq", default="exact", choices=["exact", "tensor"],
                    help="normal equations: FP64 in the oracle's order, or split-BF16 on the tensor cores")
    return ap.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_workload(synth, n_frames, seed_offset=0):
    """One rank's shard: its own seeded frames (rank r passes seed_offset = 100 r), so ranks
    fit disjoint frames with no exchange."""
    return synth.make_workload(WORKLOAD, n_frames, seed_offset)


def max_over_ranks(values, world, device="cpu"):
    """The job's clock: every rank's device times (ms), reduced with MAX over the ranks."""
    import torch
    import torch.distributed as dist
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def job_rate(frames_per_rank, world, steps, ms):
    """Whole-job fitted frames/s: every rank's frames over the slowest rank's time."""
    return frames_per_rank * world * steps / (ms / 1000.0)


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            if len(r) < 9:
                continue
            for name, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return p.get("hbm_gbs", 6650.0), p.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def algorithmic_bytes(kernel: str, V: int, T: int, K: int, n_frag: float):
    """(bytes per frame, bytes per launch) a kernel must move: what the roofline divides by."""
    if kernel == "vertex":
        # outputs per frame (object coordinates 12 B, projection x, y, Z 12 B per vertex) and
        # the coefficients; the basis (3*V*K*4 B) once per launch, shared by all its frames.
        # The stored records are two float4 per vertex (32 B): padding and the albedo copy
        # are not counted as algorithmic bytes.
        return 24.0 * V + 4.0 * K, 12.0 * V * K
    if kernel == "raster":
        # depth pass: projections (16 B per vertex), triangle corners and visiting order
        # (16 B per triangle), one 8-byte depth key per visible fragment
        return 16.0 * V + 16.0 * T + 8.0 * n_frag, 0.0
    if kernel == "render":
        # fragments, three vertices' object coordinates and albedo, four target pixels, gradients
        return n_frag * (16 + 3 * 16 + 4 * 4 + 5 * 4), 0.0
    if kernel == "jacobian":
        # three vertices' basis rows (3 coords x K) and the row written
        return n_frag * (3 * 3 * K * 4 + (K + 6) * 4), 0.0
    raise ValueError(kernel)


def vertex_flops_per_frame(V: int, K: int) -> float:
    """Fused multiply-adds of the basis x coefficient products, 2 flops each."""
    return 2.0 * 3 * V * K


def cpu_fit_rate(O, synth, m, fr, n_frames, threads):
    """Frames/s of the oracle (FP32 restatement) on the first n_frames frames."""
    om = O.Model(m)
    fs = O.FrameSet(fr, 0, n_frames)
    cfg = O.config(max_iters_rigid=MAX_ITERS)
    lam = np.tile(synth.LAMBDA_INIT, (n_frames, 1))
    L = np.full(n_frames, synth.L_INTENSITY, np.float32)
    t0 = time.perf_counter()
    O.fit_frames(om, fs, cfg, fr.state_init[:n_frames], lam, L, threads=threads)
    return n_frames / (time.perf_counter() - t0)


def reference_arm(args, world, rank):
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    synth = importlib.import_module("3di_b200.synth")
    O.build()
    n = args.cpu_frames
    m, fr = make_workload(synth, n)
    render_targets_cpu(O, synth, m, fr)
    threads = O.max_threads()
    rates = []
    for _ in range(args.warmup if args.warmup < 1 else 1):
        cpu_fit_rate(O, synth, m, fr, n, threads)
    for _ in range(args.steps):
        rates.append(cpu_fit_rate(O, synth, m, fr, n, threads))
    v = statistics.median(rates)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "frames/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": n / v * 1000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "frames_per_step": n, "max_outer_iters": MAX_ITERS,
                   "l2": "inputs larger than L2 are not applicable on the CPU"},
        "cpu_baseline": {"value": v, "unit": "frames/s", "cores": threads, "kind": "port",
                         "sample": f"{n} frames of {WORKLOAD}, FP32 CPU restatement (oracle/), "
                                   "3DI itself needs OpenCV and cannot be built"},
        "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def render_targets_cpu(O, synth, m, fr):
    om = O.Model(m)
    cfg = O.config()
    imgs = [O.render_target(om, fr, i, cfg, fr.state_true[i], fr.lam_true[i], synth.L_INTENSITY)[0]
            for i in range(fr.n_frames)]
    fr.target = synth.add_noise(np.stack(imgs), 0.02, 3)


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        return reference_arm(args, world, rank)

    import torch
    import torch.distributed as dist
    tdi = importlib.import_module("3di_b200")
    synth = importlib.import_module("3di_b200.synth")
    tdi.require_gpu()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))

    F = args.frames
    m, fr = make_workload(synth, F, seed_offset=100 * rank)
    model = tdi.Model(m)
    batch = tdi.Batch(model, F)
    # synthetic photos: the library renders the true states, noise is added on the host
    lam_true = fr.lam_true
    L = np.full(F, synth.L_INTENSITY, np.float32)
    fr.target = np.zeros((F, tdi.NPIX), np.float32)
    batch.set_frames(fr)
    batch.set_state(fr.state_true, lam_true, L)
    img, _ = batch.render()
    fr.target = synth.add_noise(img, 0.02, 3 + rank)
    batch.set_frames(fr)
    lam0 = np.tile(synth.LAMBDA_INIT, (F, 1)).astype(np.float32)
    cfg = tdi.default_config(max_iters_rigid=MAX_ITERS,
                             normal_eq=tdi.NORMAL_EQ_TENSOR if args.normal_eq == "tensor" else tdi.NORMAL_EQ_EXACT)

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up
    for _ in range(args.warmup):
        batch.set_state(fr.state_init, lam0, L)
        batch.fit(cfg)
    torch.cuda.synchronize()

    # timed: device-resident inputs
    clocks = ClockSampler(local)
    clocks.start()
    batch.profile(args.profile_kernel)
    launches0 = batch.launches()
    total_ms = 0.0
    for _ in range(args.steps):
        batch.set_state(fr.state_init, lam0, L)      # reset the fitted states (not timed)
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        batch.fit(cfg)
        e1.record()
        torch.cuda.synchronize()
        barrier()
        total_ms += e0.elapsed_time(e1)
    launches = batch.launches() - launches0
    prof_launches, prof_ms, prof_frames = batch.profile_read()
    batch.profile(None)
    clk = clocks.stop()
    x, lamf, rep = batch.get_state()
    n_frag = float(np.mean([r.n_fragments for r in rep]))

    # timed: end to end from pinned host memory through tdi_fit_frames
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    h = dict(t=pin(fr.target.astype(np.float32)), xl=pin(fr.xl), yl=pin(fr.yl), b=pin(fr.bounds),
             fs=pin(fr.face_size), cam=pin(fr.cam), o=pin(fr.x0y0.astype(np.int32)),
             x=pin(fr.state_init), lam=pin(lam0), L=pin(L))
    desc = tdi.FramesDesc(F, *[h[k].data_ptr() for k in ("t", "xl", "yl", "b", "fs", "cam", "o")])
    reps = (tdi.Report * F)()
    lib = tdi.load_library()
    import ctypes as C
    e2e_ms = 0.0
    for _ in range(args.steps):
        xs = h["x"].clone().pin_memory()
        ls = h["lam"].clone().pin_memory()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        st = lib.tdi_fit_frames(batch.handle, C.byref(desc), C.byref(cfg), C.c_void_p(xs.data_ptr()),
                                C.c_void_p(ls.data_ptr()), C.c_void_p(h["L"].data_ptr()), reps, None)
        e1.record()
        torch.cuda.synchronize()
        barrier()
        if st != 0:
            raise tdi.TdiError(lib.tdi_last_error().decode())
        e2e_ms += e0.elapsed_time(e1)
    # the other normal-equation mode on the same batch, device-resident, same step count
    other = "tensor" if args.normal_eq == "exact" else "exact"
    cfg_o = tdi.default_config(max_iters_rigid=MAX_ITERS,
                               normal_eq=tdi.NORMAL_EQ_TENSOR if other == "tensor" else tdi.NORMAL_EQ_EXACT)
    batch.set_state(fr.state_init, lam0, L)
    batch.fit(cfg_o)
    other_ms = 0.0
    for _ in range(args.steps):
        batch.set_state(fr.state_init, lam0, L)
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        batch.fit(cfg_o)
        e1.record()
        torch.cuda.synchronize()
        barrier()
        other_ms += e0.elapsed_time(e1)
    xo_gpu, _, rep_o = batch.get_state()
    h2d = sum(h[k].numel() * h[k].element_size() for k in ("t", "xl", "yl", "b", "fs", "cam", "o", "x", "lam", "L"))
    d2h = F * (m.n_expr + 6) * 4 + F * 3 * 4 + F * C.sizeof(tdi.Report)

    # max over ranks
    total_ms, e2e_ms, other_ms = max_over_ranks([total_ms, e2e_ms, other_ms], world, device="cuda")
    frames_all = F * world * args.steps
    value = job_rate(F, world, args.steps, total_ms)
    e2e = job_rate(F, world, args.steps, e2e_ms)

    hbm, tfl, peak_kind = measured_peaks()
    per_frame, per_launch = algorithmic_bytes(args.profile_kernel, m.n_vertices, m.n_triangles, m.n_expr, n_frag)
    avg_launch_s = prof_ms / 1000.0 / max(prof_launches, 1)
    frames_per_launch = prof_frames / max(prof_launches, 1)
    bytes_per_launch = per_frame * frames_per_launch + per_launch
    achieved = bytes_per_launch / avg_launch_s / 1e9 if prof_launches else None
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tr = json.load(f).get(args.profile_kernel)
        if tr:
            traffic = tr["dram_bytes_per_frame"] * frames_per_launch + tr.get("dram_bytes_per_launch", 0.0)

    line = {
        "metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded morphable model and frames)",
        "config": {"workload": WORKLOAD, "frames_per_gpu_per_step": F,
                   "vertices": m.n_vertices, "triangles": m.n_triangles, "expr": m.n_expr,
                   "max_outer_iters": MAX_ITERS, "crop": "256x256",
                   "mean_fragments": n_frag,
                   "l2": "inputs larger than L2 (256 MB of crops per 1,024 frames)",
                   "parallelism": f"frames sharded over {world} GPU(s), no collective",
                   "normal_eq": args.normal_eq},
        "e2e": {"value": e2e, "unit": "frames/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "roofline": {"kernel": args.profile_kernel, "bound": "hbm", "achieved": achieved,
                     "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm if achieved else None, "traffic": traffic,
                     "peak_source": peak_kind, "launches": prof_launches,
                     "avg_launch_ms": avg_launch_s * 1000.0, "frames_per_launch": frames_per_launch,
                     "algorithmic_bytes_per_frame": per_frame, "algorithmic_bytes_per_launch": per_launch},
        "compute": ({"kernel": "vertex", "achieved": vertex_flops_per_frame(m.n_vertices, m.n_expr) * frames_per_launch
                                                     / avg_launch_s / 1e12,
                     "peak": FP32_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                     "frac": vertex_flops_per_frame(m.n_vertices, m.n_expr) * frames_per_launch / avg_launch_s / 1e12
                             / FP32_NOMINAL_TFLOPS,
                     "peak_source": "nominal FP32 SIMT: 148 SMs x 128 lanes x 2 flops x 1.965 GHz",
                     "note": "basis x coefficients as a sequential FP32 FMA chain (bit-exact order), no tensor-core form"}
                    if args.profile_kernel == "vertex" and prof_launches else None),
        "normal_eq_modes": {args.normal_eq: {"value": value, "ms_per_step": total_ms / args.steps},
                            other: {"value": frames_all / (other_ms / 1000.0), "ms_per_step": other_ms / args.steps,
                                    "mean_renders": float(np.mean([r.renders for r in rep_o])),
                                    "failed": int(sum(1 for r in rep_o if r.flags & tdi.FLAG_FAIL))},
                            "note": "exact: FP64 normal equations in the oracle's order (bit-identical fits); "
                                    "tensor: split-BF16 tcgen05 products, FP32 chunk accumulation"},
        "clocks": clk,
        "fit": {"mean_iters_rigid": float(np.mean([r.iters_rigid for r in rep])),
                "mean_iters_lambda": float(np.mean([r.iters_lambda for r in rep])),
                "mean_renders": float(np.mean([r.renders for r in rep])),
                "failed": int(sum(1 for r in rep if r.flags & tdi.FLAG_FAIL))},
    }
    if rank == 0 and world == 1:
        nplain = min(args.plain_frames, F)
        if nplain > 0:
            # plain form: the same frames fitted one at a time (a batch of one per fit)
            one = tdi.Batch(model, 1)
            plain_ms = 0.0
            for i in range(nplain):
                one.set_frames(fr, i, i + 1)
                one.set_state(fr.state_init[i:i + 1], lam0[i:i + 1], L[i:i + 1])
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                one.fit(cfg)
                e1.record()
                torch.cuda.synchronize()
                plain_ms += e0.elapsed_time(e1)
            one.close()
            line["plain"] = {"value": nplain / (plain_ms / 1000.0), "unit": "frames/s",
                             "frames": nplain, "note": "unbatched: one frame per fit, same kernels"}
            line["batched_over_plain"] = value / line["plain"]["value"]

        if args.cpu_frames > 0:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle as O
            O.build()
            n = min(args.cpu_frames, F)
            threads = O.max_threads()
            rate = cpu_fit_rate(O, synth, m, fr, n, threads)
            line["cpu_baseline"] = {"value": rate, "unit": "frames/s", "cores": threads, "kind": "port",
                                    "sample": f"first {n} frames of the same batch, FP32 CPU restatement"}
            # parameter error of the GPU fit against the FP32 and FP64 oracles on those frames
            om = O.Model(m)
            fs = O.FrameSet(fr, 0, n)
            ocfg = O.config(max_iters_rigid=MAX_ITERS)
            errs = {args.normal_eq: {}, other: {}}
            for kind in ("f32", "f64"):
                ox, ol, orep = O.fit_frames(om, fs, ocfg, fr.state_init[:n], lam0[:n], L[:n], kind=kind)
                for mode, xg in ((args.normal_eq, x), (other, xo_gpu)):
                    rel = np.abs(xg[:n] - ox) / np.maximum(np.abs(ox), 1e-2)
                    errs[mode]["vs_" + ("fp32" if kind == "f32" else "fp64") + "_oracle"] = {
                        "max_rel": float(rel.max()), "median_rel": float(np.median(rel)),
                        "frames_within_1e-5": int(np.sum(rel.max(axis=1) <= 1e-5))}
            line["param_err"] = {"frames": n, **errs[args.normal_eq], other: errs[other],
                                 "definition": "|x_gpu - x_oracle| / max(|x_oracle|, 1e-2) over pose and expressions"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    batch.close()
    model.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
