#!/usr/bin/env python
"""Throughput of the batched 3DMM video fit (fitted frames/s) on B200.

Workload "cap53k_video": the seeded synthetic morphable model with the shapes of the
reference's full-size model (53,490 vertices, 106,466 triangles, 79 expression components),
a batch of video frames (AR(1) expressions, random-walk head pose, face boxes 120-600 px in
1080p) rescaled to the reference's 256x256 crop, fitted per frame as
VideoFitter::fit_to_video_frame does after its landmark initialisation: light fit, then the
log-barrier Gauss-Newton shape fit (pose + 79 expressions) capped at 20 outer iterations. The
fits start from the device landmark initializer's states (tdi_batch_landmark_init, run once
before timing; its own rate is the ``landmark_init`` field).

One step = one fit of the whole batch. ``value`` times ``tdi_batch_fit`` with every input
resident in device memory; ``e2e`` times ``tdi_fit_frames`` from pinned host buffers
(host->device copy of the frames and states, the fit, and the read-back of states and reports).
Inputs (256 MB of target crops for 1,024 frames) exceed the 126 MB L2 between steps.

``--impl reference`` times the CPU restatement of the same path (oracle/, OpenMP over frames,
all host threads) on a bounded sample of the same frames: 3DI's path is CUDA-only and has no
CPU implementation of its own (its kernels are built from its sources for parity tests only).
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
    ap.add_argument("--cpu-frames", type=int, default=64, help="frames of the CPU sample (about 10 s of CPU work)")
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


def shard_range(n_frames, world, rank):
    """Contiguous frames [f0, f1) of rank `rank` when one video's frames are split over `world`
    GPUs (frames are independent: no exchange until the outputs are gathered)."""
    return n_frames * rank // world, n_frames * (rank + 1) // world


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


KERNELS = ["vertex", "raster", "raster_resolve", "render", "neighbours", "jacobian", "normal_eq", "barrier",
           "solve"]
FP64_NOMINAL_TFLOPS = 40.0   # B200 FP64 tensor, nominal (no measured FP64 figure on this pool)


def algorithmic_bytes(kernel: str, V: int, T: int, K: int, n_frag: float):
    """(bytes per frame, bytes per launch) a kernel must move: what the roofline divides by.
    None for the latency-bound per-frame kernels (barrier terms, Cholesky)."""
    KT = K + 6
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
    if kernel == "raster_resolve":
        # the frame's triangle mask, the corners and projections of the triangles with
        # fragments (about one per fragment), their depth keys and the fragment records written;
        # then per fragment its record, its triangle's corners, three vertices' object
        # coordinates and albedo, and the shading records written (unit normal and n . p, albedo)
        return T / 8.0 + n_frag * (16 + 3 * 16 + 8 + 16) + n_frag * (16 + 16 + 3 * 16 + 20), 0.0
    if kernel == "render":
        # fragments, their shading records, four target pixels, gradients
        return n_frag * (16 + 20 + 4 * 4 + 5 * 4), 0.0
    if kernel == "neighbours":
        # fragment pixels in, four neighbour indices out
        return n_frag * (16 + 16), 0.0
    if kernel == "jacobian":
        # three vertices' basis rows (3 coords x K) and the row written
        return n_frag * (3 * 3 * K * 4 + KT * 4), 0.0
    if kernel == "normal_eq":
        # every Jacobian row read once, gradients and neighbour indices, the chunk partials
        return n_frag * (KT * 4 + 5 * 4 + 16) + 128 * KT * KT * 8 / 2, 0.0
    return None, None


def normal_eq_flops_per_frame(K: int, n_frag: float) -> float:
    """Algorithmic flops of J^T J and J^T r: 2 (2N) K^2 + 2 (2N) K (the x and y rows)."""
    KT = K + 6
    return 2.0 * 2 * n_frag * KT * KT + 2.0 * 2 * n_frag * KT


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
    om = O.Model(m)
    fs = O.FrameSet(fr)
    p0L = landmark_points(m)
    fr.state_init = np.stack([O.landmark_init(om, fs, i, p0L)[0] for i in range(n)])
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
                         "sample": f"{n} frames of {WORKLOAD} from the landmark initializer's states, "
                                   "FP32 CPU restatement (oracle/); 3DI's path is CUDA-only, it has no "
                                   "CPU implementation"},
        "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def landmark_points(m):
    """The landmark vertices of the subject's shape, [3][51] (the reference's p0L_mat.dat)."""
    return np.ascontiguousarray(m.mean[:, m.lis].astype(np.float32))


def render_targets_cpu(O, synth, m, fr):
    om = O.Model(m)
    cfg = O.config()
    imgs = [O.render_target(om, fr, i, cfg, fr.state_true[i], fr.lam_true[i], synth.L_INTENSITY)[0]
            for i in range(fr.n_frames)]
    fr.target = synth.add_noise(np.stack(imgs), 0.02, 3)


def fit_timed(batch, cfg, fr, lam0, L, steps, barrier):
    """Device time (ms) of `steps` fits of the resident batch, each from the initial states."""
    import torch
    total = 0.0
    for _ in range(steps):
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
        total += e0.elapsed_time(e1)
    return total


def kernel_table(batch, cfg, fr, lam0, L, m, n_frag, hbm, tfl, names=None):
    """Every major kernel timed live with CUDA events on its stream, one untimed fit per kernel
    (tdi_batch_profile): launches, device time, frames processed, share of the kernels' sum,
    and its roofline against its algorithmic bytes (or flops)."""
    rows = {}
    for name in (names or KERNELS):
        batch.set_state(fr.state_init, lam0, L)
        batch.profile(name)
        batch.fit(cfg)
        n, ms, frames = batch.profile_read()
        batch.profile(None)
        rows[name] = {"launches": n, "ms": ms, "frames": frames}
    total = sum(r["ms"] for r in rows.values())
    for name, r in rows.items():
        r["share"] = r["ms"] / total if total and names is None else None
        r["us_per_frame"] = 1000.0 * r["ms"] / r["frames"] if r["frames"] else None
        per_frame, per_launch = algorithmic_bytes(name, m.n_vertices, m.n_triangles, m.n_expr, n_frag)
        if per_frame is not None and r["launches"]:
            avg_s = r["ms"] / 1000.0 / r["launches"]
            fpl = r["frames"] / r["launches"]
            bpl = per_frame * fpl + per_launch
            r["hbm_gbs"] = bpl / avg_s / 1e9
            r["hbm_frac"] = r["hbm_gbs"] / hbm
        if name == "vertex" and cfg.vertex_stage == 1 and r["launches"]:
            r["tflops_tensor"] = 6 * vertex_flops_per_frame(m.n_vertices, m.n_expr) * r["frames"] / (r["ms"] / 1000.0) / 1e12
            r["tflops_tensor_note"] = "six split-BF16 products per FP32 product, against the measured bf16 peak"
            r["tflops_tensor_frac"] = r["tflops_tensor"] / tfl
        if name == "normal_eq" and r["launches"]:
            fl = normal_eq_flops_per_frame(m.n_expr, n_frag) * r["frames"] / (r["ms"] / 1000.0) / 1e12
            r["tflops"] = fl
            r["tflops_frac_of_peak"] = fl / (tfl if cfg.normal_eq == 1 else FP64_NOMINAL_TFLOPS)
            r["tflops_peak"] = "measured bf16" if cfg.normal_eq == 1 else "nominal FP64 tensor (40 TFLOP/s)"
        if name == "vertex" and r["launches"]:
            r["fp32_tflops"] = vertex_flops_per_frame(m.n_vertices, m.n_expr) * r["frames"] / (r["ms"] / 1000.0) / 1e12
            r["fp32_frac_of_nominal"] = r["fp32_tflops"] / FP32_NOMINAL_TFLOPS
    return rows


def step_error_table(O, om, fs, fr, lam0, L, tdi, batch, n, cfg):
    """Errors of every output of one Gauss-Newton step against the FP64 oracle, from the same
    state (the frames' initial states), by parameter group: H blocks (relative Frobenius), g,
    d and the first trial point x + d (relative max norm), the objective (relative)."""
    K = om.K
    groups = {"expr": slice(0, K), "pose": slice(K, K + 6)}
    batch.set_state(fr.state_init, lam0, L)
    batch.evaluate(cfg)
    acc = {}
    for i in range(n):
        x = fr.state_init[i]
        e = O.evaluate(om, fs, i, O.config(), x, lam0[i], float(L[i]), kind="f64")
        ne = batch.read(i, tdi.READ_NORMAL_EQ)
        sc = batch.read(i, tdi.READ_SCALARS)
        H, Ho = ne["H"].astype(np.float64), e["H"].astype(np.float64)
        r = {}
        for a, sa in groups.items():
            for b, sb in groups.items():
                r[f"H_{a}_{b}"] = np.linalg.norm(H[sa, sb] - Ho[sa, sb]) / np.linalg.norm(Ho[sa, sb])
        for a, sa in groups.items():
            for name, v, vo in (("g", ne["g"], e["g"]), ("d", ne["d"], e["d"]), ("trial", x + ne["d"], x + e["d"])):
                vo = vo.astype(np.float64)
                r[f"{name}_{a}"] = np.abs(v[sa] - vo[sa]).max() / max(np.abs(vo[sa]).max(), 1e-30)
        r["objective"] = abs(sc["objective"] - e["objective"]) / abs(e["objective"])
        for k, v in r.items():
            acc.setdefault(k, []).append(float(v))
    # a direction of NaN (the factorisation of an indefinite H failed, which ends the frame's fit
    # as the reference's failed potrf does) is counted, not averaged
    out = {}
    for k, v in acc.items():
        v = np.asarray(v)
        ok = v[np.isfinite(v)]
        out[k] = {"median": float(np.median(ok)) if ok.size else None, "max": float(ok.max()) if ok.size else None}
        if ok.size < v.size:
            out[k]["failed_factorisations"] = int(v.size - ok.size)
    return out


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
    # every fit starts from the device landmark initializer's output (computed once here; its
    # own rate is measured below)
    p0L = landmark_points(m)
    lm_ok, _, lm_it = batch.landmark_init(p0L)
    fr.state_init = batch.get_state()[0].copy()
    lam0 = np.tile(synth.LAMBDA_INIT, (F, 1)).astype(np.float32)
    neq = tdi.NORMAL_EQ_TENSOR if args.normal_eq == "tensor" else tdi.NORMAL_EQ_EXACT
    cfg = tdi.default_config(max_iters_rigid=MAX_ITERS, normal_eq=neq)

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
    launches0 = batch.launches()
    total_ms = fit_timed(batch, cfg, fr, lam0, L, args.steps, barrier)
    launches = batch.launches() - launches0
    clk = clocks.stop()
    x, lamf, rep = batch.get_state()
    n_frag = float(np.mean([r.n_fragments for r in rep]))
    gn_iters = int(sum(r.iters_rigid + r.iters_finetune for r in rep))
    renders = int(sum(r.renders for r in rep))

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
    other_ms = fit_timed(batch, cfg_o, fr, lam0, L, args.steps, barrier)
    xo_gpu, _, rep_o = batch.get_state()
    # both contractions on the tensor cores: the vertex stage and the normal equations
    cfg_t = tdi.default_config(max_iters_rigid=MAX_ITERS, normal_eq=tdi.NORMAL_EQ_TENSOR,
                               vertex_stage=tdi.VERTEX_TENSOR)
    batch.set_state(fr.state_init, lam0, L)
    batch.fit(cfg_t)
    tensor_all_ms = fit_timed(batch, cfg_t, fr, lam0, L, args.steps, barrier)
    _, _, rep_t = batch.get_state()
    # the reference's cfg1 stage sequence: two-stage illumination and the expression finetune
    cfg1 = tdi.default_config(max_iters_rigid=MAX_ITERS, max_iters_finetune=MAX_ITERS, twostage_illum=1,
                              finetune=1, normal_eq=neq)
    batch.set_state(fr.state_init, lam0, L)
    batch.fit(cfg1)
    cfg1_ms = fit_timed(batch, cfg1, fr, lam0, L, args.steps, barrier)
    _, _, rep1 = batch.get_state()
    # the differentiable entry: loss (FP64 over the raster's fragments) and its adjoint for
    # every frame of the batch at the initial states, through torch.autograd
    ag = importlib.import_module("3di_b200.autograd")
    dev = torch.device("cuda", local)
    xd = torch.from_numpy(np.ascontiguousarray(fr.state_init, np.float32)).to(dev)
    ld = torch.from_numpy(lam0).to(dev)
    Ld = torch.from_numpy(L).to(dev)
    adj_ms = 0.0
    for it in range(args.warmup + args.steps):
        xr = xd.clone().requires_grad_(True)
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        ag.render_loss(batch, xr, ld, Ld, cfg).sum().backward()
        e1.record()
        torch.cuda.synchronize()
        barrier()
        if it >= args.warmup:
            adj_ms += e0.elapsed_time(e1)
    # the landmark initialisation of the same frames (orthographic fit + barrier method)
    lm_ms = 0.0
    for _ in range(args.steps):
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        batch.landmark_init(p0L)
        e1.record()
        torch.cuda.synchronize()
        barrier()
        lm_ms += e0.elapsed_time(e1)
    h2d = sum(h[k].numel() * h[k].element_size() for k in ("t", "xl", "yl", "b", "fs", "cam", "o", "x", "lam", "L"))
    d2h = F * (m.n_expr + 6) * 4 + F * 3 * 4 + F * C.sizeof(tdi.Report)

    # max over ranks
    total_ms, e2e_ms, other_ms, cfg1_ms, lm_ms, tensor_all_ms, adj_ms = max_over_ranks(
        [total_ms, e2e_ms, other_ms, cfg1_ms, lm_ms, tensor_all_ms, adj_ms], world, device="cuda")
    frames_all = F * world * args.steps
    value = job_rate(F, world, args.steps, total_ms)
    e2e = job_rate(F, world, args.steps, e2e_ms)

    # per-kernel live timing (untimed fits) and the roofline of the largest-share kernel
    hbm, tfl, peak_kind = measured_peaks()
    kt = kernel_table(batch, cfg, fr, lam0, L, m, n_frag, hbm, tfl)
    kt_t = kernel_table(batch, cfg_t, fr, lam0, L, m, n_frag, hbm, tfl, names=("vertex", "normal_eq"))
    top = max((k for k in kt if "hbm_gbs" in kt[k]), key=lambda k: kt[k]["ms"])
    per_frame, per_launch = algorithmic_bytes(top, m.n_vertices, m.n_triangles, m.n_expr, n_frag)
    tr_ = kt[top]
    fpl = tr_["frames"] / max(tr_["launches"], 1)
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath):
        with open(tpath) as f:
            tr = json.load(f).get(top)
        if tr:
            traffic = tr["dram_bytes_per_frame"] * fpl + tr.get("dram_bytes_per_launch", 0.0)

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
        "gn_iters_per_s": gn_iters * world * args.steps / (total_ms / 1000.0),
        "evaluations_per_s": renders * world * args.steps / (total_ms / 1000.0),
        "roofline": {"kernel": top, "bound": "hbm", "achieved": tr_["hbm_gbs"], "peak": hbm, "unit": "GB/s",
                     "frac": tr_["hbm_frac"], "traffic": traffic, "peak_source": peak_kind,
                     "share": tr_["share"], "launches": tr_["launches"],
                     "avg_launch_ms": tr_["ms"] / max(tr_["launches"], 1), "frames_per_launch": fpl,
                     "algorithmic_bytes_per_frame": per_frame, "algorithmic_bytes_per_launch": per_launch},
        "kernels": kt,
        "normal_eq_modes": {args.normal_eq: {"value": value, "ms_per_step": total_ms / args.steps},
                            other: {"value": frames_all / (other_ms / 1000.0), "ms_per_step": other_ms / args.steps,
                                    "mean_renders": float(np.mean([r.renders for r in rep_o])),
                                    "failed": int(sum(1 for r in rep_o if r.flags & tdi.FLAG_FAIL))},
                            "tensor_vertex_and_normal_eq": {
                                "value": frames_all / (tensor_all_ms / 1000.0), "ms_per_step": tensor_all_ms / args.steps,
                                "mean_renders": float(np.mean([r.renders for r in rep_t])),
                                "failed": int(sum(1 for r in rep_t if r.flags & tdi.FLAG_FAIL)),
                                "kernels": kt_t},
                            "note": "exact: FP64 normal equations in the oracle's order (bit-identical fits); "
                                    "tensor: split-BF16 tcgen05 products, FP32 chunk accumulation; "
                                    "tensor_vertex_and_normal_eq: the vertex stage's basis products on tcgen05 "
                                    "as well (split BF16, FP32 accumulation)"},
        "stage_sequences": {"light_shape": {"value": value, "note": "light fit + shape fit (one face scale)"},
                            "cfg1": {"value": frames_all / (cfg1_ms / 1000.0), "ms_per_step": cfg1_ms / args.steps,
                                     "mean_iters_finetune": float(np.mean([r.iters_finetune for r in rep1])),
                                     "note": "light, shape, two-stage illumination (2 more light + shape fits) "
                                             "and the expression finetune, as the reference's cfg1 runs each "
                                             "face scale"}},
        "differentiable_loss": {"value": frames_all / (adj_ms / 1000.0), "unit": "frames/s",
                                "note": "tdi_batch_loss + tdi_batch_loss_backward through torch.autograd on the "
                                        "same batch (raster, FP64 forward and hand-written adjoint per frame)"},
        "landmark_init": {"value": frames_all / (lm_ms / 1000.0), "unit": "frames/s",
                          "succeeded": int(lm_ok.sum()), "frames": F,
                          "mean_newton_iters": float(np.mean(lm_it)),
                          "note": "tdi_batch_landmark_init: orthographic fit, mirrored refit, barrier method "
                                  "with slack; the fits above start from its output"},
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
            # CPU baseline leg: the oracle timed on the host cores, then used as the checker
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
                t0 = time.perf_counter()
                ox, ol, orep = O.fit_frames(om, fs, ocfg, fr.state_init[:n], lam0[:n], L[:n], kind=kind, threads=threads)
                if kind == "f64":
                    # the FP64 restatement, the survey's named CPU baseline, on the same sample
                    line["cpu_baseline"]["fp64_oracle"] = {"value": n / (time.perf_counter() - t0), "unit": "frames/s",
                                                           "cores": threads}
                for mode, xg in ((args.normal_eq, x), (other, xo_gpu)):
                    key = "vs_" + ("fp32" if kind == "f32" else "fp64") + "_oracle"
                    rel = np.abs(xg[:n] - ox) / np.maximum(np.abs(ox), 1e-2)
                    K = m.n_expr
                    # pose: translation relative to the depth, rotation vector in radians
                    dt = np.abs(xg[:n, K:K + 3] - ox[:, K:K + 3]).max(axis=1) / np.abs(ox[:, K + 2])
                    du = np.abs(xg[:n, K + 3:K + 6] - ox[:, K + 3:K + 6]).max(axis=1)
                    errs[mode][key] = {
                        "max_rel": float(rel.max()), "median_rel": float(np.median(rel)),
                        "expr_median_rel": float(np.median(rel[:, :K])),
                        "tau_over_depth_median": float(np.median(dt)), "tau_over_depth_max": float(dt.max()),
                        "rotation_rad_median": float(np.median(du)), "rotation_rad_max": float(du.max()),
                        "frames_within_1e-5": int(np.sum(rel.max(axis=1) <= 1e-5))}
                    if mode == args.normal_eq:
                        errs[mode][key]["light_max_rel"] = float(
                            (np.abs(lamf[:n] - ol) / np.maximum(np.abs(ol), 1e-6)).max())
            line["param_err"] = {"frames": n, **errs[args.normal_eq], other: errs[other],
                                 "definition": "|x_gpu - x_oracle| / max(|x_oracle|, 1e-2) over pose and expressions "
                                               "after the whole fit; tau_over_depth: |tau_gpu - tau_oracle|_inf / "
                                               "|tau_z|; rotation_rad: |u_gpu - u_oracle|_inf; light: "
                                               "|lam_gpu - lam_oracle| / |lam_oracle|"}
            # every output of one Gauss-Newton step against the FP64 oracle, both modes
            line["step_err"] = {
                "frames": n,
                args.normal_eq: step_error_table(O, om, fs, fr, lam0, L, tdi, batch, n, cfg),
                other: step_error_table(O, om, fs, fr, lam0, L, tdi, batch, n, cfg_o),
                "definition": "one evaluation at the initial states vs the FP64 oracle: H blocks relative "
                              "Frobenius, g, d and x + d relative max norm per group, objective relative"}
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
