"""The N > 1 path of bench.py on CPU: two gloo ranks (127.0.0.1). Frames shard across ranks
with no data-path exchange; the only collective is the MAX over ranks of the device times,
and the whole-job rate counts every rank's frames over the slowest rank's time."""
import importlib
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    synth = importlib.import_module("3di_b200.synth")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        times = [10.0 + rank, 20.0 - 5.0 * rank, 7.0]         # this rank's device times, ms
        reduced = bench.max_over_ranks(times, world)
        m, fr = bench.make_workload(synth, 2, seed_offset=100 * rank)
        q.put((rank, reduced, fr.state_init.copy(), fr.x0y0.copy()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_times_and_shard_frames():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        rank, reduced, x0, o = q.get(timeout=300)
        got[rank] = (reduced, x0, o)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # the MAX over ranks, identical on both
    assert got[0][0] == got[1][0] == [11.0, 20.0, 7.0]
    # disjoint shards: each rank fits its own seeded frames
    assert not np.array_equal(got[0][1], got[1][1])


def test_job_rate_counts_every_ranks_frames():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.job_rate(1024, 1, 3, 900.0) == pytest.approx(3413.333, rel=1e-6)
    assert bench.job_rate(1024, 8, 3, 900.0) == pytest.approx(8 * 3413.333, rel=1e-6)


def _fit_rank(rank, world, port, q):
    """Fits this rank's contiguous share of the frames (the CPU oracle stands in for the GPU
    path, which this machine cannot run) and gathers every rank's results."""
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import bench
    import oracle as O
    from conftest import make_case
    synth = importlib.import_module("3di_b200.synth")
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        m, fr, om = make_case(synth, O, 5000, 9800, 0, 3, dict(image_wh=(256, 256), tz=0.6))
        f0, f1 = bench.shard_range(fr.n_frames, world, rank)
        lam = np.tile(synth.LAMBDA_INIT, (f1 - f0, 1))
        L = np.full(f1 - f0, synth.L_INTENSITY, np.float32)
        x, _, _ = O.fit_frames(om, O.FrameSet(fr, f0, f1), O.config(max_iters_rigid=3), fr.state_init[f0:f1], lam, L,
                               threads=1)
        parts = [None] * world
        dist.all_gather_object(parts, (f0, f1, x))
        q.put((rank, parts))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_fit_disjoint_frames_like_one_process(O, synth, small_case):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_fit_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=600) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    m, fr, om = small_case
    lam = np.tile(synth.LAMBDA_INIT, (fr.n_frames, 1))
    L = np.full(fr.n_frames, synth.L_INTENSITY, np.float32)
    ref, _, _ = O.fit_frames(om, O.FrameSet(fr), O.config(max_iters_rigid=3), fr.state_init, lam, L)
    for rank in (0, 1):
        parts = got[rank]
        assert [p[:2] for p in parts] == [(0, 1), (1, 3)]
        x = np.concatenate([p[2] for p in parts])
        assert np.array_equal(x, ref)
