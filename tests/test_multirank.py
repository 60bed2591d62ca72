"""Multi-rank rendering on the CPU (gloo, world size 2): each rank renders its own
slice of the sample stream with the oracle (the GPU kernels are bit-identical to it,
see test_gpu_render.py), the accumulators meet in one reduction to rank 0, and the
result equals the per-rank accumulators added up. A rank that dies before the
reduction makes the survivor's reduction fail with an error instead of hanging."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

W, H, SPP = 48, 32, 4


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def rank_accumulator(rank):
    import cpt
    from cpt.multi import rank_frame0
    from oracle import cpu

    tris, infos = cpt.scene_random(20000, seed=5)
    b = cpu.build(tris, 30)
    cam = cpt.camera_look_at((0.5, 0.5, -1.2), (0.5, 0.5, 0.0), aspect=W / H)
    rad, _ = cpu.render(b, infos, None, W, H, SPP, rank_frame0(0, rank), 3, 3.0, True, 5,
                        cpu.ocam_from(cam.eye, cam.as_array()[3:]))
    s, c, n = cpu.accumulate_kahan(rad)
    acc = np.zeros((2, H, W, 4), np.float32)
    acc[0, ..., :3], acc[0, ..., 3], acc[1, ..., :3] = s, n, c
    return acc


def worker(rank, world, port, outdir, die_rank):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "cuda-path-tracer_b200")]
    import datetime

    import torch
    import torch.distributed as dist

    from cpt.multi import reduce_accumulator

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    acc = rank_accumulator(rank)
    np.save(os.path.join(outdir, f"local{rank}.npy"), acc)
    if rank == die_rank:
        os._exit(0)  # leaves between steps, without joining the reduction
    t = torch.from_numpy(acc.copy())
    out = torch.zeros_like(t)
    try:
        reduce_accumulator(t, out, dst=0)
        status = "ok"
    except Exception as e:  # the peer is gone: the collective must fail, not hang
        status = "error: " + type(e).__name__
    np.save(os.path.join(outdir, f"reduced{rank}.npy"), out.numpy())
    np.save(os.path.join(outdir, f"after{rank}.npy"), t.numpy())
    with open(os.path.join(outdir, f"status{rank}.txt"), "w") as f:
        f.write(status)
    try:
        dist.destroy_process_group()
    except Exception:
        pass


def run(tmp_path, die_rank):
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, 2, port, str(tmp_path), die_rank)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode is not None, "rank did not finish"
    return procs


def test_two_rank_sample_sharding_and_reduce(tmp_path):
    run(tmp_path, die_rank=-1)
    assert open(tmp_path / "status0.txt").read() == "ok"
    a0 = np.load(tmp_path / "local0.npy")
    a1 = np.load(tmp_path / "local1.npy")
    got = np.load(tmp_path / "reduced0.npy")
    # each rank's compensated sum (sum - compensation), added across ranks; counts add up
    want = ((a0[0] - a0[1]).astype(np.float32) + (a1[0] - a1[1]).astype(np.float32)).astype(np.float32)
    assert got[0].tobytes() == want.tobytes()
    assert not got[1].any()
    assert np.all(got[0, ..., 3] == 2 * SPP)
    assert not np.array_equal(a0[0], a1[0]), "ranks must render different samples"
    # the ranks' own accumulators are untouched (they keep accumulating their frames)
    for r, a in ((0, a0), (1, a1)):
        assert np.load(tmp_path / f"after{r}.npy").tobytes() == a.tobytes()


def test_rank_frame0_ranges_are_disjoint():
    from cpt.multi import RANK_STREAM_STRIDE, rank_frame0

    assert rank_frame0(0, 1) == RANK_STREAM_STRIDE
    assert rank_frame0(RANK_STREAM_STRIDE - 1, 0) < rank_frame0(0, 1)
    with pytest.raises(ValueError):
        rank_frame0(RANK_STREAM_STRIDE, 0)


def test_dead_rank_fails_the_reduction_instead_of_hanging(tmp_path):
    run(tmp_path, die_rank=1)
    assert open(tmp_path / "status0.txt").read().startswith("error")
