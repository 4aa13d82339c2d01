"""Multi-rank sample sharding on CPU (gloo, world size 2).

Each rank renders its own sample range of the Cornell scene with the oracle's
counter-based integrator and the ranks sum their accumulation buffers with one
all-reduce, as the multi-GPU benchmark does with the library on NCCL. The sum
must equal one process rendering every one of those samples, and the ranges of
the ranks must be disjoint.
"""
import ctypes as C
import os
import socket
import sys

import numpy as np
import pytest

import mcpt
import sharding

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")

W = H = 12
STEPS, WARM = 2, 1


def _scene():
    s = mcpt.generate_scene(mcpt.SCENE_CORNELL_BOXES)
    cam = mcpt.Camera.from_buffer_copy(bytes(s.camera))
    cam.image_width = W
    cam.aspect_ratio = 1.0
    mcpt.camera_initialize(cam)
    return s, cam


def _render(samples):
    """Oracle render of the given sample indices, summed (float64 accumulation)."""
    from helpers import oracle
    orc = oracle()
    s, cam = _scene()
    tris = mcpt.host_triangles(s)
    h = orc.orc_scene_create(C.addressof(tris), len(tris), None, 0, None, 0, 0, 1.0, 0.0)
    acc = np.zeros(W * H * 3, np.float64)
    stats = np.zeros(2, np.float64)
    try:
        for smp in samples:
            orc.orc_render(h, C.addressof(cam), W, H, 1, smp, 8, 1234, 0, 0, 0, 0, W, H, 1, acc.ctypes.data,
                           stats.ctypes.data)
    finally:
        orc.orc_scene_destroy(h)
        mcpt.free_scene(s)
    return acc


def _free_port():
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [here, os.path.join(os.path.dirname(here), "monocuda-pt_b200")]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        timed, _ = sharding.sample_ranges(rank, world, STEPS, WARM)
        acc = torch.from_numpy(_render(list(timed)))
        sharding.reduce_accumulation(acc, world)
        np.save(os.path.join(out_dir, "rank%d.npy" % rank), acc.numpy())
    finally:
        dist.destroy_process_group()


def test_sample_ranges_are_disjoint_and_cover_the_job():
    world = 4
    seen = set()
    for r in range(world):
        timed, warm = sharding.sample_ranges(r, world, STEPS, WARM)
        assert len(timed) == STEPS and len(warm) == WARM
        for s in list(timed) + list(warm):
            assert s not in seen
            seen.add(s)
    assert sharding.all_timed_samples(world, STEPS, WARM) == [s for r in range(world)
                                                              for s in sharding.sample_ranges(r, world, STEPS, WARM)[0]]
    with pytest.raises(ValueError):
        sharding.sample_ranges(4, 4, 1, 1)


def test_two_ranks_all_reduce_equals_one_process(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    expected = _render(sharding.all_timed_samples(world, STEPS, WARM))
    assert expected.sum() > 0
    for r in range(world):
        got = np.load(os.path.join(tmp_path, "rank%d.npy" % r))
        np.testing.assert_allclose(got, expected, rtol=1e-12, atol=1e-12)
