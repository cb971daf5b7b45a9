"""Two-rank sharding and image reduction on CPU (gloo).

Each rank takes its whole shots of a compat case, images them with the CPU
restatement (no GPU here) and the images are reduced to rank 0, which must
equal the single-process image (up to float summation order)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from q_psdm_b200 import parallel


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _records(case):
    from q_psdm_b200 import engine as E
    h = case["hdr"]
    return E.encode_su(h[:, 0], h[:, 1], h[:, 2], h[:, 3], case["traces"], dt_us=2000,
                       scalco=case["sv"].scalco)


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from tests.compat_case import make_case, oracle_run

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        case = make_case("block")
        rec = _records(case)
        mine, idx = parallel.shard_records(rec, rank, world)
        sub = dict(case, hdr=case["hdr"][idx], traces=case["traces"][idx])
        _, _, img, npt = oracle_run(sub)
        t = torch.from_numpy(np.ascontiguousarray(img, np.float32))
        parallel.reduce_image(t, dist, dst=0)
        n = torch.tensor([len(idx), npt], dtype=torch.int64)
        dist.all_reduce(n)
        if rank == 0:
            np.save(out, t.numpy())
            np.save(out + ".n.npy", n.numpy())
    finally:
        dist.destroy_process_group()


def test_sharding_keeps_shots_whole():
    from tests.compat_case import make_case
    rec = _records(make_case("small"))
    shot = parallel.source_runs(rec)
    parts = [parallel.shard_records(rec, r, 3)[1] for r in range(3)]
    allidx = np.sort(np.concatenate(parts))
    assert np.array_equal(allidx, np.arange(rec.shape[0]))
    for p in parts:
        for s in np.unique(shot[p]):
            assert np.array_equal(np.nonzero(shot == s)[0], p[shot[p] == s])


def test_two_rank_reduce_equals_single(tmp_path):
    from tests.compat_case import make_case, oracle_run
    out = str(tmp_path / "img.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(out)
    n = np.load(out + ".n.npy")
    _, _, want, npt = oracle_run(make_case("block"))
    assert n[1] == npt
    assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()
