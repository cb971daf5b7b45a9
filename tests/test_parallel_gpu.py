"""Two ranks through the engine: shot sharding, per-rank imaging on the GPU
and the one image reduction per offset group (q_psdm_b200.parallel).

Both ranks are processes on the one GPU a test run has; each runs its own
engine on its own shots, and no kernel of one rank waits on the other (the
only exchange is the reduction, which here goes through gloo on host
tensors -- on a multi-GPU node it is NCCL over NVLink).  The reduced image
must equal one engine imaging every shot (up to the order of the two float
sums) and the oracle, with point-trace counts that add up exactly.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out, kind):
    import torch
    import torch.distributed as dist

    from q_psdm_b200 import parallel

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        if kind == "compat":
            from tests.compat_case import engine_run, make_case
            case = make_case("block")
            h = case["hdr"]
            from q_psdm_b200 import engine as E
            rec = E.encode_su(h[:, 0], h[:, 1], h[:, 2], h[:, 3], case["traces"], dt_us=2000,
                              scalco=case["sv"].scalco)
            _, idx = parallel.shard_records(rec, rank, world)
            sub = dict(case, hdr=case["hdr"][idx], traces=case["traces"][idx])
            eng, img, *_ = engine_run(sub, device=0)
        else:
            from tests import physics_case as P
            case = P.make_case(nshots=4, rstep=2)
            _, idx = parallel.shard_records(P.records(case), rank, world)
            sub = dict(case, hdr=case["hdr"][idx], traces=case["traces"][idx])
            eng, _, _ = P.engine(sub, panel_dtype=2, form=1)
            eng.submit(P.records(sub))
            img = eng.get_image(False)
        _, npt = eng.counters()
        eng.close()
        t = torch.from_numpy(np.ascontiguousarray(img, np.float32))
        parallel.reduce_image(t, dist, dst=0)
        n = torch.tensor([len(idx), npt], dtype=torch.int64)
        dist.all_reduce(n)
        if rank == 0:
            np.save(out, t.numpy())
            np.save(out + ".n.npy", n.numpy())
    finally:
        dist.destroy_process_group()


def _run_two(tmp_path, kind):
    out = str(tmp_path / f"{kind}.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out, kind), nprocs=2, join=True,
                       start_method="spawn")
    return np.load(out), np.load(out + ".n.npy")


def test_two_ranks_compat_engine(cuda, tmp_path):
    from tests.compat_case import engine_run, make_case, oracle_run
    got, n = _run_two(tmp_path, "compat")
    case = make_case("block")
    eng, one, *_ = engine_run(case, device=0)
    _, npt1 = eng.counters()
    eng.close()
    _, _, want, npt = oracle_run(case)
    assert n[0] == case["hdr"].shape[0]
    assert n[1] == npt == npt1
    peak = np.abs(want).max()
    assert np.abs(got - one).max() <= 1e-5 * peak
    assert np.abs(got - want).max() <= 1e-5 * peak


def test_two_ranks_physics_batched_engine(cuda, tmp_path):
    from tests import physics_case as P
    got, n = _run_two(tmp_path, "physics")
    case = P.make_case(nshots=4, rstep=2)
    ref, npt, _ = P.oracle_run(case)
    eng, _, _ = P.engine(case, panel_dtype=2, form=1)
    eng.submit(P.records(case))
    one = eng.get_image(False)
    eng.close()
    assert n[0] == case["hdr"].shape[0]
    assert n[1] == npt
    assert np.abs(got - one).max() <= 1e-5 * np.abs(one).max()
    assert P.nrmse(got, ref) <= 2.5e-4
