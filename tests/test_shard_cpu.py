"""Sharding one migration over ranks (poststackmig3d_b200.shard) on CPU: two gloo ranks each
migrate their slab of output inlines and rank 0 gathers the image.  The oracle stands in for
the GPU operator, so the gathered image must equal the oracle's whole image bit for bit; a
rank that fails raises on the host and the other rank's collective ends with an error."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case():
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from poststackmig3d_b200 import synth as S
    from helpers import geometry_for
    W = S.random_workload(81, 18, 6, 80, vel_kind="lateral", pad_il=2, pad_xl=1, d_il=80.0)
    return W, geometry_for(W)


def _oracle_migrate(lg, traces, vrms, device):
    import oracle as O
    return O.migrate_volume(traces, vrms, lg.out_center, lg.n_ox, lg.pad_il, lg.pad_xl,
                            lg.m_il, np.float32(lg.dt_seconds), lg.t0(), np.float32(lg.tan2),
                            lg.d_il, lg.d_xl, lg.amp)[0]


def _worker(rank, world, port, out_path, fail_rank):
    import sys
    sys.path.insert(0, ROOT)
    import datetime
    import torch.distributed as dist
    from poststackmig3d_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=20))
    try:
        W, g = _case()
        weight = np.linspace(1.0, 2.0, g.n_oi)

        def migrate(lg, tr, vr, dev):
            if rank == fail_rank:
                raise RuntimeError("injected failure on the host")
            return _oracle_migrate(lg, tr, vr, dev)

        try:
            img = shard.migrate_sharded(g, W.data, W.vrms_cube(), rank, world,
                                        weight=weight, migrate=migrate)
            if rank == 0:
                np.save(out_path, img)
        except Exception as e:  # report the failure to the parent
            with open(out_path + f".err{rank}", "w") as f:
                f.write(type(e).__name__ + ": " + str(e))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(tmp_path, fail_rank):
    out = str(tmp_path / "img.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out, fail_rank)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert not p.is_alive()
    return out


def test_sharded_image_equals_whole_image(tmp_path):
    out = _run(tmp_path, fail_rank=-1)
    assert not any(os.path.exists(out + f".err{r}") for r in range(2))
    W, g = _case()
    whole = _oracle_migrate(g, W.data, W.vrms_cube(), 0)
    assert np.array_equal(np.load(out), whole)


def test_failed_rank_surfaces_as_errors(tmp_path):
    out = _run(tmp_path, fail_rank=1)
    assert open(out + ".err1").read().startswith("RuntimeError: injected failure")
    # rank 0 waited for rank 1's rows: its receive ends with an error, not a hang
    assert os.path.exists(out + ".err0") and not os.path.exists(out)
