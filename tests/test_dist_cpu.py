"""Blocks over several ranks: partition, halo plan and the send/recv
exchange, run as gloo ranks on CPU with the oracle as the compute."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from finflo_b200 import case
from finflo_b200 import dist as fd

SIZES = ([6, 9], [5, 7], [4, 6])


def test_partition_balances_cells():
    cells = [100, 90, 80, 30, 20, 10, 5]
    own = fd.partition(cells, 3)
    load = [sum(c for c, o in zip(cells, own) if o == r) for r in range(3)]
    assert max(load) - min(load) <= 30
    assert fd.partition(cells, 1) == [0] * len(cells)


@pytest.mark.parametrize("world", [2, 3, 5])
def test_halo_plans_pair_up(world):
    """Every remote patch is packed once by its source's rank and unpacked
    once by its destination's rank, at matching offsets and sizes."""
    blocks, prms, _ = case.periodic_box_case(nb=(2, 2, 2), sizes=SIZES)
    own = fd.partition([b.interior_cells for b in blocks], world)
    plans = [fd.HaloPlan(blocks, own, r) for r in range(world)]
    nremote = sum(1 for l in fd.links(blocks) if own[l.src] != own[l.dst])
    assert sum(sum(1 for it in p.items if it.mode == 0) for p in plans) == nremote
    assert sum(sum(1 for it in p.items if it.mode == 1) for p in plans) == nremote
    for p in plans:
        for q, (o, n) in p.send_ranges.items():
            assert plans[q].recv_ranges[p.rank][1] == n
        for it in p.items:
            pats = p.patches[it.blk]
            assert all(pa.ibtype < len(p.local) for pa in pats)
    # local connections keep local ids, remote ones are negative
    for p in plans:
        for g, pats in zip(p.local, p.patches):
            for pa, orig in zip(pats, blocks[g].patches):
                if own[orig.ibtype] == p.rank:
                    assert p.local[pa.ibtype] == orig.ibtype
                else:
                    assert pa.ibtype == -1 - orig.ibtype


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, ncyc, out):
    import torch.distributed as dist
    from oracle.oracle import OracleMB
    from tests.dist_oracle import OracleBackend
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        blocks, prms, _ = case.periodic_box_case(nb=(2, 2, 2), sizes=SIZES)
        db = fd.DistributedBlocks(blocks, prms, OracleBackend())
        db.start()
        hist = db.cycles(ncyc)
        ref_b, ref_p, _ = case.periodic_box_case(nb=(2, 2, 2), sizes=SIZES)
        om = OracleMB(ref_b, ref_p)
        om.start()
        ref = np.array([np.r_[om.cycle(i + 1)] for i in range(ncyc)])
        ok = np.allclose(hist, ref, rtol=1e-13, atol=0)
        same = all(np.array_equal(blocks[g].arrays[n], ref_b[g].arrays[n])
                   for g in db.plan.local for n in ("TEMP", "U", "V", "W", "PDIFF", "RO", "P", "E"))
        out.put((rank, bool(ok), bool(same), len(db.plan.local), db.plan.nsend))
    except Exception as e:   # report instead of leaving the parent waiting
        out.put((rank, False, False, 0, 0, repr(e)))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_match_single_process(world):
    """gloo ranks holding parts of a 2x2x2-block periodic box give, cycle by
    cycle, the single-process oracle's fields (bitwise) and history."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, 5, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sum(r[3] for r in res) == 8
    assert all(r[4] > 0 for r in res)
    for r in res:
        assert r[1], ("history", r)
        assert r[2], ("fields", r)
