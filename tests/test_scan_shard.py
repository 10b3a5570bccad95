"""Multi-rank energy scans without a GPU: the cost-balanced shards of (block, energy run) units,
and a 2-rank gloo run of the sharded scan driver (hprmat_b200/scan_shard.py) with an
oracle-backed solver in place of the device scan, against a single-process run."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from hprmat_b200 import workloads
from hprmat_b200.scan_shard import block_costs, lpt_shards, run_sharded_scan, scan_units, shard_units, unit_cost
from oracle import rmatrix_oracle as orc

NR, RMAX = 16, 12.0


def _blocks():
    out = []
    for b, (nch, energies) in enumerate([(2, [3.0, 9.0]), (5, [4.0]), (3, [2.5, 6.0, 11.0]), (4, [7.0, 8.0])]):
        w = workloads.production(seed=40 + b, nch=nch, nr=NR, rmax=RMAX, energy=1.0)
        ks = [workloads.channel_kinematics(e, w.thresholds, w.hm, w.params.z1z2) for e in energies]
        out.append((w.lval, w.cpot, np.array([k[0] for k in ks]), np.array([k[1] for k in ks])))
    return out


def _oracle_solve(blocks):
    mesh = orc.rmat_ini(NR, 1, RMAX)
    res = []
    for lval, cpot, qk, eta in blocks:
        nch = len(lval)
        cu = np.zeros((qk.shape[0], nch, nch), dtype=np.complex128)
        nopen = np.zeros(qk.shape[0], dtype=np.int32)
        for e in range(qk.shape[0]):
            r = orc.rmatrix(nch, lval, qk[e], eta[e], RMAX, mesh, cpot)
            cu[e, :r.nopen, :r.nopen] = r.cu
            nopen[e] = r.nopen
        res.append((cu, nopen))
    return res


def test_lpt_shards_cover_every_block_once_and_balance():
    costs = [100.0, 7.0, 30.0, 30.0, 12.0, 55.0, 1.0, 40.0]
    for world in (1, 2, 3, 5, 9):
        shards = lpt_shards(costs, world)
        assert len(shards) == world
        assert sorted(i for s in shards for i in s) == list(range(len(costs)))
        loads = [sum(costs[i] for i in s) for s in shards]
        # LPT's bound: no shard above 4/3 of the optimum, itself >= max(mean load, largest item)
        assert max(loads) <= 4.0 / 3.0 * max(sum(costs) / world, max(costs)) + 1e-9
    assert lpt_shards(costs, 2) == lpt_shards(costs, 2)  # deterministic
    b = _blocks()
    c = block_costs(b, NR)
    assert c[1] == 1 * (5 * NR) ** 3 and c[2] == 3 * (3 * NR) ** 3
    # runs of energies: every (block, energy) in exactly one unit, and in one rank's shard
    units = scan_units(b, 2)
    seen = sorted((u, int(e)) for u, idx in units for e in idx)
    assert seen == sorted((u, e) for u in range(len(b)) for e in range(np.asarray(b[u][2]).shape[0]))
    got = []
    for r in range(3):
        mine, subs = shard_units(b, NR, r, 3, chunk=2)
        assert len(mine) == len(subs)
        got += [(u, int(e)) for u, idx in mine for e in idx]
    assert sorted(got) == seen


def _worker(rank, world, port, out_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res, mine = run_sharded_scan(_blocks(), NR, _oracle_solve, rank=rank, world=world, chunk=1)
        np.save(out_path + f".{rank}.npy", np.array([[int(b) for b, _ in mine], [r[0] for r in res],
                                                    [r[1] for r in res]], dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shifted_method_shards_whole_blocks():
    """The shifted scan reduces each unit's block once, so its shards hold whole blocks: over any
    number of ranks every block is on exactly one rank with all its energies, and the costs are
    one reduction plus the energies' O(N^2 nch) work."""
    b = _blocks()
    n1 = 5 * NR
    assert unit_cost(5, NR, 1, "shifted") == n1 ** 3 + n1 * n1 * 5
    assert unit_cost(5, NR, 1, "lu") == n1 ** 3
    for world in (1, 2, 3, 6):
        held = []
        for rank in range(world):
            mine, subs = shard_units(b, NR, rank, world, chunk=1, method="shifted")
            for (blk, idx), sub in zip(mine, subs):
                assert list(idx) == list(range(np.asarray(b[blk][2]).shape[0]))
                assert np.array_equal(sub[2], b[blk][2])
                held.append(blk)
        assert sorted(held) == list(range(len(b)))
    with pytest.raises(ValueError):
        unit_cost(2, NR, 1, "other")


def test_two_rank_gloo_sharded_scan_matches_single_process():
    blocks = _blocks()
    single, mine1 = run_sharded_scan(blocks, NR, _oracle_solve, chunk=None)
    assert [b for b, _ in mine1] == list(range(len(blocks)))
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "scan")
        mp.start_processes(_worker, args=(2, _free_port(), path), nprocs=2, start_method="spawn", join=True)
        outs = [np.load(path + f".{r}.npy", allow_pickle=True) for r in range(2)]
    mines = [list(o[0]) for o in outs]
    assert set(mines[0] + mines[1]) == set(range(len(blocks))) and mines[0] and mines[1]
    for o in outs:  # every rank holds every block's results after the gather
        for b in range(len(blocks)):
            np.testing.assert_array_equal(o[1][b], single[b][0])
            np.testing.assert_array_equal(o[2][b], single[b][1])


def test_more_ranks_than_units_leaves_some_ranks_empty():
    """With whole blocks as units and more ranks than blocks, the extra ranks get no unit (and
    solve nothing), every unit is still on exactly one rank, and a rank's results hold only
    its own blocks."""
    b = _blocks()
    world = len(b) + 2
    owners = []
    empty = 0
    for r in range(world):
        mine, subs = shard_units(b, NR, r, world, chunk=None)
        assert len(mine) == len(subs)
        empty += not mine
        owners += [u for u, _idx in mine]
    assert sorted(owners) == list(range(len(b))) and empty == 2
    res, mine = run_sharded_scan(b, NR, _oracle_solve, rank=world - 1, world=world, gather=False, chunk=None)
    assert all(r is None for r in res) == (not mine)
