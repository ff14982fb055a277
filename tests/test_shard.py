"""CPU: block sharding over two gloo ranks (the multi-GPU halo plan).

Each rank owns half of the blocks of a periodic 2x2x2 layout, builds its
share of the level's gather table and fills its ghosts with one grouped
point-to-point round; the result must equal, bit for bit, the single-rank
fill (the table applied to the whole level), and the block-ordered norm
reduction must equal the single-rank sum.  No GPU is touched."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

W, P = 4, 5
LAYOUTS = [((2, 2, 2), (8, 8, 8), [P, P, W, W, W, W], 2), ((3, 2, 1), (8, 4, 8), [P] * 6, 2)]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _level(blocks, g, seed):
    rng = np.random.default_rng(seed)
    s = 2 ** (g - 1)
    return [rng.standard_normal((d.n[2] // s + 2, d.n[1] // s + 2, d.n[0] // s + 2)) for d in blocks]


def _rank(rank, world, port, layout, out):
    import torch.distributed as tdist
    from datetime import timedelta
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    tdist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import hydro3d_b200 as h3d
        from hydro3d_b200 import shard
        nblk, n, bc, ngrid = layout
        blocks = h3d.topology.block_grid(nblk, n, bc, [1 / 16.0] * 3, ngrid)
        owner = shard.partition(blocks, world)
        res = {}
        for g in range(1, ngrid + 1):
            lev = _level(blocks, g, 7 + g)
            mine = np.concatenate([a.ravel() for a, o in zip(lev, owner) if o == rank])
            plan = shard.build_plan(blocks, g, 0, owner, rank)
            shard.exchange(plan, mine, tdist)
            sums = {b: np.array([float((a * a).sum()), float(a.sum())]) for b, (a, o) in enumerate(zip(lev, owner))
                    if o == rank}
            tot = shard.reduce_block_sums(sums, len(blocks), tdist)
            res[g] = (mine, tot, len(plan.send_idx), len(plan.recv_idx))
        out[rank] = res
        tdist.barrier()
    finally:
        tdist.destroy_process_group()


@pytest.mark.parametrize("layout", LAYOUTS)
def test_two_rank_halo_fill_matches_single_rank(h3d, layout):
    from hydro3d_b200 import shard
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_rank, args=(r, world, port, layout, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        codes = [p.exitcode for p in procs]
        for p in procs:
            if p.is_alive():
                p.terminate()
                p.join(10)
        assert codes == [0, 0], codes
        res = dict(out)
    nblk, n, bc, ngrid = layout
    blocks = h3d.topology.block_grid(nblk, n, bc, [1 / 16.0] * 3, ngrid)
    owner = shard.partition(blocks, world)
    assert sorted(set(owner)) == [0, 1]
    for g in range(1, ngrid + 1):
        lev = _level(blocks, g, 7 + g)
        flat = np.concatenate([a.ravel() for a in lev])
        dst, src = h3d.halo_table(blocks, g, 0)
        want = flat.copy()
        want[dst] = flat[src & 0x7FFFFFFF]
        sizes = [a.size for a in lev]
        starts = np.concatenate([[0], np.cumsum(sizes)])
        tot = np.zeros(2)
        for a in lev:
            tot = tot + np.array([float((a * a).sum()), float(a.sum())])
        for r in range(world):
            mine, rtot, nsend, nrecv = res[r][g]
            exp = np.concatenate([want[starts[b]:starts[b + 1]] for b, o in enumerate(owner) if o == r])
            assert np.array_equal(mine, exp), (g, r)
            assert np.array_equal(rtot, tot)
            assert nsend >= 1 and nrecv >= 1


def test_partition_balances_cells():
    from hydro3d_b200 import shard

    class D:
        def __init__(self, n):
            self.n = n
    blocks = [D((64, 64, 64))] * 5 + [D((32, 32, 32))] * 8
    own = shard.partition(blocks, 4)
    assert own == sorted(own) and set(own) == {0, 1, 2, 3}
    cells = np.zeros(4)
    for d, o in zip(blocks, own):
        cells[o] += np.prod(d.n)
    assert cells.max() <= 2.0 * cells.mean()
