"""Multi-process (gloo, world size 2, CPU) tests of the sharding logic: Monte Carlo path
ranges with one all-reduce reproduce the single-process payoff sums, and lattice
bin-packing with one gather reproduces every lattice's quotes.  The per-rank compute is
the CPU oracle here; on GPUs the same host logic drives the CUDA kernels."""
import math
import os
import socket

import numpy as np
import torch
import torch.multiprocessing as mp

from oplib_b200.shard import lpt_partition, path_range


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_path_range_covers_exactly():
    for npaths, world in [(1 << 20, 8), (1000, 3), (5, 8), (0, 2)]:
        seen = []
        for r in range(world):
            a, n = path_range(npaths, r, world)
            seen.extend(range(a, a + n))
        assert seen == list(range(npaths))


def test_lpt_partition_balances():
    rng = np.random.default_rng(20260)
    n = rng.choice(np.arange(256, 2049, 128), size=512)
    costs = (n.astype(float)) ** 3
    bins = lpt_partition(costs.tolist(), 8)
    assert sorted(i for b in bins for i in b) == list(range(512))
    loads = [costs[b].sum() for b in bins]
    assert max(loads) / (sum(loads) / 8) < 1.02


def _mc_worker(rank, world, port, out):
    import torch.distributed as dist
    from oplib_b200.shard import allreduce_sums, path_range
    from oracle import oracle as O
    from oracle import oracle_c as OC
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cfg = O.LVLattice(n=128)
    L, x = cfg.generator()
    niter, dt = O.plan_niter(L, 1 / 252, cfg.dt0)
    Cm = O.cumrows_f32(O.square(O.ek(L, dt), niter))
    a, n = path_range(3000, rank, world)
    disc = math.exp(-0.03 * 50 / 252)
    paths, s = OC.mc_paths(Cm, O.nearest_node(x), 5489, a, n, 50, x=x, disc=disc, nthreads=2)
    sums = torch.from_numpy(s)
    allreduce_sums(sums)
    out[rank] = sums.numpy().tolist()
    dist.destroy_process_group()


def test_mc_shards_reproduce_single_process():
    from oracle import oracle as O
    from oracle import oracle_c as OC
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_mc_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    cfg = O.LVLattice(n=128)
    L, x = cfg.generator()
    niter, dt = O.plan_niter(L, 1 / 252, cfg.dt0)
    Cm = O.cumrows_f32(O.square(O.ek(L, dt), niter))
    _, ref = OC.mc_paths(Cm, O.nearest_node(x), 5489, 0, 3000, 50, x=x, disc=math.exp(-0.03 * 50 / 252),
                         nthreads=1)
    for r in range(world):
        assert np.allclose(out[r], ref, rtol=1e-12)


def _batch_worker(rank, world, port, out):
    import torch.distributed as dist
    from oplib_b200.shard import gather_quotes, lpt_partition
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sizes = [64, 96, 128, 64, 160, 32, 96]
    bins = lpt_partition([float(n) ** 3 for n in sizes], world)
    local = []
    for i in bins[rank]:
        cfg = O.LVLattice(n=sizes[i], nmat=2, level=0.2 + 0.01 * i)
        L, x = cfg.generator()
        V, _, _ = O.solve_lattice_fp64(L, x, cfg.strikes[:8], cfg.r, cfg.period, cfg.nmat, cfg.dt0)
        local.append(V[:, O.nearest_node(x), :])
    q = gather_quotes(torch.from_numpy(np.stack(local)), bins, len(sizes))
    out[rank] = q.numpy()
    dist.destroy_process_group()


def test_batch_shards_gather_all_quotes():
    from oracle import oracle as O
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.spawn(_batch_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    sizes = [64, 96, 128, 64, 160, 32, 96]
    for i, n in enumerate(sizes):
        cfg = O.LVLattice(n=n, nmat=2, level=0.2 + 0.01 * i)
        L, x = cfg.generator()
        V, _, _ = O.solve_lattice_fp64(L, x, cfg.strikes[:8], cfg.r, cfg.period, cfg.nmat, cfg.dt0)
        for r in range(world):
            assert np.array_equal(out[r][i], V[:, O.nearest_node(x), :])
