"""Point sharding across ranks: block bounds, and a 2-rank gloo run whose
gathered spectra equal the single-process result.  The per-block compute is a
stand-in (the oracle on the CPU) -- what is under test is the host logic
around it: bounds, padding, gather order."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from chaos_oneapi_b200.multi import shard_bounds


@pytest.mark.parametrize("P,world", [(10, 3), (4096, 8), (3, 4), (1, 2), (0, 2), (1000003, 7)])
def test_shard_bounds_cover_exactly(P, world):
    blocks = [shard_bounds(P, world, r) for r in range(world)]
    assert blocks[0][0] == 0 and blocks[-1][1] == P
    for (s0, e0), (s1, e1) in zip(blocks, blocks[1:]):
        assert e0 == s1
    sizes = [e - s for s, e in blocks]
    assert max(sizes) - min(sizes) <= 1 and sum(sizes) == P


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    import oracle
    from chaos_oneapi_b200.multi import run_sharded
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        params = oracle.make_grid(3, [10.0, 28.0, 8.0 / 3.0], [0, 5, 20, 3], [1, 0, 200, 5])
        inits = oracle.make_inits(3, params.shape[0], [1.0, 1.0, 1.0], 1e-3, 0, 4)

        def compute(p, x):
            s, _ = oracle.fixed("lorenz", "var", p, x, 1e-7, 0.01, 3, 1.0, 0.5, 2.0, 50.0,
                                threads=1)
            return s, np.zeros(len(p), dtype=np.int32)

        spec, status = run_sharded(params, inits, 3, compute)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), spec)
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_matches_single_process(tmp_path, orc):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    params = orc.make_grid(3, [10.0, 28.0, 8.0 / 3.0], [0, 5, 20, 3], [1, 0, 200, 5])
    inits = orc.make_inits(3, params.shape[0], [1.0, 1.0, 1.0], 1e-3, 0, 4)
    want, _ = orc.fixed("lorenz", "var", params, inits, 1e-7, 0.01, 3, 1.0, 0.5, 2.0, 50.0)
    for r in range(world):
        got = np.load(tmp_path / f"r{r}.npy")
        assert np.array_equal(got, want)
