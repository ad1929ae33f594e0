"""The multi-rank path on CPU: gloo ranks split a DEM's computable rows, each
computes only its own rows (here with the oracle's row-range sweep, the
test's stand-in for each rank's GPU), the rows are gathered, and the result is
the single-process run bit for bit; timings reduce to the max over ranks."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import load_oracle, load_package


def test_shard_rows_cover_the_grid(tvs):
    import total_viewsheds_b200.sharding as sh
    for h in (1, 7, 101, 1201):
        for world in (1, 2, 3, 8):
            ranges = [sh.shard_rows(h, r, world) for r in range(world)]
            assert ranges[0][0] == 0 and ranges[-1][1] == h
            assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
            sizes = [e - b for b, e in ranges]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        sh.shard_rows(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, z, out_dir):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        load_package()
        import total_viewsheds_b200.sharding as sh
        oracle = load_oracle()
        g = oracle.geometry(61, 5.0, 100)
        b, e = sh.shard_rows(g.tvs_height, rank, world)
        mine, mine_total = oracle.run_ex(g, z, 1.65, 0, 24, rows=(b, e), threads=1)
        assert mine.size == (e - b) * g.tvs_width
        full = sh.gather_rows(mine, g.tvs_width, g.tvs_height, world)
        full_total = sh.gather_rows(mine_total, g.tvs_width, g.tvs_height, world)
        t = sh.max_over_ranks(1.0 + rank)
        if rank == 0:
            np.save(os.path.join(out_dir, "full.npy"), full)
            np.save(os.path.join(out_dir, "total.npy"), full_total)
            np.save(os.path.join(out_dir, "tmax.npy"), np.array([t]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_compute_their_rows_and_reassemble(synth, oracle, tmp_path, world):
    z = synth.fbm(61, 61, 0.8, 5, 0.0, 300.0)
    mp.start_processes(_rank, args=(world, _free_port(), z, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    g = oracle.geometry(61, 5.0, 100)
    want, want_total, _ = oracle.run(g, z, 1.65, 0, 24, threads=1)
    full = np.load(tmp_path / "full.npy")
    assert np.array_equal(full.view(np.uint32), want.view(np.uint32))
    assert np.array_equal(np.load(tmp_path / "total.npy").view(np.uint32),
                          want_total.view(np.uint32))
    assert float(np.load(tmp_path / "tmax.npy")[0]) == float(world)
