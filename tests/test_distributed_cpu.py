"""Multi-GPU sharding logic on the CPU: tile-pair shards and the one all-reduce, with gloo ranks.

Each rank of a 2-process gloo group computes its shard of the upper-triangle tile pairs with a NumPy
restatement of the pair loop (FP64, L2SF, squared-edge bins), the shards are added with the package's
all-reduce helper, and the sum must equal the unsharded computation: counts exactly, sums to
rounding. The shard arithmetic itself (the library's partition, sfb200_shard_bounds, which needs no
GPU) is checked for every small case: the shards tile the tile pairs and hold equal pair counts to
within one tile pair.
"""
import math
import os
import socket

import numpy as np
import pytest

from sfb200.distributed import shard_bounds, shard_value, tile_pair_pairs

T = 32


def tile_pairs(n):
    nt = (n + T - 1) // T
    return [(ti, tj) for ti in range(nt) for tj in range(ti, nt)]


def histogram_of_tile_pairs(x, u, sqedges, pairs):
    """(sums, counts) of L2SF over the listed tile pairs (i < j inside a diagonal tile)."""
    n = x.shape[1]
    nb = len(sqedges) - 1
    sums = np.zeros(nb)
    counts = np.zeros(nb, dtype=np.int64)
    for ti, tj in pairs:
        i = np.arange(ti * T, min(n, ti * T + T))
        j = np.arange(tj * T, min(n, tj * T + T))
        I, J = np.meshgrid(i, j, indexing="ij")
        keep = (J > I) if ti == tj else np.ones_like(I, dtype=bool)
        I, J = I[keep], J[keep]
        dx = x[:, J] - x[:, I]
        du = u[:, J] - u[:, I]
        r2 = np.sum(dx * dx, axis=0)
        p = np.sum(dx * du, axis=0)
        b = np.searchsorted(sqedges, r2, side="left") - 1
        ok = (b >= 0) & (b < nb)
        v = p[ok] * p[ok] / r2[ok]
        sums += np.bincount(b[ok], weights=v, minlength=nb)
        counts += np.bincount(b[ok], minlength=nb)
    return sums, counts


@pytest.mark.parametrize("count", [1, 2, 3, 7, 8])
def test_shard_bounds_partition_the_tile_pairs(count):
    for n in (0, 1, 2, 31, 32, 33, 300, 1000, 8256):
        nt = (n + T - 1) // T
        tp = tile_pairs(n)
        ntp = nt * (nt + 1) // 2
        assert len(tp) == ntp
        bounds = [shard_bounds(n, T, k, count) for k in range(count)]
        assert bounds[0][0] == 0 and bounds[-1][1] == ntp
        for (a0, a1), (b0, b1) in zip(bounds, bounds[1:]):
            assert a1 == b0 and a0 <= a1
        # each shard within one tile pair of its exact share
        work = [sum(tile_pair_pairs(n, T, *tp[p]) for p in range(lo, hi)) for lo, hi in bounds]
        assert sum(work) == n * (n - 1) // 2
        if n > T:
            assert max(work) - min(work) <= 2 * T * T, (n, count, work)


def test_shard_bounds_balance_pairs_at_the_benchmark_size():
    """65536 points in 256-point tiles over 8 shards: equal tile-pair counts would differ by the
    diagonal tiles' half-empty blocks; balanced by pairs each shard is within one tile pair of its
    exact share (so two shards differ by less than two)."""
    n, tile = 65536, 256
    nt = n // tile
    for count in (2, 4, 8):
        work = []
        for k in range(count):
            lo, hi = shard_bounds(n, tile, k, count)
            # rows are contiguous: count the pairs of [lo, hi) row by row
            w, p = 0, 0
            for ti in range(nt):
                row = nt - ti
                a, b = max(lo, p), min(hi, p + row)
                if a < b:
                    w += (b - a) * tile * tile - (tile * tile - tile * (tile - 1) // 2 if a == p else 0)
                p += row
            work.append(w)
        assert sum(work) == n * (n - 1) // 2
        share = n * (n - 1) // 2 / count
        assert all(abs(w - share) <= tile * tile for w in work), (count, work)


def test_shard_value_encoding():
    assert shard_value(0, 1) == 1 << 32
    assert shard_value(3, 8) == (8 << 32) | 3
    with pytest.raises(ValueError):
        shard_value(2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist

    from sfb200.distributed import allreduce_histogram

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        n = 300
        x = rng.random((2, n))
        u = rng.standard_normal((2, n))
        edges = np.exp(np.linspace(math.log(1e-2), math.log(math.sqrt(2.0)), 9))
        sq = edges * edges
        tp = tile_pairs(n)
        lo, hi = shard_bounds(n, T, rank, world)
        s, c = histogram_of_tile_pairs(x, u, sq, tp[lo:hi])
        st = torch.from_numpy(s)
        ct = torch.from_numpy(c)
        allreduce_histogram(st, ct)
        np.savez(os.path.join(out_dir, f"rank{rank}.npz"), sums=st.numpy(), counts=ct.numpy(),
                 ref_sums=histogram_of_tile_pairs(x, u, sq, tp)[0], ref_counts=histogram_of_tile_pairs(x, u, sq, tp)[1])
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_add_up_to_the_full_histogram(tmp_path):
    torch = pytest.importorskip("torch")
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    for r in range(world):
        d = np.load(tmp_path / f"rank{r}.npz")
        assert np.array_equal(d["counts"], d["ref_counts"])
        assert int(d["counts"].sum()) > 0
        np.testing.assert_allclose(d["sums"], d["ref_sums"], rtol=1e-12, atol=0)
