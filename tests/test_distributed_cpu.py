"""Multi-GPU sharding logic on the CPU: tile-pair shards and the one all-reduce, with gloo ranks.

Each rank of a 2-process gloo group computes its shard of the upper-triangle tile pairs with a NumPy
restatement of the pair loop (FP64, L2SF, squared-edge bins), the shards are added with the package's
all-reduce helper, and the sum must equal the unsharded computation: counts exactly, sums to
rounding. The shard arithmetic itself (the library's partition) is checked for every small case.
"""
import math
import os
import socket

import numpy as np
import pytest

from sfb200.distributed import shard_bounds, shard_value

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
    for ntp in (0, 1, 5, 36, 1000, 8256):
        bounds = [shard_bounds(ntp, k, count) for k in range(count)]
        assert bounds[0][0] == 0 and bounds[-1][1] == ntp
        for (a0, a1), (b0, b1) in zip(bounds, bounds[1:]):
            assert a1 == b0 and a0 <= a1
        sizes = [hi - lo for lo, hi in bounds]
        assert max(sizes) - min(sizes) <= 1


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
        lo, hi = shard_bounds(len(tp), rank, world)
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
