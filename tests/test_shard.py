"""A mesh partitioned over ranks (fe_demo_cpp_b200/shard.py), world size 2
and 3 on gloo (CPU): each rank's apply plus the interface exchange equals the
global operator (1e-14), shared nodes hold the same bits on every rank, dots
count every DoF once, the exchanged diagonal is e_i^T M e_i, and the
distributed PCG recovers a known solution."""
import socket

import numpy as np
import pytest

from fe_demo_cpp_b200.mesh import box_mesh
from fe_demo_cpp_b200.shard import Shard, element_range


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_element_ranges_cover_the_mesh():
    for ne, world in [(10, 3), (7, 7), (1000, 8), (5, 2)]:
        spans = [element_range(ne, world, r) for r in range(world)]
        assert spans[0][0] == 0 and spans[-1][1] == ne
        assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
        assert max(b - a for a, b in spans) - min(b - a for a, b in spans) <= 1


def test_shard_interfaces_and_owners_single_process():
    """Without collectives: the peers' shared sets agree pairwise, and the
    owned masks partition the global nodes."""
    m = box_mesh((3, 2, 5), 3, seed=1)
    world = 3
    shards = [Shard(m.offsets, 27, world, r) for r in range(world)]
    owned = np.concatenate([s.l2g[s.owned] for s in shards])
    assert np.array_equal(np.sort(owned), np.arange(m.num_nodes))
    for a in shards:
        for q, idx in a.peers:
            b = shards[q]
            back = dict(b.peers)[a.rank]
            assert np.array_equal(a.l2g[idx], b.l2g[back])
    # the local numbering reproduces the global offsets of the rank's elements
    for s in shards:
        glob = m.offsets[s.e0 * 27:s.e1 * 27]
        assert np.array_equal(s.l2g[s.offsets], glob)


@pytest.mark.parametrize("world,nc,shape,P", [(2, 1, (3, 3, 4), 3), (2, 3, (2, 3, 4), 4), (3, 2, (3, 2, 5), 3)])
def test_partitioned_operator_on_gloo(world, nc, shape, P):
    import torch.multiprocessing as mp
    import shard_worker
    mp.spawn(shard_worker.run, args=(world, free_port(), nc, shape, P), nprocs=world, join=True)
