"""The partitioned operator through the device path: two ranks, each
building and applying its elements with the fused kernels, exchanging the
interface over gloo; against the oracle's global apply (1e-13) and a known
solution of the distributed PCG (1e-9)."""
import socket

import pytest

pytestmark = pytest.mark.gpu


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("nc,shape,P", [(1, (4, 4, 6), 4), (3, (3, 4, 5), 5)])
def test_partitioned_device_operator(fem, cuda, orc, nc, shape, P):
    import torch.multiprocessing as mp
    import shard_worker
    mp.spawn(shard_worker.run_device, args=(2, free_port(), nc, shape, P), nprocs=2, join=True)
