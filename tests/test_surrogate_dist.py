"""Data-parallel surrogate training on CPU: world size 2 over gloo.

The U-Net gradient hook (gradenna_b200.unet.allreduce_mean) must leave every
rank with the mean of the ranks' flat gradients, so that the identical Adam
step keeps the replicas equal; the field targets of a rank re-expressed in
the ranks' common scale must equal targets computed with that scale."""

import os
import socket

import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    from gradenna_b200.unet import allreduce_mean

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        g = torch.arange(10, dtype=torch.float32) * (rank + 1)
        allreduce_mean()(g)
        out[rank] = g.tolist()
    finally:
        dist.destroy_process_group()


def test_gradient_hook_averages_over_ranks():
    port = _free_port()
    out = mp.Manager().dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn")
    want = [1.5 * i for i in range(10)]
    assert out[0] == want and out[1] == want


def test_field_targets_rescale_to_common_scale():
    ez = torch.randn(4, 5, 5, 2, dtype=torch.float64) * 3.0
    own, common = 0.7, 1.9
    t_own = torch.asinh(ez / own)
    t_common = torch.asinh(torch.sinh(t_own) * (own / common))
    torch.testing.assert_close(t_common, torch.asinh(ez / common), rtol=1e-12, atol=1e-12)
