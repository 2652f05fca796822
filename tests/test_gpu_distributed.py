"""The exchange join's GPU pieces on one GPU: the grouping of tuples by
destination rank with the library's partitioner, and the whole
exchange_join over a one-rank NCCL group (ranks that wait on each other on
one GPU are not run; the multi-rank logic is covered on CPU by
test_distributed.py)."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist

from _helpers import to_dev

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dt", [torch.int32, torch.int64])
@pytest.mark.parametrize("g,shift", [(1, 8), (3, 18), (2, 0)])
def test_group_by_destination(fi, dt, g, shift):
    import distributed as D
    n = (1 << 20) + 77
    keys = torch.empty(n, dtype=dt, device="cuda")
    fi.gen_primary_keys(keys, 31)
    pays = keys * 3
    tuples, counts = D.gpu_group_by_destination(keys, pays, shift, g)
    d = D.destinations(keys, shift, g)
    assert counts.tolist() == torch.bincount(d, minlength=1 << g).tolist()
    assert tuples.shape == (n, 2)
    got_d = D.destinations(tuples[:, 0], shift, g)
    assert bool((got_d[1:] >= got_d[:-1]).all())  # grouped by destination
    assert bool((tuples[:, 1] == tuples[:, 0] * 3).all())
    assert torch.equal(torch.sort(tuples[:, 0]).values, torch.sort(keys).values)


def test_exchange_join_one_rank_nccl(fi, oracle):
    import distributed as D
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        n = 1 << 20
        r = oracle.primary_keys(n, 41, np.int64)
        s = oracle.uniform_foreign_keys(2 * n, 2 * n, 42, np.int64)
        got = D.exchange_join(to_dev(r), to_dev(r), to_dev(s), to_dev(s), bits=(6, 6),
                              exchange="nccl")
    finally:
        dist.destroy_process_group()
    exp_s, exp_c, _, _ = oracle.cpu_radix_join(r, r.copy(), s, s.copy(), 6, 6, 4,
                                               use_reference=False)
    assert got == ((exp_s + (1 << 63)) % (1 << 64) - (1 << 63), exp_c)
