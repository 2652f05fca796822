"""The u64 prefix scans (the reference's scan test exports,
sql-ops/tests/test_prefix_scan.rs) against numpy: block-wise and
device-wide, with and without the per-thread padding term."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
M64 = (1 << 64) - 1


def expected(data, threads, padding):
    n = len(data)
    out = np.zeros(n, dtype=object)
    ti = -(-n // threads) if n else 1
    run = 0
    for j in range(n):
        out[j] = (run + (j // ti + 1) * padding) & M64
        run = (run + int(data[j])) & M64
    return out


def to_u64(t):
    return np.array([int(x) & M64 for x in t.cpu().numpy().tolist()], dtype=object)


@pytest.mark.parametrize("n,grid,block", [(1024, 1, 1024), (4096, 4, 1024),
                                          (1000, 3, 256), (777, 1, 32)])
@pytest.mark.parametrize("padding", [0, 5])
def test_block_exclusive_prefix_sum(fi, n, grid, block, padding):
    g = torch.Generator().manual_seed(n + grid)
    data = torch.randint(-(1 << 62), 1 << 62, (n,), generator=g, dtype=torch.int64)
    d = data.cuda()
    fi.block_exclusive_prefix_sum(d, padding, grid, block)
    got = to_u64(d)
    src = [int(x) & M64 for x in data.tolist()]
    bs = n // grid
    for b in range(grid):
        seg = src[b * bs:(b + 1) * bs]
        assert list(got[b * bs:(b + 1) * bs]) == list(expected(seg, block, padding))
    assert list(got[grid * bs:]) == src[grid * bs:]  # the remainder is left alone


@pytest.mark.parametrize("n,grid,block", [(1 << 20, 148, 1024), (1_000_003, 296, 512),
                                          (64, 2, 32), (0, 4, 128)])
@pytest.mark.parametrize("padding", [0, 3])
def test_device_exclusive_prefix_sum(fi, n, grid, block, padding):
    data = torch.randint(0, 1 << 40, (n,), dtype=torch.int64)
    d = data.cuda()
    fi.device_exclusive_prefix_sum(d, padding, grid, block)
    if padding == 0:
        exp = torch.cumsum(data, 0) - data
        assert torch.equal(d.cpu(), exp)
    else:
        src = data.numpy()
        ex = np.concatenate([[0], np.cumsum(src)[:-1]]) if n else src
        ti = -(-n // (grid * block)) if n else 1
        owner = np.arange(n) // ti
        assert np.array_equal(d.cpu().numpy(), ex + (owner + 1) * padding)


def test_state_len(fi):
    assert fi.prefix_sum_state_len(148, 1024) == 148 * 1024 // 32 + 32
