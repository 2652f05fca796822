"""Radix join of relations sharded over several GPUs (one process per GPU,
torch.distributed for the plumbing).

The reference has no multi-GPU path.  Radix partitioning is the exchange
step of a distributed hash join: every rank partitions its shards of R and
S on g = log2(world size) exchange bits that lie above the bits of the local
join, an all-to-all moves partition d to rank d, and every rank then joins
what it received with the single-GPU engine; an all-reduce adds the ranks'
{sum, count} (int64, wrapping).  Tuples with equal keys meet on one rank, so
the result equals the single-GPU join of the whole relations.

    dist.init_process_group("nccl", ...)        # one process per GPU
    s, c = exchange_join(rk, rp, sk, sp, bits=(9, 9))

The grouping by destination is the library's radix partitioner (a
Contiguous pass on the exchange bits); the all-to-all is NCCL's.  The
exchange moves each tuple once over NVLink; a fused partition + peer-store
kernel is the next step (it needs several GPUs to test).
"""
import torch
import torch.distributed as dist


def exchange_bits(world):
    g = world.bit_length() - 1
    if world < 1 or (1 << g) != world:
        raise ValueError("the exchange needs a power-of-two world size, got %d" % world)
    return g


def destinations(keys, shift, g):
    """key_to_partition on bits [shift, shift + g): (u64(key) >> shift) &
    (2^g - 1), int32 keys sign-extended as in the kernels (an arithmetic
    shift gives the same low g bits while shift + g <= 64)."""
    return (keys.to(torch.int64) >> shift) & ((1 << g) - 1)


def gpu_group_by_destination(keys, pays, shift, g):
    """Tuples (AoS, [n, 2]) grouped by destination rank and the count per
    destination, with the library's Contiguous radix partitioner."""
    import fi_sqlops as fi
    n = keys.numel()
    F = 1 << g
    if g == 0 or n == 0:
        return torch.stack([keys, pays], 1).contiguous(), \
            torch.tensor([n], dtype=torch.int64, device=keys.device)
    sms = torch.cuda.get_device_properties(keys.device).multi_processor_count
    p = fi.GpuRadixPartitioner(fi.GpuHistogramAlgorithm.Contiguous,
                               fi.GpuRadixPartitionAlgorithm.SSWWCv2,
                               fi.RadixBits(shift, g), sms, 1024)
    o = fi.PartitionOffsets(fi.GpuHistogramAlgorithm.Contiguous, sms, g, keys.dtype)
    rel = fi.PartitionedRelation(n, fi.GpuHistogramAlgorithm.Contiguous, g, sms,
                                 keys.dtype)
    p.prefix_sum(fi.RadixPass.Second, keys, o)
    p.partition(fi.RadixPass.Second, keys, pays, o, rel)
    # partition d spans [off[d], off[d+1] - pad); the last ends at the
    # padded length (partitioned_relation.rs:510-537)
    pad = fi.padding_len(keys.dtype)
    off = rel.offsets[:F].tolist()
    ends = [o - pad for o in off[1:]] + [rel.padded_len()]
    parts = [rel.relation[b:e] for b, e in zip(off, ends)]
    counts = torch.tensor([len(x) for x in parts], dtype=torch.int64,
                          device=keys.device)
    return torch.cat(parts).contiguous(), counts


def shuffle(keys, pays, shift, group=None, group_by=gpu_group_by_destination):
    """Sends every tuple to the rank given by its key bits [shift, shift+g)
    and returns the (keys, payloads) this rank received."""
    world = dist.get_world_size(group)
    g = exchange_bits(world)
    tuples, counts = group_by(keys, pays, shift, g)
    recv = torch.empty_like(counts)
    dist.all_to_all_single(recv, counts, group=group)
    out = tuples.new_empty((int(recv.sum().item()), 2))
    dist.all_to_all_single(out, tuples, output_split_sizes=recv.tolist(),
                           input_split_sizes=counts.tolist(), group=group)
    return out[:, 0].contiguous(), out[:, 1].contiguous()


def gpu_local_join(rk, rp, sk, sp, bits, scheme):
    import fi_sqlops as fi
    e = fi.RadixJoinEngine(max(rk.numel(), 1), max(sk.numel(), 1), rk.dtype,
                           fi.RadixBits(*bits), scheme)
    s, c = e.run(rk, rp, sk, sp)
    e.status()
    return s, c


def exchange_join(rk, rp, sk, sp, bits=(9, 9), scheme=None, group=None,
                  group_by=gpu_group_by_destination, local_join=gpu_local_join):
    """Join of R and S sharded over the ranks: exchange on the bits above
    the local join's, join locally, add up.  Returns (sum, count) of the
    whole join on every rank."""
    if scheme is None:
        import fi_sqlops as fi
        scheme = fi.HashingScheme.BucketChaining
    shift = sum(bits)
    rk2, rp2 = shuffle(rk, rp, shift, group, group_by)
    sk2, sp2 = shuffle(sk, sp, shift, group, group_by)
    s, c = local_join(rk2, rp2, sk2, sp2, bits, scheme)
    t = torch.tensor([s, c], dtype=torch.int64, device=rk.device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return int(t[0].item()), int(t[1].item())
