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

Two exchanges move each tuple once over NVLink:
 * exchange="nccl": the library's radix partitioner groups the tuples by
   destination (a Contiguous pass on the exchange bits), then NCCL's
   all-to-all sends them;
 * exchange="peer" (PeerExchange): one fused kernel partitions and stores
   every tuple straight into the destination rank's receive columns, which
   every rank maps by CUDA IPC.  The ranks' counts are all-gathered first,
   so each sender owns a fixed region of every receiver's columns; no
   kernel waits on another rank (the host orders the steps).
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


def region_bases(counts, rank):
    """counts[s][d] = tuples sender s sends to rank d (a W x W list or
    tensor).  Returns (base, recv): base[d] = first slot of `rank`'s region
    in d's receive columns (the tuples of senders s < rank come first) and
    recv[d] = tuples d receives in all."""
    rows = [[int(x) for x in row] for row in (counts.tolist() if hasattr(counts, "tolist")
                                               else counts)]
    w = len(rows)
    base = [sum(rows[s][d] for s in range(rank)) for d in range(w)]
    recv = [sum(rows[s][d] for s in range(w)) for d in range(w)]
    return base, recv


def all_gather_counts(counts, group=None):
    """The W x W count matrix (row s = sender s's counts) on every rank;
    device tensors under NCCL, host tensors otherwise."""
    world = dist.get_world_size(group)
    if dist.get_backend(group) != "nccl":
        counts = counts.cpu()
    out = counts.new_empty(world * counts.numel())
    dist.all_gather_into_tensor(out, counts.contiguous(), group=group)
    return out.view(world, counts.numel()).cpu()


_opened = {}  # IPC handle -> [mapped base pointer, users]: one mapping per allocation


def _ipc_open(handle):
    import fi_sqlops as fi
    ent = _opened.get(handle)
    if ent is None:
        ent = _opened[handle] = [fi.ipc_open(handle), 0]
    ent[1] += 1
    return ent[0]


def _ipc_release(handle):
    import fi_sqlops as fi
    ent = _opened[handle]
    ent[1] -= 1
    if ent[1] == 0:
        del _opened[handle]
        fi.ipc_close(ent[0])


class PeerExchange:
    """Receive columns of `capacity` tuples on every rank (keys, then
    payloads, in one allocation), mapped into every other rank by CUDA IPC.
    shuffle() sends each tuple to the rank given by its key bits
    [shift, shift + g) with one fused partition + peer-store kernel and
    returns the (keys, payloads) this rank received.

    Order of a shuffle: histogram -> all-gather of the counts (a rendezvous:
    no rank sends before every rank has finished with its columns) ->
    capacity check on the shared matrix (every rank raises alike) -> fused
    scatter -> synchronize -> all-reduce of the senders' status (every
    sender is done; an error on any rank raises on every rank) -> read."""

    def __init__(self, capacity, dtype, group=None, device=None):
        import fi_sqlops as fi
        self.group = group
        self.world = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.g = exchange_bits(self.world)
        self.capacity = capacity
        dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.buf = torch.empty((2, max(capacity, 1)), dtype=dtype, device=dev)
        self.keys, self.pays = self.buf[0], self.buf[1]
        self.cursors = torch.empty(1 << self.g, dtype=torch.int64, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        handle, off = fi.ipc_handle(self.buf)
        peers = [None] * self.world
        dist.all_gather_object(peers, (handle, off, capacity), group=group)
        self.handles, self.dests = [], []
        for r, (h, o, cap) in enumerate(peers):
            if r == self.rank:
                self.dests.append((self.keys.data_ptr(), self.pays.data_ptr(), cap))
            else:
                base = _ipc_open(h)
                self.handles.append(h)
                pstep = max(cap, 1) * self.buf.element_size()
                self.dests.append((base + o, base + o + pstep, cap))

    def shuffle(self, keys, pays, shift):
        import fi_sqlops as fi
        counts = fi.exchange_histogram(keys, shift, self.g)
        mat = all_gather_counts(counts, self.group)
        base, recv = region_bases(mat, self.rank)
        caps = [d[2] for d in self.dests]
        if any(n > c for n, c in zip(recv, caps)):
            raise fi.SqlOpsError(-7, "a rank receives %d tuples; its exchange holds %d"
                                 % max(zip(recv, caps), key=lambda x: x[0] - x[1]))
        dests = [(k, p, b, c) for (k, p, c), b in zip(self.dests, base)]
        fi.exchange_scatter(keys, pays, shift, self.g, dests, self.cursors,
                            self.status)
        if self.buf.is_cuda:
            torch.cuda.synchronize()
        # every sender is done; a status recorded by any sender fails every
        # rank alike (a receiver's columns are incomplete then)
        st = self.status.to(torch.int32).reshape(1).clone()
        if dist.get_backend(self.group) != "nccl":
            st = st.cpu()
        dist.all_reduce(st, op=dist.ReduceOp.MIN, group=self.group)
        code = int(st.item())
        if code != 0:
            self.status.zero_()
            raise fi.SqlOpsError(code, "exchange scatter recorded an error on a rank")
        n = recv[self.rank]
        return self.keys[:n], self.pays[:n]

    def close(self):
        """Unmaps the peers' columns once every rank is done with them."""
        if self.handles:
            if self.buf.is_cuda:
                torch.cuda.synchronize()
            dist.barrier(group=self.group)
            for h in self.handles:
                _ipc_release(h)
            self.handles = []


def shard_primary_keys(pk, world, rank):
    """Rank `rank`'s shard of a primary-key column spread over `world`
    ranks: a permutation `pk` of 1..n becomes key = (pk - 1) * world + rank
    + 1 (in place), so the shards of all ranks together are a permutation
    of 1..world * n and no key is on two ranks."""
    return pk.sub_(1).mul_(world).add_(rank + 1)


class EngineJoin:
    """Local join for exchange_join that keeps one RadixJoinEngine (sized for
    at most max_build x max_probe tuples) across calls, instead of
    allocating an engine per join."""

    def __init__(self, max_build, max_probe, dtype, bits, scheme):
        import fi_sqlops as fi
        self.engine = fi.RadixJoinEngine(max(max_build, 1), max(max_probe, 1), dtype,
                                         fi.RadixBits(*bits), scheme)

    def __call__(self, rk, rp, sk, sp, bits, scheme):
        s, c = self.engine.run(rk, rp, sk, sp)
        self.engine.status()
        return s, c


def gpu_local_join(rk, rp, sk, sp, bits, scheme):
    import fi_sqlops as fi
    e = fi.RadixJoinEngine(max(rk.numel(), 1), max(sk.numel(), 1), rk.dtype,
                           fi.RadixBits(*bits), scheme)
    s, c = e.run(rk, rp, sk, sp)
    e.status()
    return s, c


def exchange_join(rk, rp, sk, sp, bits=(9, 9), scheme=None, group=None,
                  group_by=gpu_group_by_destination, local_join=gpu_local_join,
                  exchange="peer", peers=None):
    """Join of R and S sharded over the ranks: exchange on the bits above
    the local join's, join locally, add up.  Returns (sum, count) of the
    whole join on every rank.  exchange="peer" (the default) uses the fused
    kernel through `peers` = (PeerExchange for R, PeerExchange for S),
    created here (and closed again) when not given; exchange="nccl" groups
    with `group_by` and moves the tuples with NCCL's all-to-all (also the
    path for CPU tensors under gloo)."""
    if scheme is None:
        import fi_sqlops as fi
        scheme = fi.HashingScheme.BucketChaining
    shift = sum(bits)
    if exchange == "peer":
        own = peers is None
        if own:  # receive columns sized to the largest share of each relation
            import fi_sqlops as fi
            g = exchange_bits(dist.get_world_size(group))
            rank = dist.get_rank(group)
            caps = [max(region_bases(all_gather_counts(
                fi.exchange_histogram(k, shift, g), group), rank)[1])
                for k in (rk, sk)]
            peers = (PeerExchange(caps[0], rk.dtype, group),
                     PeerExchange(caps[1], sk.dtype, group))
        try:
            rk2, rp2 = peers[0].shuffle(rk, rp, shift)
            sk2, sp2 = peers[1].shuffle(sk, sp, shift)
            s, c = local_join(rk2, rp2, sk2, sp2, bits, scheme)
        finally:
            if own:
                for p in peers:
                    p.close()
    elif exchange == "nccl":
        rk2, rp2 = shuffle(rk, rp, shift, group, group_by)
        sk2, sp2 = shuffle(sk, sp, shift, group, group_by)
        s, c = local_join(rk2, rp2, sk2, sp2, bits, scheme)
    else:
        raise ValueError("exchange must be 'nccl' or 'peer', got %r" % (exchange,))
    dev = rk.device if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.tensor([s, c], dtype=torch.int64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return int(t[0].item()), int(t[1].item())
