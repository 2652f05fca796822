#!/usr/bin/env python
"""Tuning sweep of the autotuner: measures every candidate plan of the radix
join on one GPU and writes the table that fi_autotune_load reads.

For each (tuple type, log2 |R|, log2 k, skew) of the grid, with
|S| = k |R|, R a seeded permutation of 1..|R| and S foreign keys (uniform, or
Zipf 1.0 when skewed), every candidate plan -- total radix bits around the
model's choice, one or two passes, bucket chaining, join blocks of 256, 512
and 1024 threads, TMA-fed or register-fed scatters -- runs on one engine and
the fastest correct one is kept.  Perfect hashing is not a candidate: it is
valid only for dense unique build keys, which the server cannot assume.

    python fast-interconnects_b200/autotune.py [--out tuning_table.txt]
        [--log2r 16,18,20,22,24,26,28] [--log2k 0,2,4] [--reps 3]
"""
import argparse
import os
import sys
import time

import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import fi_sqlops as fi  # noqa: E402


def candidates(log2r):
    """Radix-bit plans around about 4K build tuples per final partition."""
    base = max(0, log2r - 12)
    out = set()
    for total in range(max(0, base - 1), base + 3):
        if total <= 11:
            out.add((total,))
        if total >= 8:
            for b1 in range((total + 1) // 2 - 1, (total + 1) // 2 + 2):
                b2 = total - b1
                if 0 <= b1 <= 12 and 0 <= b2 <= 10:
                    out.add((b1, b2))
    return sorted(out)


def time_plan(e, cols, reps):
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    e.run_async(*cols)
    t0.record()
    for _ in range(reps):
        e.run_async(*cols)
    t1.record()
    torch.cuda.synchronize()
    return t0.elapsed_time(t1) / reps


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "tuning_table.txt"))
    ap.add_argument("--log2r", default="16,18,20,22,24,26,28")
    ap.add_argument("--log2k", default="0,2,4")
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    lines = ["# tuple_bytes log2_build log2_ratio skew bits1 bits2 scheme "
             "join_block scatter   (ms of the winner; measured by autotune.py)"]
    for tb, dt in ((8, torch.int32), (16, torch.int64)):
        for lr in [int(x) for x in a.log2r.split(",")]:
            for lk in [int(x) for x in a.log2k.split(",")]:
                rn, sn = 1 << lr, 1 << (lr + lk)
                if (rn + sn) * tb > 40e9:
                    continue
                for skew in (0, 1):
                    rk = torch.empty(rn, dtype=dt, device="cuda")
                    sk = torch.empty(sn, dtype=dt, device="cuda")
                    fi.gen_primary_keys(rk, 11)
                    if skew:
                        fi.gen_zipf_foreign_keys(sk, rn, 1.0, 12, 11)
                    else:
                        fi.gen_uniform_foreign_keys(sk, rn, 12)
                    exp = (int(sk.to(torch.int64).sum().item()), sn)
                    e = fi.RadixJoinEngine(rn, sn, dt, fi.RadixBits(12, 10),
                                           fi.HashingScheme.BucketChaining)
                    best = None
                    for bits in candidates(lr):
                        for jb in (256, 512, 1024):
                            for sc in (0, 1):
                                e.set_plan(fi.RadixBits(*bits),
                                           fi.HashingScheme.BucketChaining, jb, sc)
                                if e.run(rk, rk, sk, sk) != exp:
                                    raise SystemExit("wrong result for plan %s" % (bits,))
                                ms = time_plan(e, (rk, rk, sk, sk), a.reps)
                                if best is None or ms < best[0]:
                                    best = (ms, bits, jb, sc)
                    ms, bits, jb, sc = best
                    b2 = bits[1] if len(bits) > 1 else -1
                    lines.append("%d %d %d %d %d %d %d %d %d   # %.3f ms" % (
                        tb, lr, lk, skew, bits[0], b2, int(fi.HashingScheme.BucketChaining),
                        jb, sc, ms))
                    print(lines[-1], flush=True)
                    del e, rk, sk
                    torch.cuda.empty_cache()
    with open(a.out, "w") as f:
        f.write("\n".join(lines) + "\n")
    print("wrote", a.out)


if __name__ == "__main__":
    main()
