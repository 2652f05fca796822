"""Generates the golden fixtures in tests/golden/ by running the reference's
own CPU operators, compiled from the reference sources by
oracle/build_ref.sh into oracle/_ref/libref_cpu.so:

* cpu_chunked_prefix_sum_int{32,64}      (sql-ops/cpputils/radix_partition.cpp:228-267)
* cpu_chunked_radix_partition_*          (radix_partition.cpp:409-446, NC)
* cpu_chunked_radix_partition_swwc_*     (radix_partition.cpp:491-557, SWWC)
* cpu_ht_{build,probe_aggregate}_*       (sql-ops/cpputils/no_partitioning_join.cpp)

The join-pinning cases (``join_pin_*``) hold build and probe columns with
misses, duplicate build keys, negative keys and payloads, and keys that leave
most radix partitions empty.  Their expected sums come from the reference's
linear-probing join (no_partitioning_join.cpp:27-140), which adds s.value once
for every build tuple whose key equals the probe key: the same quantity the
radix join aggregates (sql-ops/cudautils/radix_join.cu:199-311).  The match
count is the same join run with every probe payload set to 1.

Inputs are stored explicitly (not regenerated), so the fixtures pin the
oracle on machines where the reference tree is absent.

Usage:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle as O  # noqa: E402


JOIN_PIN_KINDS = ("misses", "duplicates", "negative", "sparse")


def join_pin_inputs(kind, dt, rng, nb, npr):
    """Build and probe columns (key, payload) of one join-pinning case.

    misses     unique build keys 0..nb-1, probe keys over 0..2nb-1: about
               half of the probe tuples find no partner
    duplicates build keys drawn from 0..nb/4-1 (about four copies each):
               every copy matches
    negative   keys and payloads over the whole signed range (the null key
               -1 left out): sign extension through key_to_partition and the
               wrapping sum
    sparse     unique build keys that are multiples of 64: with up to 6
               radix bits all but one partition are empty
    """
    info = np.iinfo(dt)
    pay_lo, pay_hi = int(info.min), int(info.max)
    if kind == "misses":
        rk = rng.permutation(nb)
        sk = rng.integers(0, 2 * nb, npr)
    elif kind == "duplicates":
        rk = rng.integers(0, nb // 4, nb)
        sk = rng.integers(0, nb // 2, npr)
    elif kind == "negative":
        rk = rng.integers(info.min, info.max, nb, endpoint=True)
        rk[rk == -1] = -2
        hit = rng.integers(0, nb, npr)
        fresh = rng.integers(info.min, info.max, npr, endpoint=True)
        sk = np.where(rng.random(npr) < 0.6, rk[hit], fresh)
        sk[sk == -1] = -3
    elif kind == "sparse":
        rk = rng.permutation(nb) * 64
        sk = rng.integers(0, 2 * nb, npr) * 64
    else:
        raise ValueError(kind)
    rp = rng.integers(pay_lo, pay_hi, nb, endpoint=True)
    sp = rng.integers(pay_lo, pay_hi, npr, endpoint=True)
    return (rk.astype(dt), rp.astype(dt), sk.astype(dt), sp.astype(dt))


def ref_join_sum_count(rk, rp, sk, sp):
    """(wrapping sum of matched probe payloads, match count) from the
    reference's compiled linear-probing join."""
    entries = 1 << int(2 * len(rk) - 1).bit_length()
    s, _ = O.ref_ht_linearprobing_sum(rk, rp, sk, sp, entries)
    c, _ = O.ref_ht_linearprobing_sum(rk, rp, sk, np.ones_like(sp), entries)
    return s, c


def main():
    if not O.ref_available():
        O.build()
    assert O.ref_available(), "the reference library could not be built"
    rng = np.random.default_rng(20261203)
    out = {}
    for dt, name in ((np.int32, "i32"), (np.int64, "i64")):
        n = 1001
        keys = rng.permutation(n).astype(dt) + 1
        pays = rng.integers(-1000, 1000, n).astype(dt)
        out["%s_keys" % name] = keys
        out["%s_pays" % name] = pays
        for chunks, bits in ((1, 0), (3, 4), (7, 6), (4, 9)):
            off = O.ref_chunked_prefix_sum(keys, chunks, bits)
            out["%s_offsets_c%d_b%d" % (name, chunks, bits)] = off
            rel = O.ref_chunked_radix_partition(keys, pays, off, chunks, bits,
                                                swwc=False)
            out["%s_nc_c%d_b%d" % (name, chunks, bits)] = rel
            rel_s = O.ref_chunked_radix_partition(keys, pays, off, chunks, bits,
                                                  swwc=True)
            out["%s_swwc_c%d_b%d" % (name, chunks, bits)] = rel_s
        fk = rng.integers(1, n + 1, 2003).astype(dt)
        fpay = rng.integers(-50, 50, 2003).astype(dt)
        out["%s_fk" % name] = fk
        out["%s_fpay" % name] = fpay
        s_lp, _ = O.ref_ht_linearprobing_sum(keys, pays, fk, fpay, 1 << 13)
        s_pf, _ = O.ref_ht_perfect_sum(keys, pays, fk, fpay, n + 1)
        out["%s_lp_sum" % name] = np.array([s_lp], np.uint64)
        out["%s_perfect_sum" % name] = np.array([s_pf], np.uint64)
    pin_rng = np.random.default_rng(20261204)
    for kind in JOIN_PIN_KINDS:
        for dt, name in ((np.int32, "i32"), (np.int64, "i64")):
            rk, rp, sk, sp = join_pin_inputs(kind, dt, pin_rng, 1500, 3001)
            pre = "join_pin_%s_%s_" % (kind, name)
            out[pre + "r_key"], out[pre + "r_pay"] = rk, rp
            out[pre + "s_key"], out[pre + "s_pay"] = sk, sp
            ssum, scnt = ref_join_sum_count(rk, rp, sk, sp)
            out[pre + "sum"] = np.array([ssum], np.uint64)
            out[pre + "count"] = np.array([scnt], np.uint64)
    path = os.path.join(HERE, "reference_cpu_ops.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
