"""Generates the golden fixtures in tests/golden/ by running the reference's
own CPU operators, compiled from the reference sources by
oracle/build_ref.sh into oracle/_ref/libref_cpu.so:

* cpu_chunked_prefix_sum_int{32,64}      (sql-ops/cpputils/radix_partition.cpp:228-267)
* cpu_chunked_radix_partition_*          (radix_partition.cpp:409-446, NC)
* cpu_chunked_radix_partition_swwc_*     (radix_partition.cpp:491-557, SWWC)
* cpu_ht_{build,probe_aggregate}_*       (sql-ops/cpputils/no_partitioning_join.cpp)

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
    path = os.path.join(HERE, "reference_cpu_ops.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
