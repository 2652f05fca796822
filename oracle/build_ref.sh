#!/usr/bin/env bash
# Compiles the reference's own CPU operators for the radix-partition / hash-join
# path straight from the read-only reference tree into oracle/_ref/libref_cpu.so.
#
# Test infrastructure only: the library is the checker for the oracle
# restatement (oracle/oracle.c) and the timed CPU baseline of bench.py.
# Nothing is copied out of the reference; the sources are compiled where they
# lie.  The reference normally generates `constants.h` from
# sql-ops/build.rs:74-120; this script writes the same values.
#
# Usage: oracle/build_ref.sh REFERENCE_ROOT
#    or: FI_REFERENCE_ROOT=... oracle/build_ref.sh
# Without either, or when the tree is absent, nothing is built.
set -euo pipefail

REF="${1:-${FI_REFERENCE_ROOT:-}}"
if [ -z "$REF" ]; then
  echo "build_ref: no reference root given; skipping" >&2
  exit 0
fi
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
SRC="$REF/sql-ops"

if [ ! -d "$SRC/cpputils" ]; then
  echo "build_ref: reference sources not found under $SRC; skipping" >&2
  exit 0
fi

mkdir -p "$OUT/include"
# sql-ops/build.rs:30-72 (x86_64 values): cache line 64 B, GPU cache line
# 128 B, ALIGN_BYTES 128, PADDING_BYTES 128, 32 banks, LASWWC 5 tuples/thread.
cat > "$OUT/include/constants.h" << 'EOF'
#define CACHE_LINE_SIZE 64U
#define GPU_CACHE_LINE_SIZE 128U
#define ALIGN_BYTES 128U
#define LOG2_NUM_BANKS 5U
#define LASWWC_TUPLES_PER_THREAD 5U
EOF

# Fixed ISA level instead of -march=native, because the library is built once
# and may run on another machine: x86-64-v4 = AVX-512, so the reference's SWWC
# flush takes its AVX-512 streaming-store path
# (sql-ops/cpputils/radix_partition.cpp:170-176).  Override with
# FI_REF_ISA=-march=x86-64-v3 on an AVX2-only host.
ISA="${FI_REF_ISA:--march=x86-64-v4}"

g++ -std=c++14 -O3 $ISA -fPIC -shared -DNO_WARN_X86_INTRINSICS \
  -I "$SRC/include" -I "$OUT/include" \
  "$SRC/cpputils/radix_partition.cpp" \
  "$SRC/cpputils/gpu_common.cpp" \
  "$SRC/cpputils/no_partitioning_join.cpp" \
  -o "$OUT/libref_cpu.so"

echo "build_ref: wrote $OUT/libref_cpu.so"
