#!/bin/sh
# Writes patched copies of the two reference files that do not compile for
# sm_100a into a temporary directory OUTSIDE the repository ($1):
#   util/Math.h: getRow() declares a local that shadows its parameter and reads
#     an undeclared `idx` (line 219); operator/ lacks a ';' (line 404);
#   rt/tracer/HipTracerBinKernels.cu: inline PTX uses `vote.ballot.b32` without
#     `.sync`, which ptxas rejects for sm_70 and later; it becomes
#     `vote.sync.ballot.b32` over the active lanes.
# Everything else is compiled from the reference tree where it lies.
# REF (the reference's src/hippie directory) is set by the Makefile.
set -e
: "${REF:?REF must name the reference's src/hippie directory}"
OUT=$1
mkdir -p "$OUT/util" "$OUT/tracer"
tr -d '\r' < "$REF/util/Math.h" \
  | sed -e 's/getRow(int r) const { Vec<T, L> r;/getRow(int idx) const { Vec<T, L> r;/' \
        -e 's/return operator\*(inverse(v))$/return operator*(inverse(v));/' > "$OUT/util/Math.h"
tr -d '\r' < "$REF/rt/tracer/HipTracerBinKernels.cu" \
  | sed -e 's/"vote\.ballot\.b32    %0,p;       \\n"/"activemask.b32 %0; vote.sync.ballot.b32 %0, p, %0; \\n"/' \
  > "$OUT/tracer/HipTracerBinKernels.cu"
grep -q "getRow(int idx)" "$OUT/util/Math.h"
grep -q "operator\*(inverse(v));" "$OUT/util/Math.h"
if grep -q "vote\.ballot\.b32" "$OUT/tracer/HipTracerBinKernels.cu"; then echo "tracer patch failed" >&2; exit 1; fi
