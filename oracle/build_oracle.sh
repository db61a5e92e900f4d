#!/bin/sh
# Builds the CPU restatement (oracle/tpcf_oracle.c) into oracle/lib/.
# TEST INFRASTRUCTURE ONLY.  -ffp-contract=off keeps every float operation
# singly rounded, as in the reference's x86-64 SSE code.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$HERE/lib"
${TPCF_CC:-gcc} -O3 -std=c11 -fopenmp -ffp-contract=off -fPIC -shared "$HERE/tpcf_oracle.c" \
    -o "$HERE/lib/libtpcf_oracle.so.tmp" -lm
mv "$HERE/lib/libtpcf_oracle.so.tmp" "$HERE/lib/libtpcf_oracle.so"
