#!/bin/sh
# Builds the parity oracle from the reference's own, unmodified sources.
#
# TEST INFRASTRUCTURE ONLY.  Compiles the reference translation units where
# they lie (src/*.cpp except main.cpp, and the vendored src/healpix/*.cpp)
# together with oracle/ref_harness.cpp into two shared libraries under
# oracle/_ref/ (git-ignored; they travel with the working tree):
#
#   libtwopcf_ref_plain.so  default build: -D_ANGULAR_PI_DEFN -D_N_MASK_INTS=1
#   libtwopcf_ref_invp.so   inverse-p build: + -D_HAVE_HDF5 -D_USE_INV_WEIGHTS
#                           -D_N_MASK_INTS=32, linked against the in-memory
#                           HDF5 stand-in in oracle/hdf5_stub/ (libhdf5 is not
#                           installed here)
#   twopcf_ref              the reference's own command-line program (plain
#                           build, src/main.cpp included), for end-to-end
#                           comparisons of parameter file -> ASCII outputs
#
# Flags follow the reference makefile (makefile:3-7) with g++ in place of icc
# (icc is not available): -O3 -std=c++11 -fopenmp.  -ffp-contract=off keeps
# every float/double operation singly rounded (no FMA contraction), which is
# what x86-64 SSE code generation gives by default; no -march flags are used.
#
# The reference tree is read from $TPCF_REFERENCE_DIR (default
# /root/reference); nothing is written there.  Shipped .o files in the
# reference are never used.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${TPCF_REFERENCE_DIR:-/root/reference}
OUT="$HERE/_ref"
CXX=${TPCF_CXX:-g++}

if [ ! -f "$REF/src/correlators.cpp" ]; then
    echo "build_ref.sh: reference sources not found under $REF; keeping any prebuilt oracle/_ref" >&2
    exit 0
fi
mkdir -p "$OUT"

SRCS="$REF/src/boxes.cpp $REF/src/correlators.cpp $REF/src/correlators_invpweight.cpp \
      $REF/src/cosmology.cpp $REF/src/dataset.cpp $REF/src/galaxy.cpp $REF/src/hist.cpp \
      $REF/src/io.cpp $REF/src/healpix/error_handling.cpp $REF/src/healpix/healpix_base.cpp \
      $REF/src/healpix/pointing.cpp $REF/src/healpix/geom_utils.cpp \
      $REF/src/healpix/healpix_tables.cpp $REF/src/healpix/string_utils.cpp"
FLAGS="-O3 -std=c++11 -fopenmp -ffp-contract=off -fPIC -shared -w -D_ANGULAR_PI_DEFN"

$CXX $FLAGS -D_N_MASK_INTS=1 -I"$REF/src" -I"$REF/src/healpix" \
    "$HERE/ref_harness.cpp" $SRCS -o "$OUT/libtwopcf_ref_plain.so.tmp"
mv "$OUT/libtwopcf_ref_plain.so.tmp" "$OUT/libtwopcf_ref_plain.so"

$CXX $FLAGS -D_HAVE_HDF5 -D_USE_INV_WEIGHTS -D_N_MASK_INTS=32 -I"$HERE/hdf5_stub" -I"$REF/src" \
    -I"$REF/src/healpix" "$HERE/ref_harness.cpp" "$HERE/hdf5_stub/hdf5_stub.cpp" $SRCS \
    -o "$OUT/libtwopcf_ref_invp.so.tmp"
mv "$OUT/libtwopcf_ref_invp.so.tmp" "$OUT/libtwopcf_ref_invp.so"
$CXX -O3 -std=c++11 -fopenmp -ffp-contract=off -w -D_ANGULAR_PI_DEFN -D_N_MASK_INTS=1 -I"$REF/src" \
    -I"$REF/src/healpix" "$REF/src/main.cpp" $SRCS -o "$OUT/twopcf_ref.tmp"
mv "$OUT/twopcf_ref.tmp" "$OUT/twopcf_ref"
echo "built $OUT/libtwopcf_ref_plain.so $OUT/libtwopcf_ref_invp.so $OUT/twopcf_ref"
