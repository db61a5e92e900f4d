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
#   libtwopcf_ref_midpoint.so        plain build without -D_ANGULAR_PI_DEFN (pi
#                                    along x1 + x2, src/correlators.cpp:172-182)
#   libtwopcf_ref_invp_dither.so     inverse-p build with -D_USE_DITHER_WEIGHTS
#   libtwopcf_ref_invp4.so           inverse-p build with -D_N_MASK_INTS=4
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
BASE="-O3 -std=c++11 -fopenmp -ffp-contract=off -fPIC -shared -w"
INVP="-D_HAVE_HDF5 -D_USE_INV_WEIGHTS -I$HERE/hdf5_stub"
INC="-I$REF/src -I$REF/src/healpix"

# build <output name> <flags...>: one shared library of the harness and the
# reference sources; the builds run in parallel and each is checked.
build() {
    name=$1
    shift
    stub=""
    case "$*" in *_USE_INV_WEIGHTS*) stub="$HERE/hdf5_stub/hdf5_stub.cpp" ;; esac
    $CXX $BASE "$@" $INC "$HERE/ref_harness.cpp" $stub $SRCS -o "$OUT/$name.tmp" && mv "$OUT/$name.tmp" "$OUT/$name"
}

build libtwopcf_ref_plain.so -D_ANGULAR_PI_DEFN -D_N_MASK_INTS=1 & p1=$!
build libtwopcf_ref_invp.so -D_ANGULAR_PI_DEFN $INVP -D_N_MASK_INTS=32 & p2=$!
build libtwopcf_ref_midpoint.so -D_N_MASK_INTS=1 & p3=$!
build libtwopcf_ref_invp_dither.so -D_ANGULAR_PI_DEFN $INVP -D_USE_DITHER_WEIGHTS -D_N_MASK_INTS=32 & p4=$!
build libtwopcf_ref_invp4.so -D_ANGULAR_PI_DEFN $INVP -D_N_MASK_INTS=4 & p5=$!
$CXX -O3 -std=c++11 -fopenmp -ffp-contract=off -w -D_ANGULAR_PI_DEFN -D_N_MASK_INTS=1 $INC \
    "$REF/src/main.cpp" $SRCS -o "$OUT/twopcf_ref.tmp" && mv "$OUT/twopcf_ref.tmp" "$OUT/twopcf_ref" & p6=$!
rc=0
for p in $p1 $p2 $p3 $p4 $p5 $p6; do wait $p || rc=1; done
if [ $rc -ne 0 ]; then
    echo "build_ref.sh: a reference build failed" >&2
    exit 1
fi
echo "built $(ls "$OUT" | tr '\n' ' ')"
