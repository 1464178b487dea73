#!/usr/bin/env bash
# Builds the reference program (Marco-Mendivil-Carboni/Spin-Glass, Program/src)
# for sm_100a into oracle/_ref/ (git-ignored), for timing it on the same B200 as
# the engine and for recording its outputs as test fixtures.  Only the
# compile-time constants of eamsim.cuh change: the lattice side L and the
# sweeps per invocation SPFILE (the reference fixes both at compile time,
# eamsim.cuh:13,22); everything else is the reference as shipped.
# Usage: bash oracle/build_ref.sh [reference root] [L] [SPFILE]
# The reference root defaults to $CSG_REFERENCE_ROOT, else to a directory
# named "reference" beside this repository.
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${1:-${CSG_REFERENCE_ROOT:-$HERE/../../reference}}
L=${2:-16}
SPFILE=${3:-16384}
OUT="$HERE/_ref"
SRC="$OUT/src_L${L}"
[ -f "$REF/Program/src/eamsim.cu" ] || { echo "no reference at $REF" >&2; exit 1; }
mkdir -p "$SRC"
cp "$REF"/Program/src/*.cu "$REF"/Program/src/*.cuh "$SRC"/
sed -i -E "s/static constexpr int L = [0-9]+;/static constexpr int L = ${L};/; s/static constexpr int SPFILE = [0-9]+;/static constexpr int SPFILE = ${SPFILE};/" "$SRC/eamsim.cuh"
grep -q "static constexpr int L = ${L};" "$SRC/eamsim.cuh"
grep -q "static constexpr int SPFILE = ${SPFILE};" "$SRC/eamsim.cuh"
BIN="$OUT/csg_ref_L${L}"
[ "$SPFILE" = 16384 ] || BIN="${BIN}_S${SPFILE}"
nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o "$BIN" \
    "$SRC/util.cu" "$SRC/eamsim.cu" "$SRC/main.cu" -lcurand
echo "$BIN"
