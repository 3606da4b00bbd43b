#!/bin/sh
# Compiles the reference's own scalar physics (oracle/ref_physics.cpp, which includes the
# reference's headers where they lie) into oracle/_ref/libvshe_ref.so, to pin the oracle's
# restatement.  Usage: oracle/build_ref.sh [viennashe-dev root] (default: $VIENNASHE_REF_ROOT, else
# /root/reference).  Exits 3 without building when the reference headers are absent.
# -ffp-contract=off: no FMA contraction, as the oracle.
set -e
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${VIENNASHE_REF_ROOT:-/root/reference}}"
if [ ! -f "$REF/viennashe/physics/dispersion.hpp" ]; then
  echo "reference headers not found under $REF"
  exit 3
fi
mkdir -p "$HERE/_ref"
g++ -std=c++11 -O2 -ffp-contract=off -fPIC -shared -w \
    -I"$HERE/ref_stub/cfg" -I"$REF" -I"$HERE/ref_stub/grid" \
    -o "$HERE/_ref/libvshe_ref.so" "$HERE/ref_physics.cpp"
echo "built $HERE/_ref/libvshe_ref.so"
