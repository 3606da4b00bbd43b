#!/bin/sh
# Compiles the drop-in adapter harness (tests/adapter/adapter_check.cpp) against the reference's
# own headers into tests/adapter/_build/libadapter_check.so, linked to libvshe_b200.so.
# Usage: tests/adapter/build.sh [viennashe-dev root]  (default: $VIENNASHE_REF_ROOT, else
# /root/reference).  Exits 3 without building when the reference headers are absent.
set -e
HERE="$(cd "$(dirname "$0")" && pwd)"
ROOT="$(cd "$HERE/../.." && pwd)"
REF="${1:-${VIENNASHE_REF_ROOT:-/root/reference}}"
if [ ! -f "$REF/viennashe/solvers/config.hpp" ]; then
  echo "reference headers not found under $REF"
  exit 3
fi
mkdir -p "$HERE/_build"
g++ -std=c++11 -O1 -fPIC -shared -Wall -Wno-unused-parameter -Wno-unused-variable -Wno-unused-but-set-variable \
    -Wno-deprecated-declarations \
    -I"$ROOT/viennashe-dev_b200/adapter" -I"$ROOT/include" -I"$REF" -I"$ROOT/oracle/ref_stub/grid" \
    -o "$HERE/_build/libadapter_check.so" "$HERE/adapter_check.cpp" \
    -L"$ROOT/viennashe-dev_b200/lib" -lvshe_b200 -Wl,-rpath,'$ORIGIN/../../../viennashe-dev_b200/lib'
echo "built $HERE/_build/libadapter_check.so"
