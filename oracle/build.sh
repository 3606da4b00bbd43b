#!/bin/sh
# Builds the CPU oracle (test infrastructure) into oracle/_build/libvshe_oracle.so.
# -ffp-contract=off: no FMA contraction, the arithmetic a default x86-64 build of
# the reference performs.
set -e
HERE="$(cd "$(dirname "$0")" && pwd)"
mkdir -p "$HERE/_build"
g++ -std=c++17 -O2 -ffp-contract=off -fPIC -shared -Wall -Wextra -Wno-unused-parameter \
    -o "$HERE/_build/libvshe_oracle.so" "$HERE/she_oracle.cpp"
echo "built $HERE/_build/libvshe_oracle.so"
