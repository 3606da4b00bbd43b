#!/bin/sh
# Builds the CPU oracle (test infrastructure) into oracle/_build/:
#   libvshe_oracle.so     the single-threaded restatement of the SHE path (she_oracle.cpp) and
#                         of the outer loop's Poisson system (poisson_oracle.cpp);
#   libvshe_oracle_mt.so  the reference's serial ILU(0) + BiCGStab on all host threads
#                         (serial_solver_mt.cpp), for bench.py's reference arm and CPU baseline.
# -ffp-contract=off: no FMA contraction, the arithmetic a default x86-64 build of
# the reference performs.
set -e
HERE="$(cd "$(dirname "$0")" && pwd)"
mkdir -p "$HERE/_build"
g++ -std=c++17 -O2 -ffp-contract=off -fPIC -shared -Wall -Wextra -Wno-unused-parameter \
    -o "$HERE/_build/libvshe_oracle.so" "$HERE/she_oracle.cpp" "$HERE/poisson_oracle.cpp"
g++ -std=c++17 -O2 -ffp-contract=off -fopenmp -fPIC -shared -Wall -Wextra -Wno-unused-parameter \
    -o "$HERE/_build/libvshe_oracle_mt.so" "$HERE/serial_solver_mt.cpp"
echo "built $HERE/_build/libvshe_oracle.so $HERE/_build/libvshe_oracle_mt.so"
