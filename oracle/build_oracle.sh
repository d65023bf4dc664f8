#!/usr/bin/env bash
# Builds the CPU oracle (test infrastructure only) into oracle/lib/liboracle_acoular.so.
# -ffp-contract=off keeps the C arithmetic in the reference's (numba, no fastmath) order.
set -euo pipefail
here="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
mkdir -p "$here/lib"
gcc -O3 -march=x86-64-v3 -fopenmp -fPIC -shared -ffp-contract=off -fno-fast-math -std=c11 \
    -o "$here/lib/liboracle_acoular.so.tmp" "$here/oracle_core.c" -lm
mv "$here/lib/liboracle_acoular.so.tmp" "$here/lib/liboracle_acoular.so"
