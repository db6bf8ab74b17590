#!/usr/bin/env bash
# Builds the CPU oracle (test infrastructure): oracle/liboracle.so (FP64) and
# oracle/liboracle_xp.so (the same source with __float128 arithmetic, the
# extended-precision truth).  x86-64-v3 (AVX2 + FMA) so the libraries also run on
# the GPU hosts' CPUs.
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
flags=(-O3 -march=x86-64-v3 -std=gnu++17 -ffp-contract=off -fPIC -shared -pthread -Wl,-Bsymbolic)
g++ "${flags[@]}" -o "$here/liboracle.so" "$here/dpg_oracle.cpp"
g++ "${flags[@]}" -DORC_QUAD -o "$here/liboracle_xp.so" "$here/dpg_oracle.cpp" -lquadmath
