#!/usr/bin/env bash
# Builds the CPU oracle (test infrastructure) into oracle/liboracle.so.
# x86-64-v3 (AVX2 + FMA) so the library also runs on the GPU hosts' CPUs.
set -euo pipefail
here="$(cd "$(dirname "$0")" && pwd)"
g++ -O3 -march=x86-64-v3 -std=c++17 -fPIC -shared -pthread \
    -o "$here/liboracle.so" "$here/dpg_oracle.cpp"
