#!/bin/sh
# Builds the CPU oracle (test infrastructure) into oracle/_build/.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$HERE/_build"
g++ -O2 -std=c++17 -fopenmp -ffp-contract=off -fno-fast-math -fPIC -shared \
  -o "$HERE/_build/liboracle.so" "$HERE/wx_oracle.cpp"
