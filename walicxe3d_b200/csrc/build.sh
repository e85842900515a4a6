#!/bin/sh
# Builds libwx3d.so for sm_100a next to the package.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/../libwx3d.so"
TMP="$HERE/../_build"
mkdir -p "$TMP"
FLAGS="-gencode arch=compute_100a,code=sm_100a -O3 -lineinfo -std=c++17 -Xcompiler -fPIC -Xcompiler -fopenmp ${WX3D_NVCC_FLAGS:-}"
nvcc $FLAGS -c -o "$TMP/wx3d_api.o" "$HERE/wx3d_api.cu" &
P1=$!
nvcc $FLAGS -c -o "$TMP/wx3d_mlp.o" "$HERE/wx3d_mlp.cu" &
P2=$!
wait $P1
wait $P2
nvcc -gencode arch=compute_100a,code=sm_100a -shared -Xcompiler -fopenmp -o "$OUT" "$TMP/wx3d_api.o" "$TMP/wx3d_mlp.o" -lgomp
