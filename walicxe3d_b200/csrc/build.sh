#!/bin/sh
# Builds libwx3d.so for sm_100a next to the package.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
OUT="$HERE/../libwx3d.so"
nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo -std=c++17 \
  -Xcompiler -fPIC -shared ${WX3D_NVCC_FLAGS:-} \
  -o "$OUT" "$HERE/wx3d_api.cu"
