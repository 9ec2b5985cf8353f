#!/bin/sh
# Test infrastructure (the checker), never shipped and never on the product path.
#
# Builds oracle/_ref/libmgref.so: the reference's own serial CPU correctness
# functions, compiled host-only with g++ from the reference tree where it lies.
# Nothing is copied into the repository: the four function bodies are cut out of
# the reference drivers by line range into oracle/_ref/ (git-ignored) and compiled
# together with oracle/ref_wrap.cpp, which adds a C ABI around them.
#
#   CPUBFS   Algorithms/BFS/bfs.cu:56-143
#   CPUSSSP  Algorithms/SSSP/sssp.cu:127-199
#   CPUCC    Algorithms/CC/cc.cu:132-199
#   CPUPR    Algorithms/PageRank/PageRank.cu:108-163
#
# plus the reference's Matrix Market ingest (b40c/graph/builder/market.cuh and
# b40c/graph/csr_graph.cuh), included straight from the reference tree.
#
# The reference's GPU engine is not built (CUDA 12 removed texture references and
# its arch flags stop at sm_35); only this CPU path compiles here.
set -e
REF="${MG_REFERENCE_DIR:-/root/reference}"
HERE="$(cd "$(dirname "$0")" && pwd)"
OUT="$HERE/_ref"
CUDA="${CUDA_HOME:-/usr/local/cuda}"

if [ ! -f "$REF/Algorithms/BFS/bfs.cu" ]; then
  echo "reference tree not found at $REF; oracle/_ref not rebuilt" >&2
  exit 3
fi
mkdir -p "$OUT"
sed -n '56,143p'  "$REF/Algorithms/BFS/bfs.cu"           > "$OUT/cpubfs.inc"
sed -n '127,199p' "$REF/Algorithms/SSSP/sssp.cu"         > "$OUT/cpusssp.inc"
sed -n '132,199p' "$REF/Algorithms/CC/cc.cu"             > "$OUT/cpucc.inc"
sed -n '108,163p' "$REF/Algorithms/PageRank/PageRank.cu" > "$OUT/cpupr.inc"

g++ -O3 -std=c++14 -shared -fPIC -w \
    -I"$REF" -I"$OUT" -I"$CUDA/include" \
    "$HERE/ref_wrap.cpp" -o "$OUT/libmgref.so" \
    -L"$CUDA/lib64" -lcudart_static -ldl -lrt -lpthread
echo "built $OUT/libmgref.so"
