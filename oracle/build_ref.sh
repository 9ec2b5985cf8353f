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
HERE="$(cd "$(dirname "$0")" && pwd)"
# The reference checkout: MG_REFERENCE_DIR, else "reference" beside this repository.
REF="${MG_REFERENCE_DIR:-$(cd "$HERE/../.." && pwd)/reference}"
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

# MapGraph's own bundled vertex programs (Algorithms/*/*.h, unchanged) compiled
# against the compat GASengine headers of this repository and linked with the
# engine library: oracle/_ref/gas_ref_tuned dispatches them to the tuned entry
# points, oracle/_ref/gas_ref_generic runs them on the generic kernels.
ROOT="$(cd "$HERE/.." && pwd)"
LIBDIR="$ROOT/mirrorofmapgraph_b200/lib"
if [ -x "$CUDA/bin/nvcc" ] && [ -f "$LIBDIR/libmapgraph_b200.so" ]; then
  for mode in tuned generic; do
    flag=""
    [ "$mode" = generic ] && flag="-DMG_GAS_GENERIC_ONLY"
    "$CUDA/bin/nvcc" -gencode arch=compute_100a,code=sm_100a -std=c++17 -O2 -w -Xcompiler -fpermissive $flag \
        -I"$ROOT/include/compat" -I"$ROOT/include" -I"$REF" "$ROOT/tests/cpp/gas_ref_programs.cu" \
        -o "$OUT/gas_ref_$mode" -L"$LIBDIR" -lmapgraph_b200 -Xlinker -rpath -Xlinker '$ORIGIN/../../mirrorofmapgraph_b200/lib'
  done
  echo "built $OUT/gas_ref_tuned $OUT/gas_ref_generic"
fi
