#!/bin/bash
# ORACLE build of the reference's own solver core (test infrastructure).
# Compiles the reference sources where they lie (read-only) with the shim
# headers in oracle/shim/ and links them with oracle/ref_adapter.cpp into
# oracle/_ref/libmaquis_ref.so.  The reference's CUDA numeric kernels are
# compiled too because tasks.cpp references them; they are never called.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
if [ -z "${MAQUIS_REFERENCE:-}" ]; then
  MAQUIS_REFERENCE="$(python -c 'import json, sys; print(json.load(open(sys.argv[1])).get("reference_path", ""))' "$HERE/../BASELINE.json" 2>/dev/null || true)"
fi
[ -n "$MAQUIS_REFERENCE" ] || { echo "set MAQUIS_REFERENCE to the reference source tree" >&2; exit 1; }
REF="$MAQUIS_REFERENCE/dmrg/framework"
OUT="$HERE/_ref"
[ -d "$REF/dmrg/solver" ] || { echo "reference sources not found at $REF" >&2; exit 1; }
mkdir -p "$OUT"
BLAS_DIR="$(python -c 'import scipy, os; print(os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs"))')"
BLAS_LIB="$(basename "$(ls "$BLAS_DIR"/libscipy_openblas-*.so | head -1)")"
CXX="g++ -std=c++17 -O2 -fPIC -fopenmp -DMAQUIS_OPENMP -include cstdint -I$HERE/shim -I$REF -I/usr/local/cuda/include"
for f in tasks accelerator vector_stage; do
  $CXX -c "$REF/dmrg/solver/$f.cpp" -o "$OUT/$f.o"
done
for f in gpu_dgemm_ddot gpu_vgemm; do
  /usr/local/cuda/bin/nvcc -std=c++17 -O2 -Xcompiler -fPIC -gencode arch=compute_100a,code=sm_100a \
      -I"$HERE/shim" -I"$REF" -c "$REF/dmrg/solver/numeric/$f.cu" -o "$OUT/$f.o"
done
$CXX -c "$HERE/ref_adapter.cpp" -o "$OUT/ref_adapter.o"
$CXX -c "$HERE/ref_flatten.cpp" -o "$OUT/ref_flatten.o"
g++ -shared -fopenmp -o "$OUT/libmaquis_ref.so" "$OUT"/*.o -L"$BLAS_DIR" -l:"$BLAS_LIB" -Wl,-rpath,"$BLAS_DIR" \
    -L/usr/local/cuda/lib64 -lcudart -lcublas -Wl,-rpath,/usr/local/cuda/lib64
rm -f "$OUT"/*.o
echo "$OUT/libmaquis_ref.so"
