#!/usr/bin/env bash
# Builds oracle/_ref/libaltoref.so: the UNMODIFIED reference (IntelLabs/ALTO)
# compiled in place from its own sources, plus oracle/ref_harness.cpp.
# Test infrastructure only (golden fixtures, CPU baseline timing).
#
# -march=x86-64-v3 (AVX2 + BMI2) instead of the reference's -march=native so
# the library also runs on hosts other than the one that built it.
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]   (default /root/reference)
# The reference needs cblas/LAPACK; the prototype-only headers in
# oracle/ref_shim/ declare them and the OpenBLAS shared library bundled with
# the Python environment provides them (DT_RPATH, so its own libgfortran
# dependency resolves from the same directory).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF/include/alto.hpp" ]; then
    echo "reference sources not found under $REF" >&2
    exit 3
fi
PY=$(command -v python3 || command -v python)
SITE=$("$PY" -c 'import sysconfig; print(sysconfig.get_paths()["purelib"])')
BLASDIR=$(ls -d "$SITE"/opencv_python_headless.libs 2>/dev/null || true)
BLASLIB=$(ls "$BLASDIR"/libopenblasp-r0-*.so 2>/dev/null | head -1 || true)
if [ -z "$BLASLIB" ]; then
    echo "OpenBLAS shared library not found in $SITE" >&2
    exit 4
fi
mkdir -p "$OUT"
g++ -O3 -march=x86-64-v3 -mbmi2 -fopenmp -std=c++17 -fPIC -shared \
    -include typeinfo -D_GLIBCXX_PARALLEL -DUSE_OPENBLAS_ \
    -DMAX_NUM_MODES=5 -DALTO_MODES_SPECIALIZED=0,3,4,5 \
    -DALTO_RANKS_SPECIALIZED=0,8,16,100 \
    -I"$HERE/ref_shim" -I"$REF/include" \
    -w \
    "$HERE/ref_harness.cpp" "$REF/src/kruskal_model.cpp" \
    "$REF/src/sptensor.cpp" "$REF/src/common.cpp" \
    -o "$OUT/libaltoref.so" \
    -L"$BLASDIR" -l:"$(basename "$BLASLIB")" -Wl,--disable-new-dtags -Wl,-rpath,"$BLASDIR"
echo "built $OUT/libaltoref.so (BLAS: $(basename "$BLASLIB"))"
