#!/usr/bin/env bash
# Builds oracle/_ref/libaltoref.so: the UNMODIFIED reference (IntelLabs/ALTO)
# compiled in place from its own sources, plus oracle/ref_harness.cpp.
# Test infrastructure only (golden fixtures, CPU baseline timing).
#
# The reference builds with -march=native.  The library built here must run
# on other hosts, so it is built twice: libaltoref.so for x86-64-v3 (AVX2 +
# BMI2) and libaltoref_avx512.so for x86-64-v4 (AVX-512); oracle/orc.py loads
# the AVX-512 one on hosts whose CPU has those instructions.
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]
# (default: $ALTOB_REFERENCE_ROOT, else /root/reference)
# The reference needs cblas/LAPACK; the prototype-only headers in
# oracle/ref_shim/ declare them and the OpenBLAS shared library bundled with
# the Python environment provides them (DT_RPATH, so its own libgfortran
# dependency resolves from the same directory).
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${1:-${ALTOB_REFERENCE_ROOT:-/root/reference}}"
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
build() {  # $1: -march value, $2: output name, $3...: extra flags
    local march="$1" out="$2"
    shift 2
    g++ -O3 -march="$march" -mbmi2 -fopenmp -std=c++17 -fPIC -shared \
        -include typeinfo -D_GLIBCXX_PARALLEL -DUSE_OPENBLAS_ \
        -DMAX_NUM_MODES=5 -DALTO_MODES_SPECIALIZED=0,3,4,5 \
        -DALTO_RANKS_SPECIALIZED=0,8,16,100 "$@" \
        -I"$HERE/ref_shim" -I"$REF/include" \
        -w \
        "$HERE/ref_harness.cpp" "$REF/src/kruskal_model.cpp" \
        "$REF/src/sptensor.cpp" "$REF/src/common.cpp" \
        -o "$OUT/$out" \
        -L"$BLASDIR" -l:"$(basename "$BLASLIB")" -Wl,--disable-new-dtags -Wl,-rpath,"$BLASDIR"
    echo "built $OUT/$out (-march=$march $*; BLAS: $(basename "$BLASLIB"))"
}
build x86-64-v3 libaltoref.so &
p1=$!
build x86-64-v4 libaltoref_avx512.so &
p2=$!
# the reference's ALT_PEXT build (alto.hpp:212-244): keys re-encoded with each
# mode's bits contiguous
build x86-64-v3 libaltoref_pext.so -DALT_PEXT &
p3=$!
# the OPT_ALTO build (alto.hpp:838-868): partition subspace ids
build x86-64-v3 libaltoref_opt.so -DOPT_ALTO &
p5=$!
# the reference's Poisson generator (src/poisson_generator.cpp, rng.cpp,
# rng_stream.cpp) for the generator's parity tests; floating-point
# contraction off so that uniform(low, high) = x * (high - low) + low rounds
# twice, as written, on every host
g++ -O3 -march=x86-64-v3 -ffp-contract=off -fopenmp -std=c++17 -fPIC -shared \
    -include typeinfo -DUSE_OPENBLAS_ -DMAX_NUM_MODES=5 \
    -I"$HERE/ref_shim" -I"$REF/include" -w \
    "$HERE/ref_poisson.cpp" "$REF/src/poisson_generator.cpp" "$REF/src/rng.cpp" \
    "$REF/src/rng_stream.cpp" "$REF/src/kruskal_model.cpp" "$REF/src/sptensor.cpp" \
    "$REF/src/common.cpp" \
    -o "$OUT/libaltoref_poisson.so" \
    -L"$BLASDIR" -l:"$(basename "$BLASLIB")" -Wl,--disable-new-dtags -Wl,-rpath,"$BLASDIR" &
p4=$!
wait $p1
wait $p2
wait $p3
wait $p4
wait $p5
echo "built $OUT/libaltoref_poisson.so (-ffp-contract=off)"
