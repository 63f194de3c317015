#!/usr/bin/env bash
# Test infrastructure only: compiles the reference tblis-strassen library from its
# own sources (read in place, never copied into the repository) into
# oracle/_ref/libtblis_ref.so, for use as the parity checker and the timed CPU
# baseline.  Nothing in the product links or loads this library.
#
# The reference's autotools build is not run.  Instead this script
#   1. writes the handful of configure-time headers (tblis_config.h,
#      tci_config.h, configs/foreach_*.h, configs/include_configs.hpp) for the
#      "sandybridge" + "reference" configurations with pthreads threading,
#      exactly the values configure would pick for
#      --enable-config=sandybridge on x86-64 Linux;
#   2. writes one build-local shadow of src/stra_nodes/stra_matrify.hpp in which
#      the three `stra_size(X)` template arguments (lines 145, 218, 294) are
#      replaced by a type trait, because GCC 13 rejects a call on a reference
#      parameter as a constant expression; no semantics change;
#   3. compiles the library sources listed in the reference Makefile.am, the
#      sandybridge AVX kernels and TCI, plus oracle/ref_harness.cxx, with g++/gcc
#      -O3 -mavx -fPIC into one shared object.
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]
#   (default: $TBLIS_STRA_REFERENCE_ROOT, else a directory named "reference"
#   beside this repository)
# Outputs go only to oracle/_ref/.
set -euo pipefail

HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${TBLIS_STRA_REFERENCE_ROOT:-$(cd "$HERE/../.." && pwd)/reference}}"
OUT="$HERE/_ref"
GEN="$OUT/gen"
SHADOW="$OUT/shadow"
OBJ="$OUT/obj"

if [ ! -f "$REF/src/stra_iface/3t/stra_mult.cxx" ]; then
    echo "build_ref.sh: reference sources not found under $REF" >&2
    exit 2
fi

mkdir -p "$GEN/configs" "$GEN/cfgdir" "$SHADOW/stra_nodes" "$OBJ"

# ---- 1. configure-time headers ------------------------------------------
# src/util/basic_types.h includes "../tblis_config.h"; the quoted include is
# resolved against each -I directory, so GEN/cfgdir/../tblis_config.h works.
cat > "$GEN/tblis_config.h" <<'EOF'
#ifndef _TBLIS_CONFIG_H_BUILD_LOCAL
#define _TBLIS_CONFIG_H_BUILD_LOCAL
#include <stddef.h>
#define TBLIS_LEN_TYPE ptrdiff_t
#define TBLIS_STRIDE_TYPE ptrdiff_t
#define TBLIS_LABEL_TYPE char
#define TBLIS_RESTRICT __restrict__
#define TBLIS_HAVE_CXX11 1
#define TBLIS_HAVE_SYSCONF 1
#define TBLIS_HAVE__SC_NPROCESSORS_ONLN 1
#define TBLIS_HAVE__SC_NPROCESSORS_CONF 1
#define TBLIS_HAVE_SYSCTL 0
#define TBLIS_HAVE_HWLOC_H 0
#define TBLIS_HAVE_LSCPU 0
#define TBLIS_HAVE_HBWMALLOC_H 0
#define TBLIS_HAVE_MEMKIND_H 0
#define TBLIS_HAVE_BLAS 0
#define TBLIS_TOPDIR "."
#endif
EOF

# tci_config.h: the template with its @...@ placeholders substituted, as
# TCI's configure does for pthreads threads + pthread spinlocks.
sed -e 's/@USE_ATOMIC_SPINLOCK@/0/' -e 's/@USE_OMP_LOCK@/0/' \
    -e 's/@USE_OPENMP_THREADS@/0/' -e 's/@USE_OSX_SPINLOCK@/0/' \
    -e 's/@USE_PTHREADS_THREADS@/1/' -e 's/@USE_PTHREAD_BARRIER@/0/' \
    -e 's/@USE_PTHREAD_MUTEX@/0/' -e 's/@USE_PTHREAD_SPINLOCK@/1/' \
    -e 's/@USE_SPIN_BARRIER@/1/' \
    "$REF/src/external/tci/tci/tci_config.h.in" > "$GEN/tci_config.h"
if grep -q '@[A-Z_]*@' "$GEN/tci_config.h"; then
    echo "build_ref.sh: unsubstituted placeholder in tci_config.h" >&2
    exit 3
fi

CONFIGS="sandybridge reference"
{
    for c in $CONFIGS; do echo "FOREACH_CONFIG(${c}_config)"; done
    echo; echo "#undef FOREACH_CONFIG"
} > "$GEN/configs/foreach_config.h"
{
    for t in float double scomplex dcomplex; do echo "FOREACH_TYPE($t)"; done
    echo; echo "#undef FOREACH_TYPE"
} > "$GEN/configs/foreach_type.h"
{
    for c in $CONFIGS; do
        echo "#define FOREACH_TYPE(type) \\"
        echo "FOREACH_CONFIG_AND_TYPE(type, ${c}_config)"
        echo "#include \"foreach_type.h\""
    done
    echo; echo "#undef FOREACH_CONFIG_AND_TYPE"
} > "$GEN/configs/foreach_config_and_type.h"
{
    for c in $CONFIGS; do echo "#include \"configs/$c/config.hpp\""; done
} > "$GEN/configs/include_configs.hpp"

# ---- 2. GCC 13 constant-expression shadow -------------------------------
sed -e 's/stra_block_scatter_matrix<T, stra_size(A) >/stra_block_scatter_matrix<T, oracle_stra_n<MatrixA>::value >/' \
    -e 's/stra_block_scatter_matrix<T, stra_size(B)>/stra_block_scatter_matrix<T, oracle_stra_n<MatrixB>::value>/' \
    -e 's/stra_block_scatter_matrix<T, stra_size(C)>/stra_block_scatter_matrix<T, oracle_stra_n<MatrixC>::value>/' \
    "$REF/src/stra_nodes/stra_matrify.hpp" > "$SHADOW/stra_nodes/stra_matrify.hpp.body"
{
    echo '#include "matrix/stra_tensor_view.hpp"'
    echo 'namespace tblis {'
    echo 'template <typename M> struct oracle_stra_n { static constexpr unsigned value = 1; };'
    echo 'template <typename T, unsigned N> struct oracle_stra_n<stra_tensor_view<T,N>> { static constexpr unsigned value = N; };'
    echo '}'
    cat "$SHADOW/stra_nodes/stra_matrify.hpp.body"
} > "$SHADOW/stra_nodes/stra_matrify.hpp"
n_fixed=$(grep -c 'oracle_stra_n<Matrix' "$SHADOW/stra_nodes/stra_matrify.hpp" || true)
if [ "$n_fixed" != "3" ]; then
    echo "build_ref.sh: expected 3 stra_size substitutions, got $n_fixed" >&2
    exit 3
fi

# ---- 3. compile ----------------------------------------------------------
INC="-I$SHADOW -I$GEN/cfgdir -I$GEN -I$GEN/configs -I$REF/src -I$REF -I$REF/src/external/tci -I$REF/src/external/tci/tci"
CXXFLAGS="-O3 -mavx -fPIC -std=c++11 -w -pthread -include limits -include $GEN/tci_config.h $INC"
CFLAGS="-O3 -mavx -fPIC -w -pthread -include $GEN/tci_config.h $INC"

LIB_SOURCES=$(awk '/^lib_libtblis_la_SOURCES/{f=1;next} f&&/^$/{f=0} f' "$REF/Makefile.am" \
              | tr -d '\\\t ' | grep '\.cxx$')
SB_SOURCES="src/configs/sandybridge/bli_gemm_asm_d8x4.c src/configs/sandybridge/bli_stra_asm_d8x4.c
src/configs/sandybridge/bli_stra_two_asm_d8x4.c src/configs/sandybridge/bli_stra_four_asm_d8x4.c
src/configs/sandybridge/config.cxx src/configs/reference/config.cxx"
TCI_SOURCES="src/external/tci/tci/barrier.c src/external/tci/tci/communicator.c src/external/tci/tci/context.c
src/external/tci/tci/mutex.c src/external/tci/tci/parallel.c src/external/tci/tci/work_item.c"

JOBS=$(nproc 2>/dev/null || echo 4)
objs=()
compile_one() {
    local src="$1" o="$2"
    case "$src" in
        *.c)   gcc $CFLAGS -c "$REF/$src" -o "$o" ;;
        *.cxx) g++ $CXXFLAGS -c "$REF/$src" -o "$o" ;;
    esac
}
export -f compile_one
export REF CFLAGS CXXFLAGS

list=()
for s in $LIB_SOURCES $SB_SOURCES $TCI_SOURCES; do
    o="$OBJ/$(echo "$s" | tr '/' '_').o"
    objs+=("$o")
    if [ ! -f "$o" ] || [ "$REF/$s" -nt "$o" ]; then
        list+=("$s $o")
    fi
done
if [ ${#list[@]} -gt 0 ]; then
    printf '%s\n' "${list[@]}" | xargs -P "$JOBS" -L 1 bash -c 'compile_one "$0" "$1"'
fi

g++ $CXXFLAGS -c "$HERE/ref_harness.cxx" -o "$OBJ/ref_harness.o"
g++ -shared -pthread -o "$OUT/libtblis_ref.so" "${objs[@]}" "$OBJ/ref_harness.o"
echo "build_ref.sh: built $OUT/libtblis_ref.so"
