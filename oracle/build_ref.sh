#!/usr/bin/env bash
# Builds the CPU oracle's two shared libraries (test infrastructure only):
#   oracle/_ref/libvbcsr_ref.so     the REFERENCE VBCSR C++ core (header-only,
#                                   read from $VBCSR_REFERENCE, default
#                                   /root/reference) behind oracle/ref_harness.cpp
#   oracle/_ref/libvbcsr_oracle.so  this repo's plain-C restatement
#                                   (oracle/vbcsr_oracle.c)
# The reference build needs no MPI (oracle/mpi_stub/mpi.h is a serial
# stand-in) and takes BLAS/LAPACK from scipy's bundled OpenBLAS, whose symbols
# carry a "scipy_" prefix.  None of the BLAS routines is reached at the block
# sizes the tests use (products of blocks <= 20 run the reference's own AVX2
# kernels).  Flags follow the reference's CMake Release build with its
# portable AVX2 arch option, so the library runs on any x86-64-v3 host.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
mkdir -p "$OUT"
CC=${VBCSR_ORACLE_CC:-gcc}
CXX=${VBCSR_ORACLE_CXX:-g++}

# 1. The C restatement (always buildable).
$CC -std=gnu11 -O2 -mavx2 -mfma -ffp-contract=off -fPIC -shared "$HERE/vbcsr_oracle.c" -o "$OUT/libvbcsr_oracle.so" -lm

# 2. The reference core, when its sources are present.
REF="${VBCSR_REFERENCE:-/root/reference}"
if [ ! -f "$REF/vbcsr/core/block_csr.hpp" ]; then
  echo "build_ref: reference sources not found at $REF; skipping libvbcsr_ref.so" >&2
  exit 0
fi
# where the reference checkout is, for the tests that import its Python
# package on top of this repository's host core (they skip without it)
(cd "$REF" && pwd) > "$OUT/reference_root"
PY=${PYTHON:-python}
SCIPY_LIBS="$($PY -c 'import scipy, os; print(os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs"))')"
OPENBLAS="$(ls "$SCIPY_LIBS"/libscipy_openblas-*.so | head -1)"
RENAMES=()
for s in cblas_dgemm cblas_dgemv cblas_zgemm cblas_zgemv cblas_dgemm_batch cblas_zgemm_batch \
         openblas_set_num_threads openblas_get_num_threads \
         dgemm_ dgesvd_ dgetrf_ dgetri_ dsyev_ dsyevd_ dtrsm_ \
         zgemm_ zgesvd_ zgetrf_ zgetri_ zheev_ zheevd_ ztrsm_; do
  RENAMES+=("-D$s=scipy_$s")
done
$CXX -std=gnu++17 -O3 -mavx2 -mfma -fopenmp -fPIC -shared -w \
  -I"$HERE/mpi_stub" -I"$REF/vbcsr/core" -DVBCSR_USE_OPENBLAS "${RENAMES[@]}" \
  "$HERE/ref_harness.cpp" -o "$OUT/libvbcsr_ref.so" \
  "$OPENBLAS" -Wl,-rpath,"$SCIPY_LIBS"
echo "build_ref: built $OUT/libvbcsr_ref.so"
