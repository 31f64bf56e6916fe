#!/usr/bin/env bash
# Compile the reference's own C++ headers (read in place under the reference checkout) together with
# oracle/ref_driver.cpp and the single-rank MPI stub into oracle/_ref/libdarray_ref.so, linked against the
# OpenBLAS 0.3.15 that ships inside the image's opencv wheel (the reference needs Fortran BLAS/LAPACK symbols
# with 32-bit integers).  Outputs go to oracle/_ref/ only.  Test infrastructure: the product never links it.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${DARRAY_REFERENCE:-/root/reference}"
if [ ! -d "$REF/include" ]; then
  echo "reference sources not found at $REF; nothing to build" >&2
  exit 0
fi
BLAS_DIR="$(python -c 'import os, cv2; print(os.path.join(os.path.dirname(os.path.dirname(cv2.__file__)), "opencv_python_headless.libs"))' 2>/dev/null || true)"
if [ -z "$BLAS_DIR" ] || [ ! -d "$BLAS_DIR" ]; then
  BLAS_DIR="$(python -c 'import site; print(site.getsitepackages()[0])')/opencv_python_headless.libs"
fi
BLAS_LIB="$(ls "$BLAS_DIR"/libopenblasp-*.so 2>/dev/null | head -1)"
if [ -z "$BLAS_LIB" ]; then
  echo "no OpenBLAS with Fortran symbols found; reference build skipped" >&2
  exit 0
fi
mkdir -p "$HERE/_ref"
# -ftrivial-auto-var-init=zero: read_input_file passes an uninitialised `char* line` to getline
# (include/read_input.h:15-19), which glibc only accepts as NULL; zero-initialising locals gives it that.
g++ -O2 -std=c++17 -shared -fPIC -w -ftrivial-auto-var-init=zero \
    -I "$HERE/mpi_stub" -I "$REF/include" \
    "$HERE/ref_driver.cpp" -o "$HERE/_ref/libdarray_ref.so" \
    "$BLAS_LIB" -Wl,--disable-new-dtags -Wl,-rpath,"$BLAS_DIR"
echo "$HERE/_ref/libdarray_ref.so"

# The reference's GPU kernel-block code (include/dkernel.cu: rbf_kernel, tc_gemm) compiled unmodified for
# sm_100a, with the C wrappers of oracle/ref_gpu_shim.cpp, into oracle/_ref/libdkernel_ref.so.  Linked with
# -Bsymbolic: the product library exports drop-in C++ symbols of the same names (rbf_kernel, tc_gemm, cuda_init),
# and the wrappers must reach the reference's definitions even when both libraries sit in one process.
if command -v nvcc > /dev/null && [ -f "$REF/include/dkernel.cu" ]; then
  nvcc -O2 -std=c++17 -shared -Xcompiler -fPIC -w -gencode arch=compute_100a,code=sm_100a \
      "$REF/include/dkernel.cu" "$HERE/ref_gpu_shim.cpp" -o "$HERE/_ref/libdkernel_ref.so" \
      -Xlinker -Bsymbolic -lcublas -lcusolver
  echo "$HERE/_ref/libdkernel_ref.so"
fi

# The reference's own test programs tests/test3.cpp .. test7.cpp, unmodified, compiled against this build's
# one-rank mirror headers (include/darray_b200/) and linked with libdarray_b200.so: the drop-in proof that code
# written against DArray's headers builds and runs on the product without source changes.  Outputs to
# oracle/_ref/reftests/ (the binaries find the product library through a relative rpath).
ROOT="$(cd "$HERE/.." && pwd)"
if [ -f "$ROOT/darray_optimizer_b200/lib/libdarray_b200.so" ] && [ -f "$REF/tests/test3.cpp" ]; then
  mkdir -p "$HERE/_ref/reftests"
  for t in test3 test4 test5 test6 test7; do
    g++ -O2 -std=c++17 -w -I "$ROOT/include/darray_b200" -I "$ROOT/include" "$REF/tests/$t.cpp" \
        -o "$HERE/_ref/reftests/$t" -L "$ROOT/darray_optimizer_b200/lib" -ldarray_b200 \
        -Wl,-rpath,'$ORIGIN/../../../darray_optimizer_b200/lib'
    echo "$HERE/_ref/reftests/$t"
  done
fi
