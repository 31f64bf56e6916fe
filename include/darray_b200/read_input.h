// One-rank mirror of include/read_input.h: read_input_file<T> reads the first n lines of a LIBSVM file into X
// (point i's feature k at X[k + i*d]) and Y (+1 for a label equal to 1, else -1) through the GPU reader
// (db200_read_libsvm).  Results are bit-identical to the reference's for every file it reads with defined
// behaviour.  Like the reference, rows are indexed with stride d (ldx is not used: the reference ignores it too)
// and a file that cannot be opened ends the process with EXIT_FAILURE; text the reference cannot read safely
// (a feature index above d, a last line of blanks) ends it with a message instead of writing out of bounds.
#pragma once
#include <cstdio>
#include <cstdlib>
#include <type_traits>

#include "detail.h"

template <typename T>
void read_input_file(char* filename, int n, int d, T* X, int ldx, T* Y) {
  static_assert(std::is_same<T, float>::value || std::is_same<T, double>::value, "float or double");
  (void)ldx;
  std::FILE* f = std::fopen(filename, "r");
  if (!f) std::exit(EXIT_FAILURE);
  std::fclose(f);
  const int dtype = std::is_same<T, float>::value ? DB200_F32 : DB200_F64;
  darray_b200::detail::check(
      db200_read_libsvm(darray_b200::detail::ctx(), filename, n, d, dtype, X, (long long)d, Y, nullptr),
      "read_input_file");
}
