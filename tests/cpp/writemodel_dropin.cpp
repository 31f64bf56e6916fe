// The drop-in writemodel (include/darray_b200/dbarrier.h) run on inputs read from a binary file: the model text
// the reference's tests/testsvm.cpp:324 call would write, and the same with a solved bias.  Host code only.
//   writemodel_dropin <input.bin> <model.txt> <use_bias 0|1>
// input.bin: int32 n, d, k, minus, plus; float64 C, gamma, bias; float64 a[n], Z[n*k] (column major), y[n],
// X[d*n] (point-major: feature kk of point j at j*d + kk).
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "darray_b200/darray.h"
#include "darray_b200/dbarrier.h"

int main(int argc, char** argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: %s input.bin model.txt use_bias\n", argv[0]);
    return 2;
  }
  FILE* f = std::fopen(argv[1], "rb");
  if (!f) return 3;
  int hdr[5];
  double par[3];
  if (std::fread(hdr, sizeof(int), 5, f) != 5 || std::fread(par, sizeof(double), 3, f) != 3) return 4;
  const int n = hdr[0], d = hdr[1], k = hdr[2], minus = hdr[3], plus = hdr[4];
  std::vector<double> a(n), Z((size_t)n * k), y(n), X((size_t)d * n);
  if (std::fread(a.data(), 8, a.size(), f) != a.size() || std::fread(Z.data(), 8, Z.size(), f) != Z.size() ||
      std::fread(y.data(), 8, y.size(), f) != y.size() || std::fread(X.data(), 8, X.size(), f) != X.size())
    return 5;
  std::fclose(f);
  DArray::LMatrix<double> A(n, 1, n, a.data()), Zm(n, k, n, Z.data()), Ym(n, 1, n, y.data()), Xm(d, n, d, X.data());
  const double bias = par[2];
  DArray::writemodel<double>(std::string(argv[2]), n, d, k, A, par[0], Zm, Ym, Xm, par[1], minus, plus,
                             std::atoi(argv[3]) ? &bias : nullptr);
  return 0;
}
