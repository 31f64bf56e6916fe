// One-rank mirror of DArray's containers (include/darray.h of rushah05/DArray_Optimizer): Grid, LMatrix,
// DMatrix and DMatrixDescriptor with the same names, members and column-major storage, for a 1 x 1 process
// grid.  Code written against the reference's headers compiles against this one without MPI; at one rank every
// replicate_* / dereplicate_* is a local copy, which is exactly what the reference's MPI calls reduce to there.
//
// Only the single-rank semantics are provided: constructing a Grid with p * q != 1 aborts.
#pragma once

#include <array>
#include <cassert>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <iostream>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "mpi_one.h"
#include "fmt_lite.h"
#include "utils.h"

namespace DArray {

enum Layout { RowMajor, ColMajor };

// dest[i + j*lddest] = src[i + j*ldsrc] for an m x n block (include/darray.h:22-31).
template <typename T>
void copy_block(int m, int n, const T* src, int ldsrc, T* dest, int lddest) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) dest[i + (size_t)j * lddest] = src[i + (size_t)j * ldsrc];
}

// dest (n x m) = src (m x n) transposed (include/darray.h:36-44).
template <typename T>
void copy_transposed_block(int m, int n, const T* src, int ldsrc, T* dest, int lddest) {
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) dest[j + (size_t)i * lddest] = src[i + (size_t)j * ldsrc];
}

inline int size_of_local_part(int globalsize, int p, int np) { return (globalsize - p + np - 1) / np; }

class Grid {
 public:
  Grid() = default;
  Grid(MPI_Comm comm, int p, int q) : m_comm(comm), m_dims{p, q} {
    if (p * q != 1) {
      std::fprintf(stderr, "darray_b200: only the 1 x 1 grid (MPI world size 1) is provided, got %d x %d\n", p, q);
      std::abort();
    }
  }
  int rank() { return 0; }
  std::array<int, 2> ranks() { return {0, 0}; }
  int np() { return 1; }
  std::array<int, 2> dims() { return m_dims; }
  MPI_Comm comm() { return m_comm; }
  std::array<MPI_Comm, 2> comms() { return {m_comm, m_comm}; }
  Layout layout() { return ColMajor; }
  int convert_to_linear(int i, int j) { return i + j * m_dims[0]; }
  std::array<int, 2> convert_to_pq(int p) { return {p % m_dims[0], p / m_dims[0]}; }
  void barrier() {}
  void barrier_col() {}
  void barrier_row() {}
  // near-square p x q factorisation of np (include/darray.h:163-172)
  static void np_to_pq(int np, int& p, int& q) {
    for (int k = (int)std::lround(std::sqrt((double)np)); k > 0; --k) {
      if (np % k == 0) {
        p = k;
        q = np / k;
        return;
      }
    }
  }
  void for_each_process_in_column(std::function<void(void)> f) { f(); }
  void for_each_process_in_row(std::function<void(void)> f) { f(); }
  void for_each_process_in_grid(std::function<void(void)> f) { f(); }

 private:
  MPI_Comm m_comm = MPI_COMM_WORLD;
  std::array<int, 2> m_dims{1, 1};
};

template <typename T>
class LMatrix {
 public:
  LMatrix() : m_dims{0, 0}, m_ld(0), m_data(nullptr) {}
  LMatrix(int m, int n) : LMatrix(m, n, m) {}
  LMatrix(int m, int n, int ld) : m_dims{m, n}, m_ld(ld) {
    m_storage = std::shared_ptr<T[]>(new T[(size_t)std::max(ld, 1) * std::max(n, 1)]());
    m_data = m_storage.get();
  }
  // a view on caller-owned memory (no ownership)
  LMatrix(int m, int n, int ld, T* buffer) : m_dims{m, n}, m_ld(ld), m_data(buffer) {}

  T& operator[](int i) { return m_data[i]; }
  T operator[](int i) const { return m_data[i]; }
  T& operator()(int i, int j) { return m_data[i + (size_t)j * m_ld]; }
  T operator()(int i, int j) const { return m_data[i + (size_t)j * m_ld]; }
  int& ld() { return m_ld; }
  void set_ld(int ld) { m_ld = ld; }
  T* data() { return m_data; }
  std::array<int, 2> dims() { return m_dims; }

  void print(const std::string& title) {
    std::cout << title << std::endl;
    for (int i = 0; i < m_dims[0]; ++i) {
      for (int j = 0; j < m_dims[1]; ++j) std::printf("%8.3f ", (double)(*this)(i, j));
      std::printf("\n");
    }
  }
  void save_to_file(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "w");
    if (!f) return;
    for (int i = 0; i < m_dims[0]; ++i) {
      for (int j = 0; j < m_dims[1]; ++j) std::fprintf(f, "%.17g, ", (double)(*this)(i, j));
      std::fprintf(f, "\n");
    }
    std::fclose(f);
  }
  void set_constant(T a) {
    for (int j = 0; j < m_dims[1]; ++j)
      for (int i = 0; i < m_dims[0]; ++i) (*this)(i, j) = a;
  }
  void set_Identity() {
    for (int j = 0; j < m_dims[1]; ++j)
      for (int i = 0; i < m_dims[0]; ++i) (*this)(i, j) = (i == j) ? T(1) : T(0);
  }
  void set_normal(T mean, T stddev) {
    std::mt19937 gen((unsigned)std::chrono::system_clock::now().time_since_epoch().count());
    std::normal_distribution<T> dist(mean, stddev);
    for (int j = 0; j < m_dims[1]; ++j)
      for (int i = 0; i < m_dims[0]; ++i) (*this)(i, j) = dist(gen);
  }
  void add(LMatrix<T>& A) {
    for (int j = 0; j < m_dims[1]; ++j)
      for (int i = 0; i < m_dims[0]; ++i) (*this)(i, j) += A(i, j);
  }
  void diag(LMatrix<T> E) {
    for (int j = 0; j < m_dims[1]; ++j)
      for (int i = 0; i < m_dims[0]; ++i) (*this)(i, j) = (i == j) ? E.data()[i + (size_t)j * E.ld()] : T(0);
  }
  LMatrix<T> diag() {
    LMatrix<T> E(m_dims[0], 1);
    for (int i = 0; i < m_dims[0] && i < m_dims[1]; ++i) E.data()[i] = (*this)(i, i);
    return E;
  }
  void set_function(std::function<T(int, int)> func) {
    for (int i = 0; i < m_dims[0]; ++i)
      for (int j = 0; j < m_dims[1]; ++j) (*this)(i, j) = func(i, j);
  }
  LMatrix<T> transpose() {
    LMatrix<T> At(m_dims[1], m_dims[0]);
    copy_transposed_block(m_dims[0], m_dims[1], m_data, m_ld, At.data(), At.ld());
    return At;
  }
  void clear_upper() {
    for (int j = 0; j < m_dims[1]; ++j)
      for (int i = 0; i < j && i < m_dims[0]; ++i) (*this)(i, j) = 0;
  }
  void clear_lower() {
    for (int j = 0; j < m_dims[1]; ++j)
      for (int i = j + 1; i < m_dims[0]; ++i) (*this)(i, j) = 0;
  }
  void float_to_double(float* sA, int lda) {
    for (int j = 0; j < m_dims[1]; ++j)
      for (int i = 0; i < m_dims[0]; ++i) (*this)(i, j) = static_cast<T>(sA[i + (size_t)j * lda]);
  }

 private:
  std::shared_ptr<T[]> m_storage;
  std::array<int, 2> m_dims;
  int m_ld;
  T* m_data;
};

template <typename T>
class DMatrix {
 public:
  DMatrix(Grid& grid, int m, int n)
      : m_grid(grid), m_dims{m, n}, m_lld(std::max(m, 1)), m_ipiv(std::max(m, 0), -1) {
    m_storage = std::shared_ptr<T[]>(new T[(size_t)m_lld * std::max(n, 1)]());
    m_data = m_storage.get();
  }
  // attach to a caller buffer holding the global block starting at (i1, j1)
  DMatrix(Grid& grid, int m, int n, T* buf, int ld, int i1, int j1)
      : m_grid(grid), m_dims{m, n}, m_lld(ld), m_ipiv(std::max(m, 0), -1), m_data(buf - (i1 + (size_t)j1 * ld)) {}

  DMatrix<T> clone() {
    DMatrix<T> A(m_grid, m_dims[0], m_dims[1]);
    copy_block(m_dims[0], m_dims[1], m_data, m_lld, A.m_data, A.m_lld);
    return A;
  }
  std::array<int, 2> dims() { return m_dims; }
  std::array<int, 2> ldims() { return m_dims; }
  Grid& grid() { return m_grid; }
  T* data() { return m_data; }
  int lld() { return m_lld; }
  T& at(int i, int j) { return m_data[i + (size_t)j * m_lld]; }
  T operator()(int i, int j) { return m_data[i + (size_t)j * m_lld]; }

  void set_uniform(T a, T b) {
    std::mt19937 gen((unsigned)std::chrono::system_clock::now().time_since_epoch().count());
    std::uniform_real_distribution<T> dist(a, b);
    fill([&](int, int) { return dist(gen); });
  }
  void set_normal(T mean, T stddev) {
    std::mt19937 gen((unsigned)std::chrono::system_clock::now().time_since_epoch().count());
    std::normal_distribution<T> dist(mean, stddev);
    fill([&](int, int) { return dist(gen); });
  }
  void set_normal_seed(T mean, T stddev, int seed) {
    std::mt19937 gen(seed);
    std::normal_distribution<T> dist(mean, stddev);
    fill([&](int, int) { return dist(gen); });
  }
  void set_constant(T a) { fill([&](int, int) { return a; }); }
  void set_identity() { fill([](int i, int j) { return i == j ? T(1) : T(0); }); }
  void set_value_from_matrix(T* x, int ldx) { fill([&](int i, int j) { return x[i + (size_t)j * ldx]; }); }
  void set_function(std::function<T(int, int)> func) { fill(func); }

  double fnorm() {
    double s = 0;
    for (int j = 0; j < m_dims[1]; ++j)
      for (int i = 0; i < m_dims[0]; ++i) s += (double)at(i, j) * (double)at(i, j);
    return std::sqrt(s);
  }
  LMatrix<T> collect(int) { return replicate_in_all(0, 0, m_dims[0], m_dims[1]); }
  void collect_and_print(const std::string& title, int root = 0) { collect(root).print(title); }

  // local part of the global block A[i1:i2, j1:j2] (a view)
  LMatrix<T> local_view(int i1, int j1, int i2, int j2) {
    return LMatrix<T>(i2 - i1, j2 - j1, m_lld, m_data + i1 + (size_t)j1 * m_lld);
  }
  LMatrix<T> replicate_in_all(int i1, int j1, int i2, int j2) { return copy_out(i1, j1, i2, j2); }
  LMatrix<T> replicate_in_columns(int i1, int j1, int i2, int j2) { return copy_out(i1, j1, i2, j2); }
  LMatrix<T> replicate_in_rows(int i1, int j1, int i2, int j2) { return copy_out(i1, j1, i2, j2); }
  LMatrix<T> transpose_and_replicate_in_rows(int i1, int j1, int i2, int j2) {
    LMatrix<T> r(j2 - j1, i2 - i1);
    copy_transposed_block(i2 - i1, j2 - j1, m_data + i1 + (size_t)j1 * m_lld, m_lld, r.data(), r.ld());
    return r;
  }
  void dereplicate_in_all(LMatrix<T> A, int i1, int j1, int i2, int j2) { copy_in(A, i1, j1, i2, j2); }
  void dereplicate_in_columns(LMatrix<T> A, int i1, int j1, int i2, int j2) { copy_in(A, i1, j1, i2, j2); }
  void dereplicate_in_rows(LMatrix<T> A, int i1, int j1, int i2, int j2) { copy_in(A, i1, j1, i2, j2); }
  LMatrix<T> copy_upper_to_lower(LMatrix<T> A, int, int) { return A; }
  LMatrix<T> copy_lower_to_upper(LMatrix<T> A, int, int) { return A; }
  static std::array<int, 2> global_to_local_index(std::array<int, 2> ij, int, int, int) { return ij; }
  // pivot rows of the last LU factorisation, 1-based (include/darray.h:437-486)
  std::vector<int>& ipiv() { return m_ipiv; }
  // exchange rows i1 and i2 in columns [j1, j2)
  void swap_rows(int i1, int i2, int j1, int j2) {
    for (int j = j1; j < j2; ++j) std::swap(at(i1, j), at(i2, j));
  }
  // the row interchanges ipiv (1-based, relative to i1) applied in order to rows [i1, i2) of columns [j1, j2)
  // (include/darray.h:1202-1212)
  void permute_rows_ipiv(int i1, int j1, int i2, int j2, int* ipiv, int n_ipiv) {
    (void)i2;
    for (int k = 0; k < n_ipiv; ++k) {
      const int p = ipiv[k] - 1 + i1;
      if (p != i1 + k) swap_rows(i1 + k, p, j1, j2);
    }
  }
  // the inverse: the same interchanges in reverse order (include/darray.h:1181-1200)
  void permute_rows_inverse_ipiv(int i1, int j1, int i2, int j2, int* ipiv, int n_ipiv) {
    (void)i2;
    for (int k = n_ipiv - 1; k >= 0; --k) {
      const int p = ipiv[k] - 1 + i1;
      if (p != i1 + k) swap_rows(i1 + k, p, j1, j2);
    }
  }
  void substract(DMatrix<T>& A) {
    for (int j = 0; j < m_dims[1]; ++j)
      for (int i = 0; i < m_dims[0]; ++i) at(i, j) -= A.at(i, j);
  }

 private:
  template <class F>
  void fill(F f) {
    for (int i = 0; i < m_dims[0]; ++i)
      for (int j = 0; j < m_dims[1]; ++j) at(i, j) = f(i, j);
  }
  LMatrix<T> copy_out(int i1, int j1, int i2, int j2) {
    LMatrix<T> r(i2 - i1, j2 - j1);
    copy_block(i2 - i1, j2 - j1, m_data + i1 + (size_t)j1 * m_lld, m_lld, r.data(), r.ld());
    return r;
  }
  void copy_in(LMatrix<T>& A, int i1, int j1, int i2, int j2) {
    copy_block(i2 - i1, j2 - j1, A.data(), A.ld(), m_data + i1 + (size_t)j1 * m_lld, m_lld);
  }

  Grid m_grid;
  std::array<int, 2> m_dims;
  int m_lld;
  std::vector<int> m_ipiv;
  std::shared_ptr<T[]> m_storage;
  T* m_data = nullptr;
};

template <typename T>
struct DMatrixDescriptor {
  DMatrix<T> matrix;
  int i1, j1, i2, j2;
  int m() { return i2 - i1; }
  int n() { return j2 - j1; }
  LMatrix<T> replicate_in_rows() { return matrix.replicate_in_rows(i1, j1, i2, j2); }
  LMatrix<T> replicate_in_columns() { return matrix.replicate_in_columns(i1, j1, i2, j2); }
  LMatrix<T> replicate_in_all() { return matrix.replicate_in_all(i1, j1, i2, j2); }
  void print(const std::string& title) { replicate_in_all().print(title); }
};

}  // namespace DArray
