// Staging helpers shared by the one-rank DArray mirror headers: host <-> device copies through the C ABI on the
// process-wide default context, with the reference's failure behaviour (message + exit, include/dkernel.cu:20-26).
#pragma once
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../darray_b200.h"

namespace darray_b200 {
namespace detail {

inline db200_context* ctx() {
  db200_context* c = db200_default_context();
  if (!c) {
    std::fprintf(stderr, "darray_b200: no usable sm_100 device\n");
    std::exit(EXIT_FAILURE);
  }
  return c;
}

inline void check(int st, const char* where) {
  if (st != DB200_OK) {
    std::fprintf(stderr, "darray_b200: %s failed: %s (status %d)\n", where, db200_last_error(ctx()), st);
    std::exit(st < 0 ? -st : st);
  }
}

// Device buffer of T elements.
template <class T>
struct Dev {
  T* p = nullptr;
  size_t count = 0;
  explicit Dev(size_t n) : count(n) {
    void* v = nullptr;
    check(db200_malloc(ctx(), sizeof(T) * (n ? n : 1), &v), "device allocation");
    p = static_cast<T*>(v);
  }
  Dev(const Dev&) = delete;
  Dev& operator=(const Dev&) = delete;
  ~Dev() { db200_free(ctx(), p); }
};

// Upload an m x n column-major host block (leading dimension ld, element type S) as packed FP64 or FP32 (T).
template <class T, class S>
inline void upload(Dev<T>& d, const S* src, int m, int n, int ld) {
  std::vector<T> h((size_t)m * n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) h[i + (size_t)j * m] = static_cast<T>(src[i + (size_t)j * ld]);
  check(db200_copy_to_device(ctx(), d.p, h.data(), sizeof(T) * h.size()), "copy to device");
}

// Download a packed m x n block into a host block with leading dimension ld; with upper_only only i <= j.
template <class T, class S>
inline void download(S* dst, int m, int n, int ld, const Dev<T>& d, bool upper_only = false) {
  std::vector<T> h((size_t)m * n);
  check(db200_copy_to_host(ctx(), h.data(), d.p, sizeof(T) * h.size()), "copy to host");
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i)
      if (!upper_only || i <= j) dst[i + (size_t)j * ld] = static_cast<S>(h[i + (size_t)j * m]);
}

}  // namespace detail
}  // namespace darray_b200
