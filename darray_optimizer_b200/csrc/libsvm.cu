// LIBSVM text input on the GPU: read_input_file<T> (include/read_input.h:8-36) for text held in device memory.
//
// The reference reads n lines with getline, splits each line on ' ' with strtok, takes the first token's atof as
// the label (y = +1 when it equals 1 after conversion to T, else -1) and, for every further token, atoi of the
// part before the first ':' as a 1-based feature index and atof of the part after it as the value
// (X[(index - 1) + i*d] = value when index >= 1).  This file does the same in four passes:
//
//   nl_count_kernel    newlines per 16 KB chunk                       (one block per chunk, 16-byte loads)
//   nl_scan_kernel     exclusive prefix of the chunk counts, the line count
//   nl_starts_kernel   byte offset of the start of every line < n     (block-wide ranks of the newlines)
//   parse_kernel       one warp per line: a 512-byte window staged in shared memory (the next one already in
//                      flight), token starts by ballot, one token per lane parsed in one pass
//
// Values are converted exactly as glibc's strtod does (correctly rounded to double; for float output the double
// is then rounded to float, as the reference's `T value = atof(...)`).  Short decimals take Clinger's fast path
// (an integer mantissa <= 2^53 times or divided by an exact power of ten <= 1e22: one correctly rounded IEEE
// operation); everything else goes through an exact big-integer quotient with round-half-even.
//
// Where the reference has undefined behaviour the parser reports an error instead: a feature index above d (the
// reference writes past the row), a line of blanks at the end of the text (strtok returns NULL and atof
// dereferences it).  Hexadecimal values, NaN payloads "nan(...)", values with more than 38 significant digits
// and NUL bytes inside a line (the reference's C strings would end there) are rejected as unsupported rather
// than read differently.
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace db200 {

namespace {

constexpr int CHUNK = 16384;            // bytes per block of the newline passes
constexpr int NL_THREADS = 256;         // x 16 bytes = 4096 bytes per step
constexpr int NL_STEPS = CHUNK / (NL_THREADS * 16);
constexpr int PARSE_THREADS = 256;      // 8 warps, one line each at a time
constexpr int WIN = 512;                // bytes of a line one warp scans per step (32 lanes x 16)
constexpr int MAX_SIG = 38;             // significant digits a value may carry (two 19-digit words)
constexpr int LIMBS = 44;               // 32-bit limbs of the exact path: 10^361 * 2^57 < 2^1408

enum : unsigned { E_NONE = 0, E_INDEX = 1, E_HEX = 2, E_DIGITS = 3, E_NOLABEL = 4, E_NANPAYLOAD = 5, E_NUL = 6 };

// ------------------------------------------------------------------ newline passes
template <bool AL>
__device__ __forceinline__ uint4 load_seg(const unsigned char* text, long long bytes, long long off) {
  if (AL && off + 16 <= bytes) return __ldg(reinterpret_cast<const uint4*>(text + off));
  uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (int k = 0; k < 16; ++k)
    if (off + k < bytes) w[k >> 2] |= (uint32_t)__ldg(text + off + k) << (8 * (k & 3));
  return make_uint4(w[0], w[1], w[2], w[3]);
}

// bit k set when byte k of the 16-byte segment is '\n'
__device__ __forceinline__ uint32_t nl_mask(uint4 v) {
  const uint32_t w[4] = {v.x, v.y, v.z, v.w};
  uint32_t m = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t r = __vcmpeq4(w[i], 0x0a0a0a0au);
#pragma unroll
    for (int j = 0; j < 4; ++j) m |= ((r >> (8 * j + 7)) & 1u) << (4 * i + j);
  }
  return m;
}

__device__ __forceinline__ int block_sum(int v, int* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (lane == 0) red[w] = v;
  __syncthreads();
  int t = 0;
  if (threadIdx.x < 32) {
    t = lane < (int)(blockDim.x / 32) ? red[lane] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  return t;  // valid in thread 0
}

template <bool AL>
__global__ void __launch_bounds__(NL_THREADS) nl_count_kernel(const unsigned char* text, long long bytes,
                                                              int* counts) {
  __shared__ int red[NL_THREADS / 32];
  const long long base = (long long)blockIdx.x * CHUNK;
  int c = 0;
#pragma unroll
  for (int s = 0; s < NL_STEPS; ++s) {
    const long long off = base + (long long)s * NL_THREADS * 16 + threadIdx.x * 16;
    if (off < bytes) c += __popc(nl_mask(load_seg<AL>(text, bytes, off)));
  }
  const int t = block_sum(c, red);
  if (threadIdx.x == 0) counts[blockIdx.x] = t;
}

// One block: prefix[c] = newlines before chunk c; meta[0] = newlines in the text, meta[1] = lines to parse
// (min(n, newlines + 1 if the text does not end with '\n')).  meta[2] (lines that do not name all d features)
// is counted by the parse kernel.
__global__ void __launch_bounds__(1024) nl_scan_kernel(const int* counts, int nchunks, long long* prefix,
                                                       const unsigned char* text, long long bytes, int n,
                                                       long long* meta) {
  __shared__ long long wsum[32];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x % 32, w = threadIdx.x / 32;
  for (int base = 0; base < nchunks; base += 1024) {
    const int c = base + (int)threadIdx.x;
    const long long v = c < nchunks ? counts[c] : 0;
    long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
      long long s = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const long long y = __shfl_up_sync(0xffffffffu, s, o);
        if (lane >= o) s += y;
      }
      wsum[lane] = s;  // inclusive over warps
    }
    __syncthreads();
    const long long excl = carry + (w > 0 ? wsum[w - 1] : 0) + x - v;
    if (c < nchunks) prefix[c] = excl;
    __syncthreads();
    if (threadIdx.x == 0) carry += wsum[31];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const long long nl = carry;
    const long long lines = nl + ((bytes > 0 && text[bytes - 1] != '\n') ? 1 : 0);
    meta[0] = nl;
    meta[1] = lines < (long long)n ? lines : (long long)n;
  }
}

// starts[L] = offset of the first byte of line L, for 1 <= L <= min(n, newlines); starts[0] = 0.
template <bool AL>
__global__ void __launch_bounds__(NL_THREADS) nl_starts_kernel(const unsigned char* text, long long bytes,
                                                               const long long* prefix, int n,
                                                               long long* starts) {
  __shared__ int wtot[NL_THREADS / 32];
  const int lane = threadIdx.x % 32, w = threadIdx.x / 32;
  const long long base = (long long)blockIdx.x * CHUNK;
  long long run = prefix[blockIdx.x];
  if (blockIdx.x == 0 && threadIdx.x == 0) starts[0] = 0;
  for (int s = 0; s < NL_STEPS; ++s) {
    if (run >= n) break;  // block-uniform: every later newline starts a line >= n + 1
    const long long off = base + (long long)s * NL_THREADS * 16 + threadIdx.x * 16;
    const uint32_t m = off < bytes ? nl_mask(load_seg<AL>(text, bytes, off)) : 0u;
    const int c = __popc(m);
    int x = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wtot[w] = x;
    __syncthreads();
    int before = 0, total = 0;
#pragma unroll
    for (int k = 0; k < NL_THREADS / 32; ++k) {
      before += k < w ? wtot[k] : 0;
      total += wtot[k];
    }
    long long rank = run + before + x - c;  // newlines before this thread's first one
    uint32_t mm = m;
    while (mm) {
      const int k = __ffs(mm) - 1;
      mm &= mm - 1;
      const long long line = rank + 1;  // the line that starts after this newline
      if (line <= n) starts[line] = off + k + 1;
      ++rank;
    }
    run += total;
    __syncthreads();
  }
}

// ------------------------------------------------------------------ number conversion
__device__ __forceinline__ bool c_digit(unsigned c) { return c - '0' < 10u; }
__device__ __forceinline__ bool c_hex(unsigned c) { return c_digit(c) || ((c | 0x20u) - 'a' < 6u); }
// C whitespace other than the blank, which ends a token
__device__ __forceinline__ bool c_ctl_space(unsigned c) { return c >= 9u && c <= 13u; }

// The bytes of one line as the token parser reads them, by offset q from a window start w0: the warp's staged
// window in shared memory for 0 <= q < lim, global memory up to the line end beyond it, a blank past the line
// end.  A token ends at its first blank.
struct LineBytes {
  const unsigned char* sm;
  unsigned lim;           // WIN when the window is staged, 0 to read global memory only
  long long w0;
  const unsigned char* text;
  long long e;            // line end
  __device__ __forceinline__ unsigned at(int q) const {
    if ((unsigned)q < lim) return sm[q];
    const long long pos = w0 + q;
    return (q >= 0 && pos < e) ? (unsigned)__ldg(text + pos) : (unsigned)' ';
  }
};
__device__ __forceinline__ bool c_end(unsigned c) { return c == ' ' || c == 0u; }

// Little-endian 32-bit limb arithmetic for the exact path (lengths in limbs, no leading zero limbs).
__device__ int bn_mul_add(uint32_t* a, int n, uint32_t mul, uint32_t add) {
  uint64_t carry = add;
  for (int i = 0; i < n; ++i) {
    const uint64_t t = (uint64_t)a[i] * mul + carry;
    a[i] = (uint32_t)t;
    carry = t >> 32;
  }
  if (carry) a[n++] = (uint32_t)carry;
  return n;
}

__device__ int bn_pow10_mul(uint32_t* a, int n, int k) {
  while (k >= 9) {
    n = bn_mul_add(a, n, 1000000000u, 0u);
    k -= 9;
  }
  const uint32_t p[9] = {1u, 10u, 100u, 1000u, 10000u, 100000u, 1000000u, 10000000u, 100000000u};
  if (k > 0) n = bn_mul_add(a, n, p[k], 0u);
  return n;
}

__device__ int bn_bitlen(const uint32_t* a, int n) { return n ? 32 * (n - 1) + (32 - __clz(a[n - 1])) : 0; }

__device__ int bn_shl(uint32_t* a, int n, int s) {
  if (n == 0 || s == 0) return n;
  const int ws = s / 32, bs = s % 32;
  int m = n + ws + 1;
  for (int i = m - 1; i >= 0; --i) {
    const int src = i - ws;
    uint32_t hi = (src >= 0 && src < n) ? a[src] : 0u;
    uint32_t lo = (src - 1 >= 0 && src - 1 < n) ? a[src - 1] : 0u;
    a[i] = bs ? (hi << bs) | (lo >> (32 - bs)) : hi;
  }
  while (m > 0 && a[m - 1] == 0) --m;
  return m;
}

__device__ bool bn_bit(const uint32_t* a, int n, int b) {
  const int w = b / 32;
  return w < n && ((a[w] >> (b % 32)) & 1u);
}

__device__ bool bn_any_below(const uint32_t* a, int n, int b) {  // any bit at position < b
  for (int w = 0; w < n && 32 * w < b; ++w) {
    const int hi = b - 32 * w;
    const uint32_t mask = hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u);
    if (a[w] & mask) return true;
  }
  return false;
}

// Round the integer a (n limbs, a > 0) to the nearest double, ties to even.
__device__ double bn_to_double(const uint32_t* a, int n) {
  int tb = bn_bitlen(a, n) - 1;
  if (tb > 1023 + 1) return INFINITY;
  uint64_t m = 0;
  for (int b = tb; b >= tb - 52; --b) m = (m << 1) | (b >= 0 && bn_bit(a, n, b) ? 1ull : 0ull);
  const int hb = tb - 53;
  const bool half = hb >= 0 && bn_bit(a, n, hb);
  const bool sticky = hb > 0 && bn_any_below(a, n, hb);
  if (half && (sticky || (m & 1ull))) {
    if (++m == (1ull << 53)) {
      m >>= 1;
      ++tb;
    }
  }
  if (tb > 1023) return INFINITY;
  return ldexp((double)m, tb - 52);
}

// W * 10^e10 (W > 0 given as w_hi * 10^n_lo + w_lo), correctly rounded to double.  Magnitude cut-offs are
// applied by the caller.
__device__ __noinline__ double slow_convert(uint64_t w_hi, uint64_t w_lo, int n_lo, int e10) {
  uint32_t N[LIMBS], D[LIMBS];
  int nn;
  N[0] = (uint32_t)w_hi;
  N[1] = (uint32_t)(w_hi >> 32);
  nn = N[1] ? 2 : (N[0] ? 1 : 0);
  if (n_lo > 0) {
    nn = bn_pow10_mul(N, nn, n_lo);
    uint64_t carry = w_lo;  // + w_lo
    for (int i = 0; carry; ++i) {
      if (i == nn) N[nn++] = 0u;
      const uint64_t t = (uint64_t)N[i] + (carry & 0xffffffffull);
      N[i] = (uint32_t)t;
      carry = (carry >> 32) + (t >> 32);
    }
  }
  if (e10 >= 0) {
    nn = bn_pow10_mul(N, nn, e10);
    return bn_to_double(N, nn);
  }
  // value = N / 10^k: quotient of 56..57 bits, then round with the remainder as sticky
  D[0] = 1u;
  int dn = bn_pow10_mul(D, 1, -e10);
  const int bw = bn_bitlen(N, nn), bd = bn_bitlen(D, dn);
  int sh = bd - bw + 56;  // N * 2^sh / D lies in [2^55, 2^57)
  if (sh >= 0) nn = bn_shl(N, nn, sh);
  else dn = bn_shl(D, dn, -sh);
  // long division for 57 quotient bits: S = D << 56, shifted right one bit per step
  dn = bn_shl(D, dn, 56);
  uint64_t q = 0;
  for (int b = 56; b >= 0; --b) {
    // compare N >= D
    int cmp = 0;
    if (nn != dn) cmp = nn > dn ? 1 : -1;
    else
      for (int i = nn - 1; i >= 0; --i)
        if (N[i] != D[i]) {
          cmp = N[i] > D[i] ? 1 : -1;
          break;
        }
    if (cmp >= 0) {
      uint64_t borrow = 0;
      for (int i = 0; i < nn; ++i) {
        const uint64_t t = (uint64_t)N[i] - (i < dn ? D[i] : 0u) - borrow;
        N[i] = (uint32_t)t;
        borrow = (t >> 63) & 1ull;
      }
      while (nn > 0 && N[nn - 1] == 0) --nn;
      q |= 1ull << b;
    }
    // D >>= 1
    for (int i = 0; i < dn; ++i) D[i] = (D[i] >> 1) | (i + 1 < dn ? (D[i + 1] << 31) : 0u);
    while (dn > 0 && D[dn - 1] == 0) --dn;
  }
  bool sticky = nn > 0;
  if (q >= (1ull << 56)) {
    sticky |= (q & 1ull) != 0;
    q >>= 1;
    --sh;
  }
  // value = q * 2^-sh (+ sticky), q in [2^55, 2^56): leading bit at 2^(55 - sh)
  const int e2 = 55 - sh;
  if (e2 >= -1022) {
    uint64_t m = q >> 3;
    const uint32_t g = (uint32_t)(q & 7ull);
    if (g > 4u || (g == 4u && (sticky || (m & 1ull)))) ++m;
    int ee = e2;
    if (m == (1ull << 53)) {
      m >>= 1;
      ++ee;
    }
    return ldexp((double)m, ee - 52);
  }
  const int shift = sh - 1074;  // bits of q below the subnormal unit 2^-1074 (> 3 here)
  if (shift > 57) return 0.0;   // below half of the smallest subnormal
  uint64_t m = q >> shift;
  const uint64_t rem = q & ((1ull << shift) - 1ull);
  const uint64_t halfv = 1ull << (shift - 1);
  if (rem > halfv || (rem == halfv && (sticky || (m & 1ull)))) ++m;
  return ldexp((double)m, -1074);
}

__device__ const double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                                      1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

// strtod of the token text from offset q (the token ends at its first blank): returns E_NONE and the value, or
// an unsupported-form code.
__device__ __forceinline__ unsigned parse_value(const LineBytes L, int q, double* out) {
  *out = 0.0;
  unsigned c = L.at(q);
  while (c_ctl_space(c)) c = L.at(++q);
  bool neg = false;
  if (c == '+' || c == '-') {
    neg = (c == '-');
    c = L.at(++q);
  }
  if ((c | 0x20u) == 'i' || (c | 0x20u) == 'n') {
    const unsigned c1 = L.at(q + 1) | 0x20u, c2 = L.at(q + 2) | 0x20u;
    if ((c | 0x20u) == 'i' && c1 == 'n' && c2 == 'f') {
      *out = neg ? -INFINITY : INFINITY;
    } else if ((c | 0x20u) == 'n' && c1 == 'a' && c2 == 'n') {
      if (L.at(q + 3) == '(') return E_NANPAYLOAD;
      *out = __longlong_as_double(neg ? (long long)0xfff8000000000000ull : 0x7ff8000000000000ll);
    }
    return E_NONE;  // otherwise no conversion: 0
  }
  if (c == '0' && (L.at(q + 1) | 0x20u) == 'x') {
    const unsigned c2 = L.at(q + 2);
    if (c_hex(c2) || (c2 == '.' && c_hex(L.at(q + 3)))) return E_HEX;
  }
  uint64_t w_hi = 0, w_lo = 0;
  int nsig = 0, e10 = 0;
  bool any = false, dropped = false;
  while (c_digit(c)) {
    const unsigned dg = c - '0';
    any = true;
    if (nsig == 0 && dg == 0) {
    } else if (nsig < MAX_SIG) {
      if (nsig < 19) w_hi = w_hi * 10 + dg;
      else w_lo = w_lo * 10 + dg;
      ++nsig;
    } else {
      dropped |= dg != 0;
      ++e10;
    }
    c = L.at(++q);
  }
  if (c == '.') {
    c = L.at(++q);
    while (c_digit(c)) {
      const unsigned dg = c - '0';
      any = true;
      if (nsig == 0 && dg == 0) {
        --e10;
      } else if (nsig < MAX_SIG) {
        if (nsig < 19) w_hi = w_hi * 10 + dg;
        else w_lo = w_lo * 10 + dg;
        ++nsig;
        --e10;
      } else {
        dropped |= dg != 0;
      }
      c = L.at(++q);
    }
  }
  if (!any) return E_NONE;  // no conversion
  if ((c | 0x20u) == 'e') {
    int r = q + 1;
    unsigned cr = L.at(r);
    bool eneg = false;
    if (cr == '+' || cr == '-') {
      eneg = (cr == '-');
      cr = L.at(++r);
    }
    if (c_digit(cr)) {
      int ev = 0;
      while (c_digit(cr)) {
        if (ev < 1000000) ev = ev * 10 + (int)(cr - '0');
        cr = L.at(++r);
      }
      e10 += eneg ? -ev : ev;
    }
  }
  if (dropped) return E_DIGITS;
  double v;
  if (nsig == 0) {
    v = 0.0;
  } else if (nsig + e10 > 310) {
    v = INFINITY;
  } else if (nsig + e10 < -323) {
    v = 0.0;
  } else if (nsig <= 19 && w_hi <= (1ull << 53) && e10 >= -22 && e10 <= 22) {
    const double x = (double)w_hi;  // exact
    v = e10 >= 0 ? __dmul_rn(x, __ldg(&kPow10[e10])) : __ddiv_rn(x, __ldg(&kPow10[-e10]));
  } else {
    v = nsig > 19 ? slow_convert(w_hi, w_lo, nsig - 19, e10) : slow_convert(w_hi, 0ull, 0, e10);
  }
  *out = neg ? -v : v;
  return E_NONE;
}

template <typename T>
__device__ __forceinline__ T to_t(double v);
// A NaN becomes the quiet NaN of its sign, as a host double-to-float conversion gives for strtod's NaNs.
template <>
__device__ __forceinline__ float to_t<float>(double v) {
  if (isnan(v)) return __int_as_float(signbit(v) ? (int)0xffc00000u : 0x7fc00000);
  return __double2float_rn(v);
}
template <>
__device__ __forceinline__ double to_t<double>(double v) { return v; }

__device__ __forceinline__ void report(unsigned long long* err, long long line, unsigned code) {
  atomicMin(err, ((unsigned long long)line << 8) | code);
}

// Parse one "index:value" token of line i starting at `pos`, in one pass over its bytes; returns the index
// written (0 when none).
template <typename T>
__device__ __forceinline__ long long feature_token(const LineBytes L, int q, long long i, int d, T* X, long long ldx,
                                                   unsigned long long* err) {
  const int start = q;
  unsigned c = L.at(q);
  while (c_ctl_space(c)) c = L.at(++q);  // atoi: leading whitespace, sign, digits
  bool neg = false;
  if (c == '+' || c == '-') {
    neg = (c == '-');
    c = L.at(++q);
  }
  long long idx = 0;
  while (c_digit(c)) {
    if (idx < (1ll << 40)) idx = idx * 10 + (c - '0');
    c = L.at(++q);
  }
  if (neg) idx = -idx;
  while (!c_end(c) && c != ':') c = L.at(++q);  // the first ':' (atoi stopped at or before it)
  if (idx < 1) return 0;                        // the reference's `index - 1 > -1` test
  if (idx > d) {
    report(err, i, E_INDEX);
    return 0;
  }
  double v;
  const unsigned code = parse_value(L, c == ':' ? q + 1 : start, &v);
  if (code != E_NONE) {
    report(err, i, code);
    return 0;
  }
  X[i * ldx + (idx - 1)] = to_t<T>(v);
  return idx;
}

// 16 bytes of the text at offset o (aligned to 16 when AL), blanks outside the line [s, e).
template <bool AL>
__device__ __forceinline__ uint4 line_seg(const unsigned char* text, long long bytes, long long o, long long s,
                                          long long e) {
  uint4 v = load_seg<AL>(text, bytes, o);
  const long long lo = s - o, hi = e - o;
  if (lo > 0 || hi < 16) {
    uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int k = 0; k < 16; ++k)
      if (k < lo || k >= hi) w[k >> 2] = (w[k >> 2] & ~(0xffu << (8 * (k & 3)))) | (0x20u << (8 * (k & 3)));
    v = make_uint4(w[0], w[1], w[2], w[3]);
  }
  return v;
}

template <typename T, bool AL>
__global__ void __launch_bounds__(PARSE_THREADS) parse_kernel(const unsigned char* text, long long bytes,
                                                              const long long* starts, long long* meta,
                                                              int d, T* X, long long ldx, T* y,
                                                              unsigned long long* err) {
  __shared__ __align__(16) unsigned char stage_all[PARSE_THREADS / 32][WIN];
  __shared__ uint16_t tstart[PARSE_THREADS / 32][WIN / 2 + 2];
  const int lane = threadIdx.x % 32, wib = threadIdx.x / 32;
  uint16_t* sh = tstart[wib];
  unsigned char* stage = stage_all[wib];
  const long long nl = meta[0], nlines = meta[1];
  const long long warps = (long long)gridDim.x * (PARSE_THREADS / 32);
  for (long long i = (long long)blockIdx.x * (PARSE_THREADS / 32) + wib; i < nlines; i += warps) {
    const long long s = starts[i];
    const long long e = (i + 1 <= nl) ? starts[i + 1] : bytes;
    bool prev_space = true;  // the line start acts as a delimiter
    long long tok = 0;       // tokens of this line seen so far
    long long maxidx = 0;    // largest feature index written so far
    bool simple = true;      // indices strictly increasing: no two tokens write one element
    long long named = 0;     // feature tokens written (distinct while `simple`)
    // Windows of 512 bytes on 16-byte boundaries of the text, bytes outside [s, e) read as blanks.  The next
    // window's segment is loaded into registers before the current window is parsed, so its memory latency hides
    // behind the token work; tokens that cross a window's end read the rest through L1.
    uint4 vn = line_seg<AL>(text, bytes, (s & ~15ll) + 16 * lane, s, e);
    for (long long w0 = s & ~15ll; w0 < e; w0 += WIN) {
      const uint4 v = vn;
      reinterpret_cast<uint4*>(stage)[lane] = v;
      if (w0 + WIN < e) vn = line_seg<AL>(text, bytes, w0 + WIN + 16 * lane, s, e);
      const uint32_t wv[4] = {v.x, v.y, v.z, v.w};
      // The reference sees a line as a C string that a NUL byte would end: reject such text.
      bool has_nul = false;
#pragma unroll
      for (int k = 0; k < 16; ++k) has_nul |= ((wv[k >> 2] >> (8 * (k & 3))) & 0xffu) == 0u;
      if (__any_sync(0xffffffffu, has_nul) && lane == 0) report(err, i, E_NUL);
      const unsigned last = (wv[3] >> 24) & 0xffu;
      const unsigned prev_last = (unsigned)__shfl_up_sync(0xffffffffu, (int)last, 1);
      bool pb = lane == 0 ? prev_space : (prev_last == ' ');
      uint32_t m = 0;
#pragma unroll
      for (int k = 0; k < 16; ++k) {
        const bool sp = ((wv[k >> 2] >> (8 * (k & 3))) & 0xffu) == ' ';
        if (!sp && pb) m |= 1u << k;
        pb = sp;
      }
      const int c = __popc(m);
      int x = c;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        const int yv = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += yv;
      }
      const int total = __shfl_sync(0xffffffffu, x, 31);
      int r = x - c;
      uint32_t mm = m;
      while (mm) {
        const int k = __ffs(mm) - 1;
        mm &= mm - 1;
        sh[r++] = (uint16_t)(16 * lane + k);
      }
      __syncwarp();
      const LineBytes L{stage, (unsigned)WIN, w0, text, e};
      for (int t0 = 0; t0 < total; t0 += 32) {
        const int t = t0 + lane;
        long long widx = 0;
        if (t < total) {
          const int q = sh[t];
          if (tok + t == 0) {
            double lv64;
            const unsigned code = parse_value(L, q, &lv64);
            if (code != E_NONE) report(err, i, code);
            const T lv = to_t<T>(lv64);
            y[i] = (lv == (T)1) ? (T)1 : (T)-1;
          } else {
            widx = feature_token<T>(L, q, i, d, X, ldx, err);
          }
        }
        // every written index must exceed all earlier ones (token order = lane order within a round)
        long long incl = widx;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const long long yv = __shfl_up_sync(0xffffffffu, incl, off);
          if (lane >= off) incl = incl > yv ? incl : yv;
        }
        long long before = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) before = 0;
        before = before > maxidx ? before : maxidx;
        if (__any_sync(0xffffffffu, widx > 0 && widx <= before)) simple = false;
        named += __popc(__ballot_sync(0xffffffffu, widx > 0));
        const long long rmax = __shfl_sync(0xffffffffu, incl, 31);
        maxidx = rmax > maxidx ? rmax : maxidx;
      }
      tok += total;
      prev_space = __shfl_sync(0xffffffffu, last == ' ' ? 1 : 0, 31) != 0;
      __syncwarp();  // the stage is rewritten by the next window
    }
    if (tok == 0 && lane == 0) report(err, i, E_NOLABEL);
    // a line that leaves some of its row's d entries to the caller's values
    if (lane == 0 && (!simple || named < d)) atomicAdd(reinterpret_cast<unsigned long long*>(meta) + 2, 1ull);
    if (!simple) {
      // Repeated or decreasing indices: replay the feature tokens in order so the last one written wins.
      if (lane == 0) {
        long long pos = s, t = 0;
        while (pos < e) {
          const unsigned c = __ldg(text + pos);
          if (c_end(c)) {  // blank (or NUL, already reported)
            ++pos;
            continue;
          }
          const LineBytes G{stage, 0u, pos, text, e};  // nothing staged: global memory from the token start
          if (t > 0) feature_token<T>(G, 0, i, d, X, ldx, err);
          ++t;
          while (pos < e && !c_end(__ldg(text + pos))) ++pos;
        }
      }
      __syncwarp();
    }
  }
}

template <typename T>
int parse_impl(db200_context* ctx, const unsigned char* text, long long bytes, int n, int d, T* X, long long ldx,
               T* y, int* lines_out, long long* partial_out) {
  const long long nchunks = bytes > 0 ? (bytes + CHUNK - 1) / CHUNK : 0;
  const size_t need = align_up((size_t)(nchunks + 1) * 4, 256) + align_up((size_t)(nchunks + 1) * 8, 256) +
                      align_up((size_t)(n + 2) * 8, 256) + 512;
  char* base = static_cast<char*>(slot_buffer(ctx, SLOT_SPARE, need));
  if (!base) return DB200_ERR_NOMEM;
  Carve cv{base};
  int* counts = cv.take<int>((size_t)nchunks + 1);
  long long* prefix = cv.take<long long>((size_t)nchunks + 1);
  long long* starts = cv.take<long long>((size_t)n + 2);
  long long* meta = cv.take<long long>(3);
  unsigned long long* err = cv.take<unsigned long long>(1);
  DB200_CUDA(ctx, cudaMemsetAsync(meta, 0, 3 * sizeof(long long), ctx->stream));
  DB200_CUDA(ctx, cudaMemsetAsync(err, 0xff, sizeof(unsigned long long), ctx->stream));
  const bool al = (reinterpret_cast<uintptr_t>(text) & 15u) == 0;
  if (nchunks > 0) {
    if (nchunks > 0x7fffffffLL) return fail(ctx, DB200_ERR_TOO_LARGE, "libsvm: text too large");
    if (al) nl_count_kernel<true><<<(unsigned)nchunks, NL_THREADS, 0, ctx->stream>>>(text, bytes, counts);
    else nl_count_kernel<false><<<(unsigned)nchunks, NL_THREADS, 0, ctx->stream>>>(text, bytes, counts);
    DB200_CUDA(ctx, cudaGetLastError());
    nl_scan_kernel<<<1, 1024, 0, ctx->stream>>>(counts, (int)nchunks, prefix, text, bytes, n, meta);
    DB200_CUDA(ctx, cudaGetLastError());
    if (al) nl_starts_kernel<true><<<(unsigned)nchunks, NL_THREADS, 0, ctx->stream>>>(text, bytes, prefix, n, starts);
    else nl_starts_kernel<false><<<(unsigned)nchunks, NL_THREADS, 0, ctx->stream>>>(text, bytes, prefix, n, starts);
    DB200_CUDA(ctx, cudaGetLastError());
    long long blocks = ((long long)n + PARSE_THREADS / 32 - 1) / (PARSE_THREADS / 32);
    const long long cap = (long long)ctx->num_sms * 8;
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    if (al)
      parse_kernel<T, true><<<(unsigned)blocks, PARSE_THREADS, 0, ctx->stream>>>(text, bytes, starts, meta, d, X,
                                                                                ldx, y, err);
    else
      parse_kernel<T, false><<<(unsigned)blocks, PARSE_THREADS, 0, ctx->stream>>>(text, bytes, starts, meta, d, X,
                                                                                 ldx, y, err);
    DB200_CUDA(ctx, cudaGetLastError());
    count_launch(ctx, 4);
  }
  // readback: lines parsed and the first error (pinned staging)
  DB200_CUDA(ctx, cudaMemcpyAsync(ctx->h_pinned, meta, 3 * sizeof(long long), cudaMemcpyDeviceToHost, ctx->stream));
  DB200_CUDA(ctx, cudaMemcpyAsync(reinterpret_cast<char*>(ctx->h_pinned) + 24, err, sizeof(unsigned long long),
                                  cudaMemcpyDeviceToHost, ctx->stream));
  DB200_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  long long hm[3];
  unsigned long long he;
  std::memcpy(hm, ctx->h_pinned, sizeof(hm));
  std::memcpy(&he, reinterpret_cast<char*>(ctx->h_pinned) + 24, sizeof(he));
  if (lines_out) *lines_out = (int)hm[1];
  if (partial_out) *partial_out = hm[2];
  if (he != ~0ull) {
    const long long line = (long long)(he >> 8);
    const unsigned code = (unsigned)(he & 0xffu);
    const char* what = code == E_INDEX     ? "feature index above d"
                       : code == E_HEX     ? "hexadecimal value (unsupported)"
                       : code == E_DIGITS  ? "value with more than 38 significant digits (unsupported)"
                       : code == E_NOLABEL ? "line without a label (only blanks)"
                       : code == E_NUL     ? "NUL byte in the line (unsupported)"
                                           : "NaN with a payload (unsupported)";
    const int st = (code == E_INDEX || code == E_NOLABEL) ? DB200_ERR_INVALID : DB200_ERR_UNSUPPORTED;
    return fail(ctx, st, "libsvm: line " + std::to_string(line + 1) + ": " + what);
  }
  return DB200_OK;
}

int parse_any(db200_context* ctx, const unsigned char* text, long long bytes, int n, int d, int dtype, void* X,
              long long ldx, void* y, int* lines_out, long long* partial_out) {
  return dtype == DB200_F32 ? parse_impl<float>(ctx, text, bytes, n, d, static_cast<float*>(X), ldx,
                                                static_cast<float*>(y), lines_out, partial_out)
                            : parse_impl<double>(ctx, text, bytes, n, d, static_cast<double*>(X), ldx,
                                                 static_cast<double*>(y), lines_out, partial_out);
}

// Read [off, off + len) of the file into dst with up to `threads` concurrent preads.
bool pread_parallel(int fd, char* dst, long long off, size_t len, int threads) {
  constexpr size_t MIN_PART = 4u << 20;
  int parts = (int)std::min<size_t>((size_t)threads, (len + MIN_PART - 1) / MIN_PART);
  if (parts < 1) parts = 1;
  const size_t step = (len + parts - 1) / parts;
  std::atomic<bool> ok{true};
  auto work = [&](int k) {
    size_t a = (size_t)k * step, b = std::min(len, a + step);
    while (a < b) {
      const ssize_t r = ::pread(fd, dst + a, b - a, off + (long long)a);
      if (r <= 0) {
        ok = false;
        return;
      }
      a += (size_t)r;
    }
  };
  std::vector<std::thread> pool;
  for (int k = 1; k < parts; ++k) pool.emplace_back(work, k);
  work(0);
  for (auto& t : pool) t.join();
  return ok;
}

}  // namespace

}  // namespace db200

using namespace db200;

extern "C" {

int db200_libsvm_parse(db200_context* ctx, const char* text, long long bytes, int n, int d, int dtype, void* X,
                       long long ldx, void* y, int* lines_out) {
  if (!ctx) return DB200_ERR_INVALID;
  if (lines_out) *lines_out = 0;
  if (bytes < 0 || n < 0 || d < 1 || ldx < d || (dtype != DB200_F32 && dtype != DB200_F64))
    return fail(ctx, DB200_ERR_INVALID, "db200_libsvm_parse: bad sizes or dtype");
  if (n == 0 || bytes == 0) return DB200_OK;
  if (!text || !X || !y) return fail(ctx, DB200_ERR_INVALID, "db200_libsvm_parse: null pointer");
  const auto* t = reinterpret_cast<const unsigned char*>(text);
  return parse_any(ctx, t, bytes, n, d, dtype, X, ldx, y, lines_out, nullptr);
}

int db200_read_libsvm(db200_context* ctx, const char* path, int n, int d, int dtype, void* X, long long ldx,
                      void* y, int* lines_out) {
  if (!ctx) return DB200_ERR_INVALID;
  if (lines_out) *lines_out = 0;
  if (!path || n < 0 || d < 1 || ldx < d || (dtype != DB200_F32 && dtype != DB200_F64))
    return fail(ctx, DB200_ERR_INVALID, "db200_read_libsvm: bad arguments");
  const int fd = ::open(path, O_RDONLY);
  if (fd < 0) return fail(ctx, DB200_ERR_INVALID, std::string("db200_read_libsvm: cannot open ") + path);
  struct stat stt;
  const long long bytes = (::fstat(fd, &stt) == 0) ? (long long)stt.st_size : -1;
  if (bytes < 0) {
    ::close(fd);
    return fail(ctx, DB200_ERR_INVALID, std::string("db200_read_libsvm: cannot stat ") + path);
  }
  if (n == 0 || bytes == 0) {
    ::close(fd);
    return DB200_OK;
  }
  if (!X || !y) {
    ::close(fd);
    return fail(ctx, DB200_ERR_INVALID, "db200_read_libsvm: null pointer");
  }
  const size_t es = dtype == DB200_F32 ? 4 : 8;
  const size_t xbytes = ((size_t)(n - 1) * (size_t)ldx + (size_t)d) * es, ybytes = (size_t)n * es;
  const size_t off_x = align_up((size_t)bytes, 256), off_y = off_x + align_up(xbytes, 256);
  char* dev = static_cast<char*>(io_buffer(ctx, off_y + ybytes));
  if (!dev) {
    ::close(fd);
    return DB200_ERR_NOMEM;
  }
  // File -> two pinned staging halves (parallel preads) -> device, each copy overlapping the next read.
  constexpr size_t PIECE = 32u << 20;
  int st = DB200_OK;
  if (ctx->h_stage_size < 2 * PIECE) {
    if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
    ctx->h_stage = nullptr;
    ctx->h_stage_size = 0;
    if (cudaMallocHost(&ctx->h_stage, 2 * PIECE) == cudaSuccess) ctx->h_stage_size = 2 * PIECE;
    else ctx->h_stage = nullptr;
  }
  char* stage = static_cast<char*>(ctx->h_stage);
  cudaEvent_t ev[2] = {nullptr, nullptr};
  if (!stage || cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) != cudaSuccess)
    st = fail(ctx, DB200_ERR_NOMEM, "db200_read_libsvm: pinned staging");
  const int threads = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  long long done = 0;
  for (int k = 0; st == DB200_OK && done < bytes; k ^= 1) {
    const size_t len = (size_t)std::min<long long>((long long)PIECE, bytes - done);
    if (cudaEventSynchronize(ev[k]) != cudaSuccess) st = fail(ctx, DB200_ERR_CUDA, "db200_read_libsvm: event");
    if (st == DB200_OK && !pread_parallel(fd, stage + k * PIECE, done, len, threads))
      st = fail(ctx, DB200_ERR_INVALID, std::string("db200_read_libsvm: short read of ") + path);
    if (st == DB200_OK &&
        (cudaMemcpyAsync(dev + done, stage + k * PIECE, len, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
         cudaEventRecord(ev[k], ctx->stream) != cudaSuccess))
      st = fail(ctx, DB200_ERR_CUDA, "db200_read_libsvm: copy to device");
    done += (long long)len;
  }
  ::close(fd);
  // Parse once into the device buffers.  Only lines that leave some of their row's entries unnamed need the
  // caller's X: then X's parsed rows go to the device first and the text is parsed again over them.  Rows and
  // labels past the last line are never touched, so only the parsed rows come back.
  int lines = 0;
  long long partial = 0;
  if (st == DB200_OK)
    st = parse_any(ctx, reinterpret_cast<const unsigned char*>(dev), bytes, n, d, dtype, dev + off_x, ldx,
                   dev + off_y, &lines, &partial);
  const size_t rows_bytes = lines > 0 ? ((size_t)(lines - 1) * (size_t)ldx + (size_t)d) * es : 0;
  if (st == DB200_OK && partial > 0) {
    if (cudaMemcpyAsync(dev + off_x, X, rows_bytes, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
      st = fail(ctx, DB200_ERR_CUDA, "db200_read_libsvm: copy to device");
    if (st == DB200_OK)
      st = parse_any(ctx, reinterpret_cast<const unsigned char*>(dev), bytes, n, d, dtype, dev + off_x, ldx,
                     dev + off_y, &lines, nullptr);
  }
  if (st == DB200_OK && lines > 0 &&
      (cudaMemcpyAsync(X, dev + off_x, rows_bytes, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
       cudaMemcpyAsync(y, dev + off_y, (size_t)lines * es, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
       cudaStreamSynchronize(ctx->stream) != cudaSuccess))
    st = fail(ctx, DB200_ERR_CUDA, "db200_read_libsvm: copy to host");
  if (lines_out) *lines_out = lines;
  cudaStreamSynchronize(ctx->stream);
  for (cudaEvent_t e : ev)
    if (e) cudaEventDestroy(e);
  return st;
}

}  // extern "C"
