// Exact conversions between decimal text and binary64, for host and device.
//
// parse_double reads a number the way std::from_chars(first, last, double&)
// does in its general format (the conversion io.cc's parse_field relies on):
// an optional '-', decimal digits with an optional '.' (at least one
// digit), an optional exponent ('e' or 'E', optional sign, at least one
// digit; without digits the 'e' is not part of the number), or "inf",
// "infinity", "nan", "nan(chars)" in any case.  No leading '+', no leading
// blanks, no hexadecimal.  The value is rounded to nearest, ties to even,
// from the exact decimal value; a nonzero value that rounds to zero or beyond
// the largest finite double is out of range.
//
// format_g6 writes a double as printf's "%g" (precision 6) does, which is
// what an std::ostream with default settings writes (io.cc's write_vtk):
// the exact binary value rounded to 6 significant digits, ties to even.
//
// Both are exact by construction, not by approximation: the decimal value
// and the candidate are compared as integers (a small fixed-size big
// integer), so the result is the correctly rounded one for every input.
// The big integers hold 3072 bits; inputs keep their first kMaxDigits
// significant digits (any further nonzero digit is remembered as a sticky
// bit), which decides every rounding exactly because a double's exact
// decimal expansion, or a midpoint between two doubles, never has more than
// 767 significant digits.
#pragma once

#include <stdint.h>

#if defined(__CUDACC__)
#define BHG_HD __host__ __device__ __forceinline__
#else
#define BHG_HD inline
#endif

namespace bhg {
namespace dec {

constexpr int kLimbs = 96;
constexpr int kMaxDigits = 800;

struct Big {
  int n;  // limbs in use (no leading zero limbs)
  uint32_t d[kLimbs];
};

BHG_HD void big_set(Big& a, uint64_t v) {
  a.d[0] = (uint32_t)v;
  a.d[1] = (uint32_t)(v >> 32);
  a.n = a.d[1] ? 2 : (a.d[0] ? 1 : 0);
}

BHG_HD void big_trim(Big& a) {
  while (a.n > 0 && a.d[a.n - 1] == 0) --a.n;
}

BHG_HD void big_mul_add(Big& a, uint32_t m, uint32_t add) {
  uint64_t carry = add;
  for (int i = 0; i < a.n; ++i) {
    const uint64_t t = (uint64_t)a.d[i] * m + carry;
    a.d[i] = (uint32_t)t;
    carry = t >> 32;
  }
  if (carry && a.n < kLimbs) a.d[a.n++] = (uint32_t)carry;
}

BHG_HD void big_mul_pow5(Big& a, int k) {
  const uint32_t p13 = 1220703125u;  // 5^13
  for (; k >= 13; k -= 13) big_mul_add(a, p13, 0);
  uint32_t r = 1;
  for (; k > 0; --k) r *= 5;
  if (r != 1) big_mul_add(a, r, 0);
}

BHG_HD void big_shl(Big& a, int s) {
  if (a.n == 0 || s == 0) return;
  const int w = s >> 5, b = s & 31;
  int n = a.n + w + 1;
  if (n > kLimbs) n = kLimbs;
  for (int i = n - 1; i >= 0; --i) {
    const int j = i - w;
    uint32_t v = 0;
    if (j >= 0 && j < a.n) v = b ? (a.d[j] << b) : a.d[j];
    if (b && j - 1 >= 0 && j - 1 < a.n) v |= a.d[j - 1] >> (32 - b);
    a.d[i] = v;
  }
  a.n = n;
  big_trim(a);
}

BHG_HD void big_shr1(Big& a) {
  for (int i = 0; i < a.n; ++i) a.d[i] = (a.d[i] >> 1) | (i + 1 < a.n ? a.d[i + 1] << 31 : 0u);
  big_trim(a);
}

BHG_HD int big_cmp(const Big& a, const Big& b) {
  if (a.n != b.n) return a.n < b.n ? -1 : 1;
  for (int i = a.n - 1; i >= 0; --i)
    if (a.d[i] != b.d[i]) return a.d[i] < b.d[i] ? -1 : 1;
  return 0;
}

// a -= b, a >= b
BHG_HD void big_sub(Big& a, const Big& b) {
  int64_t borrow = 0;
  for (int i = 0; i < a.n; ++i) {
    int64_t t = (int64_t)a.d[i] - (i < b.n ? (int64_t)b.d[i] : 0) - borrow;
    borrow = t < 0;
    a.d[i] = (uint32_t)(t + (borrow << 32));
  }
  big_trim(a);
}

BHG_HD int big_bitlen(const Big& a) {
  if (a.n == 0) return 0;
  uint32_t top = a.d[a.n - 1];
  int b = 0;
  while (top) ++b, top >>= 1;
  return 32 * (a.n - 1) + b;
}

BHG_HD uint64_t big_low64(const Big& a) {
  return (a.n > 0 ? a.d[0] : 0u) | ((uint64_t)(a.n > 1 ? a.d[1] : 0u) << 32);
}

// q = floor(a / b) for a quotient below 2^qbits (qbits <= 63); a becomes
// the remainder; b is used as scratch and restored.
BHG_HD uint64_t big_divmod(Big& a, Big& b, int qbits) {
  big_shl(b, qbits);
  uint64_t q = 0;
  for (int i = qbits; i >= 0; --i) {
    if (big_cmp(a, b) >= 0) {
      big_sub(a, b);
      q |= 1ull << i;
    }
    if (i > 0) big_shr1(b);
  }
  return q;
}

BHG_HD double make_double(bool neg, uint64_t m, int e2) {
  // m * 2^e2 exactly (m < 2^53, and the product is a representable double)
  double v = (double)m;
  while (e2 > 0) {
    const int s = e2 > 60 ? 60 : e2;
    v *= (double)(1ull << s);
    e2 -= s;
  }
  while (e2 < 0) {
    const int s = -e2 > 60 ? 60 : -e2;
    // scaling by an exact power of two is exact as long as no bit falls off
    // the subnormal end, which the caller's rounding guarantees for the
    // final product; intermediate products stay normal (m < 2^53, steps of
    // 2^60 from at most 2^53 down to 2^-1074)
    v *= 1.0 / (double)(1ull << s);
    e2 += s;
  }
  return neg ? -v : v;
}

BHG_HD double from_bits(uint64_t u) {
  union {
    uint64_t u;
    double f;
  } v;
  v.u = u;
  return v.f;
}

BHG_HD bool is_digit(char c) { return c >= '0' && c <= '9'; }
BHG_HD char lower(char c) { return (char)(c | 0x20); }

enum { kOk = 0, kInvalid = 1, kRange = 2 };

// See the file comment.  *stop: first character after the number (first
// on kInvalid).  Returns kOk, kInvalid or kRange.
BHG_HD int parse_double(const char* first, const char* last, double* out, const char** stop, Big& w, Big& b) {
  const char* s = first;
  *stop = first;
  const bool neg = s < last && *s == '-';
  if (neg) ++s;
  if (s < last && lower(*s) == 'i') {  // inf, infinity
    if (last - s >= 3 && lower(s[1]) == 'n' && lower(s[2]) == 'f') {
      s += 3;
      const char* rest = "inity";
      int k = 0;
      while (k < 5 && s + k < last && lower(s[k]) == rest[k]) ++k;
      if (k == 5) s += 5;
      *out = from_bits((neg ? 0x8000000000000000ull : 0ull) | 0x7ff0000000000000ull);
      *stop = s;
      return kOk;
    }
    return kInvalid;
  }
  if (s < last && lower(*s) == 'n') {  // nan, nan(n-char-sequence)
    if (last - s >= 3 && lower(s[1]) == 'a' && lower(s[2]) == 'n') {
      s += 3;
      if (s < last && *s == '(') {
        const char* t = s + 1;
        while (t < last && (is_digit(*t) || (lower(*t) >= 'a' && lower(*t) <= 'z') || *t == '_')) ++t;
        if (t < last && *t == ')') s = t + 1;
      }
      *out = from_bits((neg ? 0x8000000000000000ull : 0ull) | 0x7ff8000000000000ull);
      *stop = s;
      return kOk;
    }
    return kInvalid;
  }
  // significant digits go into w in chunks of 9 (and, while they fit, into
  // w64 for the 128-bit fast path)
  big_set(w, 0);
  uint64_t w64 = 0;
  int ndig = 0, chunk_len = 0;
  uint32_t chunk = 0;
  bool any = false, sticky = false;
  long exp10 = 0;
  const uint32_t pow10[10] = {1u, 10u, 100u, 1000u, 10000u, 100000u, 1000000u, 10000000u, 100000000u, 1000000000u};
  for (int frac = 0; frac < 2; ++frac) {
    if (frac) {
      if (!(s < last && *s == '.')) break;
      ++s;
    }
    for (; s < last && is_digit(*s); ++s) {
      any = true;
      const uint32_t c = (uint32_t)(*s - '0');
      if (ndig == 0 && c == 0) {  // leading zero
        if (frac) --exp10;
        continue;
      }
      if (ndig < kMaxDigits) {
        if (ndig < 19) w64 = w64 * 10 + c;
        chunk = chunk * 10 + c;
        if (++chunk_len == 9) {
          big_mul_add(w, pow10[9], chunk);
          chunk = 0, chunk_len = 0;
        }
        ++ndig;
        if (frac) --exp10;
      } else {
        if (c) sticky = true;
        if (!frac) ++exp10;
      }
    }
  }
  if (!any) return kInvalid;
  if (chunk_len) big_mul_add(w, pow10[chunk_len], chunk);
  if (s < last && lower(*s) == 'e') {
    const char* t = s + 1;
    bool eneg = false;
    if (t < last && (*t == '+' || *t == '-')) eneg = *t++ == '-';
    if (t < last && is_digit(*t)) {
      long e = 0;
      for (; t < last && is_digit(*t); ++t)
        if (e < 100000000L) e = e * 10 + (*t - '0');
      exp10 += eneg ? -e : e;
      s = t;
    }
  }
  *stop = s;
  if (ndig == 0) {
    *out = neg ? -0.0 : 0.0;
    return kOk;
  }
  // the value lies in [10^(ndig + exp10 - 1), 10^(ndig + exp10))
  if (ndig + exp10 > 310) return kRange;
  if (ndig + exp10 < -324) return kRange;  // below 10^-325: rounds to zero
  // value = q_int * 2^e + (a fraction, and the sticky bit) with q_int of 55-57 bits
  uint64_t q;
  int e;
  bool fast = false;
  if (ndig <= 19 && !sticky && exp10 >= -27 && exp10 <= 27) {
    // fast path: w and 5^|exp10| (< 2^63) fit in 64 bits, the product or
    // the scaled dividend in 128
    uint64_t p5 = 1;
    for (long i = 0; i < (exp10 < 0 ? -exp10 : exp10); ++i) p5 *= 5u;
    if (exp10 >= 0) {
      const unsigned __int128 N = (unsigned __int128)w64 * p5;  // value = N * 2^exp10
      int bl = 0;
      for (unsigned __int128 v = N; v; v >>= 1) ++bl;
      if (bl <= 57) {
        q = (uint64_t)N << (57 - bl);
        e = (int)exp10 - (57 - bl);
      } else {
        const int sh = bl - 57;
        q = (uint64_t)(N >> sh);
        if (N & ((((unsigned __int128)1) << sh) - 1u)) sticky = true;
        e = (int)exp10 + sh;
      }
      fast = true;
    } else {
      int blw = 0, bld = 0;
      for (uint64_t v = w64; v; v >>= 1) ++blw;
      for (uint64_t v = p5; v; v >>= 1) ++bld;
      const int t = 56 + bld - blw;  // value = (w64 * 2^t / p5) * 2^(exp10 - t)
      if (t >= 0) {
        const unsigned __int128 N = (unsigned __int128)w64 << t;  // below 2^(56 + bld) <= 2^119
        q = (uint64_t)(N / p5);
        if (N % p5) sticky = true;
        e = (int)exp10 - t;
        fast = true;
      }
    }
  }
  if (!fast) {
    if (exp10 >= 0) {
      big_mul_pow5(w, (int)exp10);  // value = w * 2^exp10
      const int bl = big_bitlen(w);
      if (bl <= 57) {
        q = big_low64(w) << (57 - bl);
        e = (int)exp10 - (57 - bl);
      } else {
        const int sh = bl - 57;
        // the top 57 bits, the rest into the sticky bit
        for (int i = 0; i < (sh >> 5); ++i)
          if (w.d[i]) sticky = true;
        if (sh & 31)
          if (w.d[sh >> 5] & ((1u << (sh & 31)) - 1u)) sticky = true;
        uint64_t v = 0;
        for (int i = 0; i < 57; ++i) {
          const int bit = sh + i;
          if ((w.d[bit >> 5] >> (bit & 31)) & 1u) v |= 1ull << i;
        }
        q = v;
        e = (int)exp10 + sh;
      }
    } else {
      const int k = (int)-exp10;  // value = w / (5^k * 2^k)
      big_set(b, 1);
      big_mul_pow5(b, k);
      int t = 56 + big_bitlen(b) - big_bitlen(w);
      if (t >= 0) big_shl(w, t);
      else big_shl(b, -t);
      q = big_divmod(w, b, 58);  // below 2^57
      if (w.n) sticky = true;
      e = -k - t;
    }
  }
  // round q * 2^e (+ sticky) to a double
  int bq = 0;
  for (uint64_t v = q; v; v >>= 1) ++bq;
  const int E2 = bq - 1 + e;  // value in [2^E2, 2^(E2 + 1))
  if (E2 > 1023) return kRange;
  const int mbits = E2 >= -1022 ? 53 : E2 + 1075;
  const int shift = bq - mbits;  // >= 2
  if (shift >= 64) return kRange;  // below 2^-1081: rounds to zero
  uint64_t m = q >> shift;
  const uint64_t rem = q & ((1ull << shift) - 1ull);
  const uint64_t half = 1ull << (shift - 1);
  if (rem > half || (rem == half && (sticky || (m & 1u)))) ++m;
  int ex = E2 - mbits + 1;  // value = m * 2^ex
  if (m == (1ull << 53)) {  // carried into the next binade
    m >>= 1;
    ++ex;
    if (ex + 52 > 1023) return kRange;
  }
  if (m == 0) return kRange;
  *out = make_double(neg, m, ex);
  return kOk;
}

// Writes x as "%g" (precision 6) into out (at most 13 characters, no
// terminator); returns the length.  a and b are scratch.
BHG_HD int format_g6(double x, char* out, Big& a, Big& b) {
  int len = 0;
  union {
    double f;
    uint64_t u;
  } bits;
  bits.f = x;
  const bool neg = bits.u >> 63;
  const int bexp = (int)((bits.u >> 52) & 0x7ff);
  uint64_t M = bits.u & ((1ull << 52) - 1ull);
  if (bexp == 0x7ff) {
    if (neg) out[len++] = '-';
    if (M) out[len++] = 'n', out[len++] = 'a', out[len++] = 'n';
    else out[len++] = 'i', out[len++] = 'n', out[len++] = 'f';
    return len;
  }
  if (neg) out[len++] = '-';
  if (bexp == 0 && M == 0) {
    out[len++] = '0';
    return len;
  }
  int E;
  if (bexp == 0) E = -1074;
  else M |= 1ull << 52, E = bexp - 1075;  // |x| = M * 2^E
  // decimal exponent X: 10^X <= |x| < 10^(X + 1); estimated from the binary
  // exponent (log10(2) ~ 0.30103), then corrected exactly
  int bl = 0;
  for (uint64_t v = M; v; v >>= 1) ++bl;
  int X = (int)(((long)(bl - 1 + E) * 78913L) >> 18);  // floor((bl-1+E) * log10 2)
  // D = round(|x| / 10^(X - 5)); retried when X was one too small or large
  uint64_t D = 0;
  for (int attempt = 0; attempt < 4; ++attempt) {
    const int p = X - 5;
    // fast path: |x| / 10^p = A / B with A = M 2^max(E,0) 10^max(-p,0) and
    // B = 2^max(-E,0) 10^max(p,0), exact in 128 bits for moderate exponents
    // (10^k < 2^(3.33 k): the bounds below keep A < 2^127 and B < 2^125)
    const int e_up = E > 0 ? E : 0, e_dn = E < 0 ? -E : 0, p_up = p < 0 ? -p : 0, p_dn = p > 0 ? p : 0;
    if (53 + e_up + (p_up * 10 + 2) / 3 <= 126 && e_dn + (p_dn * 10 + 2) / 3 <= 124) {
      unsigned __int128 A = (unsigned __int128)M << e_up, B = (unsigned __int128)1 << e_dn;
      for (int i = 0; i < p_up; ++i) A *= 10u;
      for (int i = 0; i < p_dn; ++i) B *= 10u;
      const unsigned __int128 qv = A / B, r = A - qv * B;
      if (qv < 100000u) {
        --X;
        continue;
      }
      if (qv >= 1000000u) {
        ++X;
        continue;
      }
      D = (uint64_t)qv;
      if (2 * r > B || (2 * r == B && (D & 1u))) ++D;
      if (D == 1000000u) D = 100000u, ++X;
      break;
    }
    big_set(a, M);
    big_set(b, 1);
    if (E >= 0) big_shl(a, E);
    else big_shl(b, -E);
    if (p >= 0) big_mul_pow5(b, p), big_shl(b, p);
    else big_mul_pow5(a, -p), big_shl(a, -p);
    // |x| / 10^p lies in [10^5, 10^6) when X is right: quotient below 2^24
    // (a too small X gives a quotient of at most 10^7, below 2^24 too)
    const uint64_t qv = big_divmod(a, b, 24);  // b comes back unchanged
    if (qv < 100000u) {  // X too large
      --X;
      continue;
    }
    if (qv >= 1000000u) {  // X too small
      ++X;
      continue;
    }
    // round: compare 2 * remainder with the divisor
    big_shl(a, 1);
    const int c = big_cmp(a, b);
    D = qv;
    if (c > 0 || (c == 0 && (D & 1u))) ++D;
    if (D == 1000000u) D = 100000u, ++X;
    break;
  }
  // six digits of D
  char dig[6];
  for (int i = 5; i >= 0; --i) dig[i] = (char)('0' + D % 10), D /= 10;
  int nd = 6;
  while (nd > 1 && dig[nd - 1] == '0') --nd;  // %g drops trailing zeros
  if (X < -4 || X >= 6) {
    out[len++] = dig[0];
    if (nd > 1) {
      out[len++] = '.';
      for (int i = 1; i < nd; ++i) out[len++] = dig[i];
    }
    out[len++] = 'e';
    int ax = X;
    if (ax < 0) out[len++] = '-', ax = -ax;
    else out[len++] = '+';
    if (ax >= 100) out[len++] = (char)('0' + ax / 100), ax %= 100, out[len++] = (char)('0' + ax / 10);
    else out[len++] = (char)('0' + ax / 10);
    out[len++] = (char)('0' + ax % 10);
  } else if (X >= 0) {
    for (int i = 0; i <= X; ++i) out[len++] = i < 6 ? dig[i] : '0';
    if (nd > X + 1) {
      out[len++] = '.';
      for (int i = X + 1; i < nd; ++i) out[len++] = dig[i];
    }
  } else {
    out[len++] = '0';
    out[len++] = '.';
    for (int i = 0; i < -X - 1; ++i) out[len++] = '0';
    for (int i = 0; i < nd; ++i) out[len++] = dig[i];
  }
  return len;
}

}  // namespace dec
}  // namespace bhg
