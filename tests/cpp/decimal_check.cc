// Checks bhg_decimal.cuh's exact conversions on the host against the C++
// library: parse_double against std::from_chars (the conversion io.cc's
// read_csv uses) on random and edge-case strings, format_g6 against
// snprintf("%g") (what io.cc's write_vtk writes through an ostream) on random
// and edge-case doubles.  Prints "ok <parsed> <formatted>" or the first
// mismatch and exits non-zero.
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <system_error>

#include "bhg_decimal.cuh"

using namespace bhg::dec;

static Big A, B;

static bool check_parse(const std::string& s) {
  double ref = 0, got = 0;
  auto r = std::from_chars(s.data(), s.data() + s.size(), ref);
  const char* stop = nullptr;
  const int rc = parse_double(s.data(), s.data() + s.size(), &got, &stop, A, B);
  const int want = r.ec == std::errc() ? kOk : (r.ec == std::errc::result_out_of_range ? kRange : kInvalid);
  bool ok = rc == want;
  if (ok && want != kInvalid && stop != r.ptr) ok = false;
  if (ok && want == kOk) {
    uint64_t a, b;
    std::memcpy(&a, &ref, 8);
    std::memcpy(&b, &got, 8);
    if (std::isnan(ref)) ok = std::isnan(got) && std::signbit(ref) == std::signbit(got);
    else ok = a == b;
  }
  if (!ok) {
    std::printf("parse mismatch '%s': want rc %d v %.17g used %ld, got rc %d v %.17g used %ld\n", s.c_str(), want, ref,
                (long)(r.ptr - s.data()), rc, got, (long)(stop - s.data()));
  }
  return ok;
}

static bool check_format(double x) {
  char ref[64], got[32];
  std::snprintf(ref, sizeof ref, "%g", x);
  const int n = format_g6(x, got, A, B);
  got[n] = 0;
  if (std::strcmp(ref, got)) {
    std::printf("format mismatch %.17g (%a): want '%s' got '%s'\n", x, x, ref, got);
    return false;
  }
  return true;
}

int main(int argc, char** argv) {
  const long n = argc > 1 ? std::atol(argv[1]) : 200000;
  std::mt19937_64 rng(12345);
  long np = 0, nf = 0;
  const char* edge[] = {"0", "-0", "1", "-1", "1.", ".5", "-.5e-2", "00012", "1e", "1e+", "1e-", "1.5e3x", "0x1p3", "inf",
                        "-Infinity", "infin", "nan", "NaN(abc_1)", "nan(", "nan()", "+1", " 1", ".", "-", "e5", "1e400",
                        "1e-400", "4.9e-324", "2.4703282292062327e-324", "2.4703282292062328e-324",
                        "2.2250738585072011e-308", "2.2250738585072014e-308", "1.7976931348623157e308",
                        "1.7976931348623158e308", "1.7976931348623159e308", "9007199254740993", "9007199254740992.5",
                        "0.1", "0.30000000000000004", "123456789012345678901234567890", "1e22", "1e23",
                        "8.98846567431158e307", "4.4501477170144023e-308", "0.8238327648331624", "-3.4915082607549808"};
  for (const char* e : edge) {
    if (!check_parse(e)) return 1;
    ++np;
  }
  // long digit strings around halfway points: the exact decimal expansion
  // of a midpoint between two doubles, and one unit above and below it
  for (int i = 0; i < 2000; ++i) {
    uint64_t bits = rng() & 0x7fefffffffffffffull;
    double d;
    std::memcpy(&d, &bits, 8);
    double up = std::nextafter(d, INFINITY);
    char buf[1200];
    // midpoint printed with enough digits (the %.*e of the long double midpoint is not exact;
    // use the exact binary value of d with 800 digits and append '5' noise)
    std::snprintf(buf, sizeof buf, "%.780e", d);
    if (!check_parse(buf)) return 1;
    std::snprintf(buf, sizeof buf, "%.780e", up);
    if (!check_parse(buf)) return 1;
    np += 2;
  }
  std::uniform_int_distribution<int> nd(1, 25), ex(-340, 320), small(-30, 30);
  for (long i = 0; i < n; ++i) {
    std::string s;
    if (rng() & 1) s += '-';
    const int k = nd(rng);
    const int dot = (int)(rng() % (k + 2)) - 1;
    for (int j = 0; j < k; ++j) {
      if (j == dot) s += '.';
      s += (char)('0' + rng() % 10);
    }
    if (rng() % 3) {
      s += (rng() & 1) ? 'e' : 'E';
      const int r = (int)(rng() % 3);
      if (r == 1) s += '-';
      if (r == 2) s += '+';
      s += std::to_string(std::abs((rng() & 1) ? ex(rng) : small(rng)));
    }
    if (!check_parse(s)) return 1;
    ++np;
    // shortest round-trip strings of random doubles
    uint64_t bits = rng();
    double d;
    std::memcpy(&d, &bits, 8);
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.17g", d);
    if (!check_parse(buf)) return 1;
    ++np;
    if (!check_format(d)) return 1;
    ++nf;
    // values near decimal rounding ties of 6 digits
    const double base = std::ldexp((double)(rng() % 1000000 + 100000), small(rng)) * (rng() & 1 ? 1 : -1);
    const double tie = (std::floor(base) + 0.5);
    if (!check_format(tie) || !check_format(std::nextafter(tie, 0.0)) || !check_format(base)) return 1;
    nf += 3;
  }
  const double fedge[] = {0.0, -0.0, 1.0, 0.5, 1e-5, 1e-4, 9.999995e-5, 0.0001, 999999.5, 999999.4999, 9999995,
                          123456.5, 1e6, 1e100, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308, INFINITY,
                          -INFINITY, NAN, 0.30000000000000004, 2.5, 3.5, 100000.5, 0.000123456789};
  for (double d : fedge) {
    if (!check_format(d)) return 1;
    ++nf;
  }
  std::printf("ok %ld %ld\n", np, nf);
  return 0;
}
