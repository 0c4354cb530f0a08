// p-values of the rank and linear-complexity tests (host, f64).
//
// Restates src/stats.rs of the modlin crate; compiled with -ffp-contract=off
// (Rust never fuses a*b+c) so every p-value, including the exact 1e-307 floor
// and 1.0 at the mode, matches the reference bit for bit.
#include <charconv>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/modlin.h"

namespace {

constexpr double kPFloor = 1e-307;  // src/stats.rs:16
constexpr double kLn2 = 0.693147180559945309417232121458176568;

// f64::powi: compiler-rt's __powidf2 square-and-multiply.
double powi(double base, int e) {
  const bool recip = e < 0;
  double r = 1.0;
  for (;;) {
    if (e & 1) r *= base;
    e /= 2;
    if (e == 0) break;
    base *= base;
  }
  return recip ? 1.0 / r : r;
}

// src/stats.rs:19-23: ln p = e*ln2 + ln(p / 2^e), fused as Rust's mul_add.
double ln_u64(uint64_t p) {
  const int e = 63 - __builtin_clzll(p);
  const double mant = static_cast<double>(p) / static_cast<double>(1ULL << e);
  return std::fma(static_cast<double>(e), kLn2, std::log(mant));
}

// src/stats.rs:26-41: sum_{j=a..b} ln(1 - p^-j), stopping once p^-j < 1e-18.
double sum_ln_1m(double p, size_t a, size_t b) {
  if (a > b) return 0.0;
  const double inv = 1.0 / p;
  double pj = powi(inv, static_cast<int>(a));
  double s = 0.0;
  for (size_t j = a; j <= b; ++j) {
    if (pj < 1e-18) break;
    s += std::log1p(-pj);
    pj *= inv;
  }
  return s;
}

double clamp(double x, double lo, double hi) { return x < lo ? lo : (x > hi ? hi : x); }

}  // namespace

extern "C" double modlin_corank_prob(uint64_t p, size_t n, size_t d) {
  if (d > n) return 0.0;
  const double pf = static_cast<double>(p);
  double lp = -powi(static_cast<double>(d), 2) * ln_u64(p);
  lp = lp + 2.0 * sum_ln_1m(pf, d + 1, n);
  lp = lp - sum_ln_1m(pf, 1, n - d);
  return lp < -745.0 ? 0.0 : std::exp(lp);
}

extern "C" double modlin_corank_tail_pvalue(uint64_t p, size_t n, size_t c) {
  if (c == 0) return 1.0;
  double s = 0.0;
  for (size_t d = c; d <= n; ++d) {
    const double pr = modlin_corank_prob(p, n, d);
    if (pr == 0.0) break;
    s += pr;
  }
  return clamp(s, kPFloor, 1.0);
}

extern "C" double modlin_lc_left_tail_pvalue(uint64_t p, size_t n, size_t ell) {
  if (ell >= n) return 1.0;
  const double lnp = ln_u64(p);
  double pr;
  if (2 * ell <= n) {
    const double a = static_cast<double>(2 * ell + 1) * lnp;
    const double ln_num = a > 0.0 ? a + std::log1p(std::exp(-a)) : std::log1p(std::exp(a));
    const double ln_den = static_cast<double>(n) * lnp + std::log(static_cast<double>(p) + 1.0);
    pr = std::exp(ln_num - ln_den);
  } else {
    const double hi = std::exp((static_cast<double>(n) - 2.0 * static_cast<double>(ell)) * lnp);
    const double lo = std::exp(-static_cast<double>(n) * lnp);
    pr = 1.0 - (hi - lo) / (static_cast<double>(p) + 1.0);
  }
  return clamp(pr, kPFloor, 1.0);
}

// src/stats.rs:129-137: "0", "1", otherwise Rust's `{:?}` for f64 — the
// shortest round-trip digits, in scientific form (exponent without '+' or
// padding) when |x| < 1e-4 or |x| >= 1e16, else positional with at least one
// fractional digit.
extern "C" int modlin_pretty_p_value(double p, char* buf, size_t cap) {
  std::string out;
  if (p == 0.0) {
    out = "0";
  } else if (p == 1.0) {
    out = "1";
  } else if (std::isnan(p)) {
    out = "NaN";
  } else if (std::isinf(p)) {
    out = p > 0 ? "inf" : "-inf";
  } else {
    char tmp[64];
    auto res = std::to_chars(tmp, tmp + sizeof tmp, p, std::chars_format::scientific);
    std::string sci(tmp, res.ptr);
    const size_t epos = sci.find('e');
    std::string mant = sci.substr(0, epos);
    const int e10 = std::atoi(sci.c_str() + epos + 1);
    bool neg = false;
    if (!mant.empty() && mant[0] == '-') {
      neg = true;
      mant.erase(0, 1);
    }
    std::string digits;
    for (char ch : mant)
      if (ch != '.') digits.push_back(ch);
    const double a = std::fabs(p);
    if (neg) out.push_back('-');
    if (a < 1e-4 || a >= 1e16) {
      out.push_back(digits[0]);
      if (digits.size() > 1) {
        out.push_back('.');
        out.append(digits, 1, std::string::npos);
      }
      out += "e" + std::to_string(e10);
    } else if (e10 < 0) {
      out += "0.";
      out.append(static_cast<size_t>(-e10 - 1), '0');
      out += digits;
    } else {
      const size_t ip = static_cast<size_t>(e10) + 1;
      if (digits.size() <= ip) {
        out += digits;
        out.append(ip - digits.size(), '0');
        out += ".0";
      } else {
        out.append(digits, 0, ip);
        out.push_back('.');
        out.append(digits, ip, std::string::npos);
      }
    }
  }
  if (buf && cap) std::snprintf(buf, cap, "%s", out.c_str());
  return static_cast<int>(out.size());
}
