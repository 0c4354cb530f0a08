// `modlin` — the -R/-L command line of the modlin crate (src/main.rs,
// src/cli.rs) on top of libmodlin_gpu.so. stdout is byte-identical to the
// reference's; progress and timing go to stderr.
//
// The reference chooses its generator at build time (a Cargo feature,
// src/prng.rs:21-25); here it is `--prng KIND` (xoroshiro128pp, mixmax,
// mixmax17, mixmax256) with a build-time default. `--kernel plain|tc|auto`
// selects the rank trailing-update kernel.
#include <chrono>
#include <cinttypes>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/modlin.h"

#ifndef MODLIN_DEFAULT_PRNG
#define MODLIN_DEFAULT_PRNG "mixmax17"
#endif

namespace {

const char* kUsage =
    "Usage: modlin [OPTIONS] --modulus <MODULUS> <--rank <SIDE>|--linear-complexity <LENGTH>> [REPS]";

[[noreturn]] void die(const std::string& msg) {  // src/cli.rs:184-189: clap-style error, exit 2
  std::fprintf(stderr, "error: %s\n\n%s\n\nFor more information, try '--help'.\n", msg.c_str(), kUsage);
  std::exit(2);
}

// src/cli.rs:53-66: decimal, or 0x/0o/0b prefixed; '_' separators allowed.
bool parse_u64(const std::string& value, uint64_t* out) {
  size_t a = 0, b = value.size();
  while (a < b && std::isspace((unsigned char)value[a])) ++a;
  while (b > a && std::isspace((unsigned char)value[b - 1])) --b;
  std::string t = value.substr(a, b - a);
  int radix = 10;
  if (t.size() >= 2 && t[0] == '0') {
    const char c = t[1];
    if (c == 'x' || c == 'X') radix = 16;
    if (c == 'o' || c == 'O') radix = 8;
    if (c == 'b' || c == 'B') radix = 2;
    if (radix != 10) t = t.substr(2);
  }
  std::string digits;
  for (char c : t)
    if (c != '_') digits.push_back(c);
  if (digits.empty()) return false;
  unsigned __int128 v = 0;
  for (char c : digits) {
    int d;
    if (c >= '0' && c <= '9') d = c - '0';
    else if (c >= 'a' && c <= 'z') d = c - 'a' + 10;
    else if (c >= 'A' && c <= 'Z') d = c - 'A' + 10;
    else return false;
    if (d >= radix) return false;
    v = v * radix + d;
    if (v > UINT64_MAX) return false;
  }
  *out = (uint64_t)v;
  return true;
}

// src/cli.rs:16-48: s/m/h/d suffixes, bare number = milliseconds.
bool parse_duration(const std::string& value, double* ms) {
  if (value.empty()) return false;
  double total = 0;
  std::string acc;
  for (char c : value) {
    if (c >= '0' && c <= '9') {
      acc.push_back(c);
    } else if (std::isspace((unsigned char)c)) {
      continue;
    } else {
      if (acc.empty()) return false;
      const double d = std::strtod(acc.c_str(), nullptr);
      if (c == 's') total += d * 1e3;
      else if (c == 'm') total += d * 60e3;
      else if (c == 'h') total += d * 3600e3;
      else if (c == 'd') total += d * 86400e3;
      else return false;
      acc.clear();
    }
  }
  if (!acc.empty()) total += std::strtod(acc.c_str(), nullptr);
  *ms = total;
  return true;
}

// src/main.rs:51-60
std::string format_memory(double bytes) {
  const double gib = 1073741824.0, mib = 1048576.0;
  char buf[64];
  if (bytes >= gib)
    std::snprintf(buf, sizeof buf, "%.3f GiB", bytes / gib);
  else
    std::snprintf(buf, sizeof buf, "%.3f MiB", bytes / mib);
  return buf;
}

std::string pretty(double p) {
  char buf[64];
  modlin_pretty_p_value(p, buf, sizeof buf);
  return buf;
}

struct Progress {
  double interval_ms;
  std::chrono::steady_clock::time_point start, last;
  const char* item;
};

void progress_cb(void* ctx, size_t done, size_t total) {
  auto* pr = static_cast<Progress*>(ctx);
  const auto now = std::chrono::steady_clock::now();
  if (std::chrono::duration<double, std::milli>(now - pr->last).count() >= pr->interval_ms) {
    pr->last = now;
    std::fprintf(stderr, "%zu/%zu %ss\n", done, total, pr->item);
  }
}

int prng_kind(const std::string& s) {
  if (s == "xoroshiro128pp") return MODLIN_PRNG_XOROSHIRO128PP;
  if (s == "mixmax" || s == "mixmax240") return MODLIN_PRNG_MIXMAX240;
  if (s == "mixmax17") return MODLIN_PRNG_MIXMAX17;
  if (s == "mixmax256") return MODLIN_PRNG_MIXMAX256;
  return -1;
}

}  // namespace

int main(int argc, char** argv) {
  bool have_r = false, have_l = false, have_p = false;
  uint64_t side = 0, length = 0, modulus = 0, seed = 0, reps = 1;
  double log_ms = 10000;
  std::string prng = MODLIN_DEFAULT_PRNG, kernel = "auto";
  bool have_reps = false;
  auto need = [&](int& i, const char* name) -> std::string {
    if (i + 1 >= argc) die(std::string("a value is required for '") + name + "' but none was supplied");
    return argv[++i];
  };
  for (int i = 1; i < argc; ++i) {
    std::string a = argv[i];
    std::string val;
    const size_t eq = a.find('=');
    const bool longopt = a.rfind("--", 0) == 0;
    if (longopt && eq != std::string::npos) {
      val = a.substr(eq + 1);
      a = a.substr(0, eq);
    }
    auto get = [&](const char* name) { return (longopt && eq != std::string::npos) ? val : need(i, name); };
    if (a == "-h" || a == "--help") {
      std::printf("Runs a modular rank or linear-complexity test on the GPU.\n\n%s\n", kUsage);
      return 0;
    } else if (a == "-R" || a == "--rank") {
      if (!parse_u64(get("--rank <SIDE>"), &side)) die("invalid value for '--rank <SIDE>'");
      have_r = true;
    } else if (a == "-L" || a == "--linear-complexity") {
      if (!parse_u64(get("--linear-complexity <LENGTH>"), &length)) die("invalid value for '--linear-complexity'");
      have_l = true;
    } else if (a == "-p" || a == "--modulus") {
      if (!parse_u64(get("--modulus <MODULUS>"), &modulus)) die("invalid value for '--modulus <MODULUS>'");
      have_p = true;
    } else if (a == "-S" || a == "--seed") {
      const std::string v = get("--seed <SEED>");
      if (!parse_u64(v, &seed)) die("invalid value '" + v + "' for '--seed <SEED>': invalid integer");
    } else if (a == "--log-interval") {
      if (!parse_duration(get("--log-interval <LOG_INTERVAL>"), &log_ms)) die("invalid value for '--log-interval'");
    } else if (a == "--prng") {
      prng = get("--prng <KIND>");
    } else if (a == "--kernel") {
      kernel = get("--kernel <plain|tc|auto>");
    } else if (!a.empty() && a[0] == '-' && a != "-") {
      die("unexpected argument '" + a + "' found");
    } else {
      if (have_reps) die("unexpected argument '" + a + "' found");
      if (!parse_u64(a, &reps)) die("invalid value '" + a + "' for '[REPS]'");
      have_reps = true;
    }
  }
  if (have_r == have_l) die("the following required arguments were not provided:\n  <--rank <SIDE>|--linear-complexity <LENGTH>>");
  if (!have_p) die("the following required arguments were not provided:\n  --modulus <MODULUS>");
  // src/cli.rs:161-181
  const uint64_t size = have_r ? side : length;
  if (size < 2) die("SIDE/LENGTH must be at least 2");
  if (have_r && size > 0 && size > UINT64_MAX / size) die("SIDE is too large: SIDE² overflows a 64-bit index");
  if (reps < 1) die("reps must be at least 1");
  if (modulus < 2) die("modulus must be at least 2");
  if (modulus >= (1ULL << 63)) die("modulus must be below 2⁶³");
  modlin_field field;
  modlin_field_new(modulus, &field);
  {
    // primal::is_prime: deterministic Miller-Rabin with the first 12 primes.
    static const uint64_t bases[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    bool prime = modulus >= 2;
    for (uint64_t q : bases)
      if (modulus % q == 0) prime = modulus == q;
    if (prime && modulus > 37) {
      uint64_t d = modulus - 1;
      int s = 0;
      while (!(d & 1)) d >>= 1, ++s;
      auto mulm = [&](uint64_t x, uint64_t y) { return (uint64_t)((unsigned __int128)x * y % modulus); };
      for (uint64_t a : bases) {
        uint64_t x = 1, b = a % modulus, e = d;
        while (e) {
          if (e & 1) x = mulm(x, b);
          b = mulm(b, b);
          e >>= 1;
        }
        if (x == 1 || x == modulus - 1) continue;
        bool comp = true;
        for (int r = 1; r < s && comp; ++r) {
          x = mulm(x, x);
          if (x == modulus - 1) comp = false;
        }
        if (comp) {
          prime = false;
          break;
        }
      }
    }
    if (!prime) die("modulus must be prime");
  }
  const int kind = prng_kind(prng);
  if (kind < 0) die("invalid value '" + prng + "' for '--prng <KIND>'");
  modlin_rank_opts ropts{kernel == "plain" ? MODLIN_RANK_PLAIN : (kernel == "tc" ? MODLIN_RANK_TC : MODLIN_RANK_AUTO),
                         0};

  std::printf("Generator: %s\n", modlin_prng_name(kind));  // src/main.rs:23
  std::printf("Seed: 0x%016" PRIx64 "\n", seed);           // src/main.rs:26
  std::fflush(stdout);
  int err = 0;
  modlin_prng* rng = modlin_prng_new(kind, seed, &err);
  if (!rng) {  // src/main.rs:29-35
    std::fprintf(stderr, "Error initializing the generator: the zero seed is not allowed for MIXMAX\n");
    return 1;
  }
  Progress pr{log_ms, std::chrono::steady_clock::now(), std::chrono::steady_clock::now(), "column"};

  if (have_r) {  // src/main.rs:66-127
    const size_t n = side;
    std::printf("Running a modular rank test using %s of RAM: %" PRIu64 " %zu×%zu %s over the field of size %" PRIu64 "\n",
                format_memory((double)n * n * 8).c_str(), reps, n, n, reps == 1 ? "matrix" : "matrices", modulus);
    std::fflush(stdout);
    // Each matrix is the next n*n outputs reduced mod p (src/main.rs:94-104),
    // generated in device memory and ranked there; several reps go into
    // batched launches (the printed results are the same as one at a time).
    if (reps == 1) {
      const auto t0 = std::chrono::steady_clock::now();
      size_t r = 0;
      const int rc = modlin_rank_prng(modulus, rng, n, &ropts, &r, progress_cb, &pr);
      if (rc) {
        std::fprintf(stderr, "rank failed: %s\n", modlin_strerror(rc));
        return 1;
      }
      const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      std::fprintf(stderr, "Matrix 1/1: generated and ranked in %.3f ms\n", ms);
      const size_t corank = n - r;
      std::printf("Matrix 1/1\tcorank=%zu\tp=%s\n", corank,
                  pretty(modlin_corank_tail_pvalue(modulus, n, corank)).c_str());
    } else {
      std::vector<size_t> ranks(reps);
      const auto t0 = std::chrono::steady_clock::now();
      const int rc = modlin_rank_prng_batch(modulus, rng, n, reps, &ropts, ranks.data(), nullptr, nullptr);
      if (rc) {
        std::fprintf(stderr, "rank failed: %s\n", modlin_strerror(rc));
        return 1;
      }
      const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      std::fprintf(stderr, "%" PRIu64 " matrices generated and ranked in %.3f ms\n", reps, ms);
      for (uint64_t i = 0; i < reps; ++i) {
        const size_t corank = n - ranks[i];
        std::printf("Matrix %" PRIu64 "/%" PRIu64 "\tcorank=%zu\tp=%s\n", i + 1, reps, corank,
                    pretty(modlin_corank_tail_pvalue(modulus, n, corank)).c_str());
      }
    }
    std::fflush(stdout);
  } else {  // src/main.rs:135-176
    const size_t n = length;
    std::printf("Running a modular linear-complexity test using %s of RAM: %" PRIu64 " %s of length %zu over the field of size %" PRIu64 "\n",
                format_memory(4.0 * n * 8).c_str(), reps, reps == 1 ? "sequence" : "sequences", n, modulus);
    std::fflush(stdout);
    // All reps are generated first and ranked in one batched launch; the
    // printed results are the same as one-at-a-time.
    std::vector<uint64_t> seqs(n * reps);
    modlin_prng_fill(rng, seqs.data(), seqs.size());
    for (auto& x : seqs) x = modlin_field_reduce(&field, x);
    std::vector<size_t> lcs(reps);
    const auto t0 = std::chrono::steady_clock::now();
    int rc;
    if (reps == 1) {
      rc = modlin_linear_complexity(modulus, seqs.data(), n, &lcs[0], nullptr, nullptr);
    } else {
      std::vector<modlin_job> jobs(reps);
      for (uint64_t t = 0; t < reps; ++t) jobs[t] = modlin_job{modulus, seqs.data() + t * n, n};
      rc = modlin_lc_batch(jobs.data(), reps, lcs.data());
    }
    if (rc) {
      std::fprintf(stderr, "linear complexity failed: %s\n", modlin_strerror(rc));
      return 1;
    }
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::fprintf(stderr, "Berlekamp-Massey over %" PRIu64 " sequence(s): %.3f ms\n", reps, ms);
    for (uint64_t t = 0; t < reps; ++t)
      std::printf("Sequence %" PRIu64 "/%" PRIu64 "\tlinear complexity=%zu\tp=%s\n", t + 1, reps, lcs[t],
                  pretty(modlin_lc_left_tail_pvalue(modulus, n, lcs[t])).c_str());
  }
  modlin_prng_free(rng);
  return 0;
}
