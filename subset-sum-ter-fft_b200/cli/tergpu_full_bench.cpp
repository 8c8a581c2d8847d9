// tergpu_full_bench: the command line of the reference's ter_full_bench
// (bench/ter_full_bench.cpp) over the device attempt path (tergpu_attempt_run in
// include/tergpu.h).
//
// Same options, modes and exit behaviour for the FiniteSanity / FullTer /
// Random-target configuration the device path implements:
//   --mode=attempt-cost|time-to-found  warmup solves, then `repeat` timed solves
//                                      that must reproduce the first exactly
//   --mode=success-curve               independent seeds (golden-ratio stride),
//                                      attempts- and time-to-found distribution
//   --preflight                        derived geometry and the predicted device
//                                      bytes, no device work
// A solve is one call of attempt_limit attempts on the reference's benchmark
// instance (the planted support fixed to the first n/4 coordinates of each
// half, bench/ter_full_bench.cpp:218-245).  --audit checks every stage whose
// scalar oracle fits against it (TERGPU_ATTEMPT_AUDIT); --guided takes every
// attempt's targets from the planted root (TERGPU_ATTEMPT_GUIDED); --fixture and
// --fixture-limit=<n> keep the first n level-3 subsets of each half
// (TERGPU_ATTEMPT_FIXTURE).  --family=paper-rounded selects a reference path the
// device does not implement; it is refused with a message and exit status 2.
#include "tergpu.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <limits>
#include <string>
#include <string_view>
#include <thread>
#include <vector>

namespace {

constexpr uint64_t kMiB = 1024ull * 1024ull;

enum class Mode { AttemptCost, TimeToFound, SuccessCurve };

const char* mode_name(Mode m) {
  switch (m) {
    case Mode::AttemptCost: return "attempt-cost";
    case Mode::TimeToFound: return "time-to-found";
    case Mode::SuccessCurve: return "success-curve";
  }
  return "unknown";
}

const char* status_name(int s) {
  switch (s) {
    case TERGPU_COMPLETED: return "Completed";
    case TERGPU_FOUND: return "Found";
    case TERGPU_NO_WITNESS_THIS_ATTEMPT: return "NoWitnessThisAttempt";
    case TERGPU_ATTEMPT_LIMIT_REACHED: return "AttemptLimitReached";
    case TERGPU_INVALID_CONFIGURATION: return "InvalidConfiguration";
    case TERGPU_INVALID_SHAPE: return "InvalidShape";
    case TERGPU_GENERATION_INCOMPLETE: return "GenerationIncomplete";
    case TERGPU_RESOURCE_LIMIT: return "ResourceLimit";
    case TERGPU_CANCELLED: return "Cancelled";
    case TERGPU_INVARIANT_VIOLATION: return "InvariantViolation";
    case TERGPU_NOT_APPLICABLE: return "NotApplicable";
    case TERGPU_UNSUPPORTED_WIDTH: return "UnsupportedWidth";
    case TERGPU_OUTPUT_OVERFLOW: return "OutputOverflow";
    case TERGPU_DEVICE_ERROR: return "DeviceError";
    case TERGPU_INVALID_INPUT: return "InvalidInput";
  }
  return "UnknownStatus";
}

struct Options {
  uint32_t n = 36;
  Mode mode = Mode::AttemptCost;
  bool preflight = false;
  bool require_found = false;
  bool audit = false;
  bool guided = false;
  bool fixture = false;
  uint64_t fixture_limit = 64;  // the reference's kDefaultFixtureLevel3Limit
  bool unsupported = false;
  std::string unsupported_what;
  uint32_t attempt_limit = 1;
  uint64_t seed = 19797034556212562ull;  // the reference's fixture seed
  uint32_t warmup = 1;
  uint32_t repeat = 5;
  uint64_t time_limit_ms = 0;
  uint64_t memory_limit_bytes = 4096ull * kMiB;
  uint32_t seeds = 32;
  int device = 0;
};

bool parse_unsigned(std::string_view text, uint64_t* out) {
  if (text.empty()) return false;
  uint64_t v = 0;
  for (const char c : text) {
    if (c < '0' || c > '9') return false;
    const uint64_t d = static_cast<uint64_t>(c - '0');
    if (v > (std::numeric_limits<uint64_t>::max() - d) / 10) return false;
    v = v * 10 + d;
  }
  *out = v;
  return true;
}

void print_usage() {
  std::cerr << "usage: tergpu_full_bench [options]\n"
               "  --n=<finite TER dimension>        default 36 (the device runs 36, 72, 108)\n"
               "  --family=finite-sanity\n"
               "  --mode=attempt-cost|time-to-found|success-curve\n"
               "  --attempt-limit=<count>           default 1 (one attempt only)\n"
               "  --require-found                   exit nonzero unless status is Found\n"
               "  --warmup=<count>                  default 1\n"
               "  --repeat=<count>                  default 5 timed replays; >=1\n"
               "  --time-limit-ms=<ms>              cooperative wall-clock cancel; 0 = none\n"
               "  --memory-limit-mib=<mib>          default 4096 (device bytes)\n"
               "  --memory-limit-bytes=<bytes>      exact cap, for fail-closed testing\n"
               "  --seed=<uint64>                   base seed\n"
               "  --seeds=<count>                   success-curve trials, default 32\n"
               "  --device=<ordinal>                CUDA device, default 0\n"
               "  --preflight                       print derived geometry and exit\n";
}

// Returns 0 on success, 1 on a malformed option.
int parse_options(int argc, char** argv, Options* o) {
  bool repeat_set = false;
  for (int i = 1; i < argc; ++i) {
    const std::string_view v(argv[i]);
    uint64_t x = 0;
    auto value_of = [&](std::string_view prefix, uint64_t* dst) {
      return v.substr(0, prefix.size()) == prefix && parse_unsigned(v.substr(prefix.size()), dst);
    };
    auto has_prefix = [&](std::string_view prefix) { return v.substr(0, prefix.size()) == prefix; };
    if (v == "--preflight") { o->preflight = true; continue; }
    if (v == "--require-found") { o->require_found = true; continue; }
    if (v == "--audit") { o->audit = true; continue; }
    if (v == "--guided") { o->guided = true; continue; }
    if (v == "--fixture") { o->fixture = true; continue; }
    if (has_prefix("--fixture-limit=")) {
      if (!value_of("--fixture-limit=", &x) || x == 0) {
        std::cerr << "invalid --fixture-limit value\n";
        return 1;
      }
      o->fixture_limit = x;
      continue;
    }
    if (has_prefix("--family=")) {
      const auto t = v.substr(9);
      if (t == "finite-sanity") continue;
      if (t == "paper-rounded") {
        o->unsupported = true;
        o->unsupported_what = "--family=paper-rounded";
        continue;
      }
      std::cerr << "invalid --family value\n";
      return 1;
    }
    if (has_prefix("--mode=")) {
      const auto t = v.substr(7);
      if (t == "attempt-cost") o->mode = Mode::AttemptCost;
      else if (t == "time-to-found") o->mode = Mode::TimeToFound;
      else if (t == "success-curve") o->mode = Mode::SuccessCurve;
      else { std::cerr << "invalid --mode value\n"; return 1; }
      continue;
    }
    if (has_prefix("--n=")) {
      if (!value_of("--n=", &x) || x == 0 || x > std::numeric_limits<uint32_t>::max()) {
        std::cerr << "invalid --n value\n";
        return 1;
      }
      o->n = static_cast<uint32_t>(x);
      continue;
    }
    if (has_prefix("--attempt-limit=")) {
      if (!value_of("--attempt-limit=", &x) || x == 0 || x > std::numeric_limits<uint32_t>::max()) {
        std::cerr << "invalid --attempt-limit value\n";
        return 1;
      }
      o->attempt_limit = static_cast<uint32_t>(x);
      continue;
    }
    if (has_prefix("--warmup=")) {
      if (!value_of("--warmup=", &x) || x > std::numeric_limits<uint32_t>::max()) {
        std::cerr << "invalid --warmup value\n";
        return 1;
      }
      o->warmup = static_cast<uint32_t>(x);
      continue;
    }
    if (has_prefix("--repeat=")) {
      if (!value_of("--repeat=", &x) || x == 0 || x > std::numeric_limits<uint32_t>::max()) {
        std::cerr << "invalid --repeat value\n";
        return 1;
      }
      o->repeat = static_cast<uint32_t>(x);
      repeat_set = true;
      continue;
    }
    if (has_prefix("--time-limit-ms=")) {
      if (!value_of("--time-limit-ms=", &o->time_limit_ms)) {
        std::cerr << "invalid --time-limit-ms value\n";
        return 1;
      }
      continue;
    }
    if (has_prefix("--memory-limit-bytes=")) {
      if (!value_of("--memory-limit-bytes=", &x) || x == 0) {
        std::cerr << "invalid --memory-limit-bytes value\n";
        return 1;
      }
      o->memory_limit_bytes = x;
      continue;
    }
    if (has_prefix("--memory-limit-mib=")) {
      if (!value_of("--memory-limit-mib=", &x) || x == 0 ||
          x > std::numeric_limits<uint64_t>::max() / kMiB) {
        std::cerr << "invalid --memory-limit-mib value\n";
        return 1;
      }
      o->memory_limit_bytes = x * kMiB;
      continue;
    }
    if (has_prefix("--seed=")) {
      if (!value_of("--seed=", &o->seed)) {
        std::cerr << "invalid --seed value\n";
        return 1;
      }
      continue;
    }
    if (has_prefix("--seeds=")) {
      if (!value_of("--seeds=", &x) || x == 0 || x > std::numeric_limits<uint32_t>::max()) {
        std::cerr << "invalid --seeds value\n";
        return 1;
      }
      o->seeds = static_cast<uint32_t>(x);
      continue;
    }
    if (has_prefix("--device=")) {
      if (!value_of("--device=", &x) || x > 1024) {
        std::cerr << "invalid --device value\n";
        return 1;
      }
      o->device = static_cast<int>(x);
      continue;
    }
    print_usage();
    return 1;
  }
  if (o->mode == Mode::SuccessCurve && repeat_set) {
    std::cerr << "--repeat does not apply to --mode=success-curve; use --seeds\n";
    return 1;
  }
  return 0;
}

// The reference's benchmark instance: SplitMix64(seed) weights, one draw per
// 64-bit word, the top word masked to n bits (src/instance.cpp:61-120); the
// planted support is the first n/4 coordinates of each half and the target
// their sum mod 2^n.
struct Instance {
  uint32_t n = 0;
  std::vector<uint64_t> values;  // n * ceil(n/64) words
  std::vector<uint64_t> target;  // ceil(n/64) words
  std::vector<uint8_t> planted;  // n digits: the planted root
};

Instance benchmark_instance(uint32_t n, uint64_t seed) {
  Instance inst;
  if (n == 0 || n % 2 != 0 || n > 128) return inst;
  const uint32_t w = (n + 63) / 64;
  uint64_t state = seed;
  auto next = [&state]() {
    uint64_t z = (state += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  };
  const uint64_t top_mask = n % 64 == 0 ? ~0ull : ((1ull << (n % 64)) - 1ull);
  inst.n = n;
  inst.values.assign(static_cast<size_t>(n) * w, 0);
  for (uint32_t i = 0; i < n; ++i) {
    for (uint32_t k = 0; k < w; ++k) inst.values[i * w + k] = next();
    inst.values[i * w + w - 1] &= top_mask;
  }
  inst.target.assign(w, 0);
  inst.planted.assign(n, 0);
  for (uint32_t half = 0; half < 2; ++half) {
    for (uint32_t off = 0; off < n / 4; ++off) {
      const uint32_t i = half * (n / 2) + off;
      inst.planted[i] = 1;
      uint64_t carry = 0;
      for (uint32_t k = 0; k < w; ++k) {
        const uint64_t a = inst.target[k], b = inst.values[i * w + k];
        const uint64_t s1 = a + b;
        const uint64_t c1 = s1 < a ? 1 : 0;
        const uint64_t s2 = s1 + carry;
        const uint64_t c2 = s2 < s1 ? 1 : 0;
        inst.target[k] = s2;
        carry = c1 | c2;
      }
    }
  }
  inst.target[w - 1] &= top_mask;
  return inst;
}

// Cooperative wall-clock cancel: sets the flag the device path polls between
// stages, so a timeout surfaces as Cancelled.
class TimeGuard {
 public:
  TimeGuard(uint64_t limit_ms, volatile int32_t* flag) : flag_(flag) {
    if (limit_ms == 0) return;
    armed_ = true;
    worker_ = std::thread([this, limit_ms] {
      const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(limit_ms);
      while (!stop_.load()) {
        if (std::chrono::steady_clock::now() >= deadline) {
          *flag_ = 1;
          return;
        }
        std::this_thread::sleep_for(std::chrono::milliseconds(2));
      }
    });
  }
  ~TimeGuard() {
    stop_.store(true);
    if (armed_ && worker_.joinable()) worker_.join();
  }
  TimeGuard(const TimeGuard&) = delete;
  TimeGuard& operator=(const TimeGuard&) = delete;

 private:
  volatile int32_t* flag_;
  std::atomic<bool> stop_{false};
  std::thread worker_;
  bool armed_ = false;
};

struct Solve {
  int status = TERGPU_DEVICE_ERROR;
  tergpu_attempt_out out{};
  std::vector<tergpu_attempt_stats> stats;
  std::string message;
};

Solve solve(const Options& o, const Instance& inst, uint64_t seed, uint64_t time_limit_ms,
            bool telemetry) {
  Solve s;
  s.stats.assign(o.attempt_limit, tergpu_attempt_stats{});
  volatile int32_t cancel = 0;
  tergpu_attempt_in in{};
  in.n = inst.n;
  in.values_le = inst.values.data();
  in.target_le = inst.target.data();
  in.seed = seed;
  in.attempt_first = 0;
  in.attempt_count = o.attempt_limit;
  in.memory_limit_bytes = o.memory_limit_bytes;
  in.cancel = &cancel;
  in.device = o.device;
  in.flags = (telemetry ? TERGPU_ATTEMPT_TELEMETRY : 0u) | (o.audit ? TERGPU_ATTEMPT_AUDIT : 0u) |
             (o.guided ? TERGPU_ATTEMPT_GUIDED : 0u) | (o.fixture ? TERGPU_ATTEMPT_FIXTURE : 0u);
  in.planted_root = o.guided ? inst.planted.data() : nullptr;
  in.fixture_level3_limit = o.fixture ? o.fixture_limit : 0;
  // the reference's bench keeps FirstWitness (include/ter/full_ter.hpp:105)
  in.root_policy = TERGPU_ROOT_POLICY_FIRST_WITNESS;
  s.out.stats = s.stats.data();
  {
    const TimeGuard guard(time_limit_ms, &cancel);
    s.status = tergpu_attempt_run(&in, &s.out);
  }
  s.message = tergpu_last_error();
  s.stats.resize(s.out.attempts_run);
  return s;
}

bool comparable(int status) {
  return status == TERGPU_FOUND || status == TERGPU_ATTEMPT_LIMIT_REACHED;
}

uint64_t median(std::vector<uint64_t> v) {
  if (v.empty()) return 0;
  std::sort(v.begin(), v.end());
  return v[v.size() / 2];
}

uint64_t percentile95(std::vector<uint64_t> v) {
  if (v.empty()) return 0;
  std::sort(v.begin(), v.end());
  return v[std::min<size_t>(v.size() - 1, static_cast<size_t>(0.95 * static_cast<double>(v.size())))];
}

uint64_t ns(double ms) { return static_cast<uint64_t>(ms * 1e6); }

void print_metadata(const Options& o, const std::string& command, uint64_t executed) {
  std::cout << "# backend=tergpu abi=" << tergpu_abi_version() << " device=" << o.device
            << " mode=" << mode_name(o.mode) << " attempt_limit=" << o.attempt_limit
            << " attempts_executed=" << executed << " warmup=" << o.warmup
            << " repeat=" << o.repeat << " time_limit_ms=" << o.time_limit_ms
            << " memory_limit_bytes=" << o.memory_limit_bytes << " seed=" << o.seed
            << " execution_mode=" << (o.fixture ? "FixtureTer" : "FullTer")
            << " target=" << (o.guided ? "GuidedPlanted" : "Random")
            << " audit=" << (o.audit ? "on" : "off")
            << " family=FiniteSanity"
            << " command=\"" << command << "\"\n";
}

// The FiniteSanity representation count m! / (k! k! (m - 2k)!) as C(m, k) *
// C(m - k, k), exact in 128 bits for n <= 108 (R1 < 2^80): the reference's
// FullTerParameters::representation1 (m = n/2, k = n/6) and representation2
// (m = n/6, k = n/18), printed by its preflight (bench/ter_full_bench.cpp:624-627).
unsigned __int128 representation_count(uint32_t m, uint32_t k) {
  unsigned __int128 a = 1, b = 1;
  for (uint32_t i = 1; i <= k; ++i) a = a * (m - k + i) / i;      // C(m, k), exact at every step
  for (uint32_t i = 1; i <= k; ++i) b = b * (m - 2 * k + i) / i;  // C(m - k, k)
  return a * b;
}

std::string decimal(unsigned __int128 v) {
  std::string digits;
  do {
    digits.insert(digits.begin(), static_cast<char>('0' + static_cast<int>(v % 10)));
    v /= 10;
  } while (v != 0);
  return digits;
}

uint32_t floor_log2(unsigned __int128 v) {
  uint32_t bits = 0;
  while (v >>= 1) ++bits;
  return bits;
}

int run_preflight(const Options& o) {
  tergpu_attempt_in in{};
  in.n = o.n;
  in.flags = TERGPU_ATTEMPT_PREFLIGHT | (o.fixture ? TERGPU_ATTEMPT_FIXTURE : 0u);
  in.fixture_level3_limit = o.fixture ? o.fixture_limit : 0;
  in.memory_limit_bytes = o.memory_limit_bytes;
  in.device = o.device;
  tergpu_attempt_out out{};
  const int st = tergpu_attempt_run(&in, &out);
  std::cout << "preflight n=" << o.n << " family=FiniteSanity\n";
  if (st == TERGPU_INVALID_CONFIGURATION) {
    std::cout << "  shape_status=InvalidConfiguration\n";
    std::cout << "  message=" << tergpu_last_error() << '\n';
    // the reference's verdict where no path can construct the shape (36 does not divide n)
    std::cout << "  VERDICT: dimension is not a constructible exact TER shape"
              << (o.n != 0 && o.n % 36 == 0 ? " on the device path" : "") << '\n';
    return EXIT_FAILURE;
  }
  std::cout << "  shape_status=Completed\n";
  const uint32_t root_q = o.n - out.r1, middle_q = out.r1 - out.r2;
  std::cout << "  r1=" << out.r1 << " r2=" << out.r2 << " root_Q=" << root_q
            << " l2_to_l1_Q=" << middle_q << '\n';
  const unsigned __int128 rep1 = representation_count(o.n / 2, o.n / 6);
  const unsigned __int128 rep2 = representation_count(o.n / 6, o.n / 18);
  std::cout << "  representation1=" << decimal(rep1) << " floor_log2=" << floor_log2(rep1) << '\n';
  std::cout << "  representation2=" << decimal(rep2) << " floor_log2=" << floor_log2(rep2) << '\n';
  std::cout << "  level3_per_half=" << out.level3_size << '\n';
  std::cout << "  l2_to_l1_backend=device ternary join on the projected quotient (streaming, "
               "no pair index)\n";
  std::cout << "  l2_to_l1_decision="
            << (middle_q <= 32 ? "quotient projection is decisive (r1-r2 <= 32)"
                               : "unsupported (r1-r2 > 32)")
            << '\n';
  std::cout << "  root_backend=device root join (radix partition + on-chip sweep, no pair index)\n";
  std::cout << "  root_decision="
            << (root_q <= 64 ? "quotient congruence is decisive (Q <= 64)"
                             : "full-Q key join + residue-word authority on the device (Q > 64)")
            << '\n';
  std::cout << "  predicted_device_bytes=" << out.device_bytes << '\n';
  std::cout << "  memory_limit_bytes=" << o.memory_limit_bytes << '\n';
  std::cout << "  execution_mode=" << (o.fixture ? "FixtureTer" : "FullTer") << '\n';
  std::cout << "  pair_materializing_fallback=no\n";
  if (st == TERGPU_RESOURCE_LIMIT) {
    std::cout << "  VERDICT: ResourceLimit (predicted device bytes exceed the ceiling)\n";
    return EXIT_FAILURE;
  }
  std::cout << "  VERDICT: bounded exact path on both merge stages\n";
  return st == TERGPU_COMPLETED ? EXIT_SUCCESS : EXIT_FAILURE;
}

int run_success_curve(const Options& o) {
  std::vector<uint64_t> attempts_to_found, time_to_found_ns, found_seeds;
  uint64_t found = 0, exhausted = 0, censored = 0;
  for (uint32_t trial = 0; trial < o.seeds; ++trial) {
    const uint64_t seed = o.seed + trial * 0x9E3779B97F4A7C15ull;
    const Instance inst = benchmark_instance(o.n, seed);
    if (inst.n == 0) {
      std::cerr << "failed to build benchmark instance for seed " << seed << '\n';
      return EXIT_FAILURE;
    }
    const Solve s = solve(o, inst, seed, o.time_limit_ms, false);
    if (s.status == TERGPU_FOUND) {
      ++found;
      attempts_to_found.push_back(static_cast<uint64_t>(s.out.found_attempt) + 1);
      time_to_found_ns.push_back(ns(s.out.total_ms));
      found_seeds.push_back(seed);
    } else if (s.status == TERGPU_ATTEMPT_LIMIT_REACHED) {
      ++exhausted;
    } else {
      ++censored;
      std::cerr << "trial seed=" << seed << " status=" << status_name(s.status)
                << " message=" << s.message << '\n';
    }
  }
  const double fraction = static_cast<double>(found) / static_cast<double>(o.seeds);
  std::cout << "independent_runs,found,attempt_limit_reached,censored,success_fraction,"
               "median_attempts_to_found,p95_attempts_to_found,"
               "median_time_to_found_ns,p95_time_to_found_ns\n";
  std::cout << o.seeds << ',' << found << ',' << exhausted << ',' << censored << ',' << fraction
            << ',' << median(attempts_to_found) << ',' << percentile95(attempts_to_found) << ','
            << median(time_to_found_ns) << ',' << percentile95(time_to_found_ns) << '\n';
  std::cout << "run_index,run_seed,attempts_to_found,time_to_found_ns\n";
  for (size_t i = 0; i < attempts_to_found.size(); ++i) {
    std::cout << i << ',' << found_seeds[i] << ',' << attempts_to_found[i] << ','
              << time_to_found_ns[i] << '\n';
  }
  std::cout << "attempt_budget,found_by_budget,cumulative_success_fraction\n";
  for (uint64_t budget = 1; budget <= o.attempt_limit; budget *= 2) {
    uint64_t reached = 0;
    for (const uint64_t a : attempts_to_found) reached += a <= budget ? 1 : 0;
    std::cout << budget << ',' << reached << ','
              << static_cast<double>(reached) / static_cast<double>(o.seeds) << '\n';
  }
  if (o.require_found && found == 0) {
    std::cerr << "no trial reached Found and --require-found was requested\n";
    return EXIT_FAILURE;
  }
  return censored == 0 ? EXIT_SUCCESS : EXIT_FAILURE;
}

std::string join_sizes(const uint64_t* v, int count) {
  std::string s;
  for (int i = 0; i < count; ++i) {
    if (i) s += ':';
    s += std::to_string(v[i]);
  }
  return s;
}

int run_timed(const Options& o, const std::string& command) {
  const Instance inst = benchmark_instance(o.n, o.seed);
  if (inst.n == 0) {
    std::cerr << "failed to build benchmark instance\n";
    return EXIT_FAILURE;
  }
  for (uint32_t i = 0; i < o.warmup; ++i) {
    const Solve s = solve(o, inst, o.seed, o.time_limit_ms, true);
    if (!comparable(s.status)) {
      std::cerr << "full TER warmup did not reach a comparable terminal status: "
                << status_name(s.status) << ": " << s.message << '\n';
      return EXIT_FAILURE;
    }
  }
  Solve first;
  std::vector<uint64_t> totals, l3, binary, middle, root, verification;
  for (uint32_t rep = 0; rep < o.repeat; ++rep) {
    Solve s = solve(o, inst, o.seed, o.time_limit_ms, true);
    if (!comparable(s.status)) {
      std::cerr << "full TER run did not reach a comparable terminal status: "
                << status_name(s.status) << ": " << s.message << '\n';
      return EXIT_FAILURE;
    }
    if (s.stats.empty()) {
      std::cerr << "measured run produced no attempt telemetry; status=" << status_name(s.status)
                << '\n';
      return EXIT_FAILURE;
    }
    const tergpu_attempt_stats& t = s.stats.back();
    totals.push_back(ns(s.out.total_ms));
    l3.push_back(ns(s.out.level3_ms));
    binary.push_back(ns(t.l2_ms));
    middle.push_back(ns(t.l1_ms));
    root.push_back(ns(t.root_ms));
    verification.push_back(ns(t.verification_ms));
    if (rep == 0) {
      first = std::move(s);
    } else if (s.status != first.status ||
               std::memcmp(s.out.witness, first.out.witness, sizeof s.out.witness) != 0 ||
               s.out.fingerprint != first.out.fingerprint) {
      // the reference's repeat check: status, witness and telemetry fingerprint
      // (bench/ter_full_bench.cpp:833-839)
      std::cerr << "full TER benchmark changed its exact result\n";
      return EXIT_FAILURE;
    }
  }
  const size_t executed = first.stats.size();
  if (executed < 1 || executed > o.attempt_limit) {
    std::cerr << "attempt-budget invariant violated: executed=" << executed
              << " attempt_limit=" << o.attempt_limit << '\n';
    return EXIT_FAILURE;
  }
  if (first.status == TERGPU_ATTEMPT_LIMIT_REACHED && executed != o.attempt_limit) {
    std::cerr << "AttemptLimitReached must consume the whole budget: executed=" << executed
              << " attempt_limit=" << o.attempt_limit << '\n';
    return EXIT_FAILURE;
  }
  const tergpu_attempt_stats& t = first.stats.back();
  if (first.status == TERGPU_FOUND && t.status != TERGPU_FOUND) {
    std::cerr << "Found result did not select a Found attempt\n";
    return EXIT_FAILURE;
  }
  std::vector<uint64_t> per_attempt;
  uint64_t sum_ns = 0, root_pairs = 0;
  for (const auto& a : first.stats) {
    per_attempt.push_back(ns(a.total_ms));
    sum_ns += ns(a.total_ms);
    root_pairs += a.root_pairs;
  }
  uint64_t l2_total = 0, l1_total = 0;
  for (int i = 0; i < 9; ++i) l2_total += t.level2_sizes[i];
  for (int i = 0; i < 3; ++i) l1_total += t.level1_sizes[i];
  print_metadata(o, command, executed);
  // The reference's column set (bench/ter_full_bench.cpp:874-895).  Columns the
  // device path has no counterpart for are printed empty: the CPU memory model
  // (l3_list_bytes .. packed_vector_bytes except peak_working_bytes, which holds
  // the device workspace's peak), the tiled reporter's internals (tile bits,
  // probes, windows, auxiliary bytes, setup and scan times) and the root's
  // output-byte accounting.  The device runs no tiled reporter (tiled_used 0)
  // and materializes no pair records.
  std::cout << "status,n,r1,r2,L3_left,L3_right,L2_sizes,L1_sizes,L0,"
               "l3_generation_ns,l3_to_l2_ns,l2_to_l1_ns,l1_to_l0_ns,"
               "verification_ns,total_solver_ns,"
               "binary_pairs,binary_modular,binary_structural_rejects,"
               "binary_distribution_rejects,binary_survivors,binary_deduplicated,"
               "middle_pairs,middle_modular,middle_structural_rejects,"
               "middle_distribution_rejects,middle_survivors,middle_deduplicated,"
               "root_pairs,root_modular,root_structural_rejects,"
               "root_distribution_rejects,root_survivors,root_deduplicated,"
               "l3_list_bytes,arithmetic_bytes,l2_list_bytes,l1_list_bytes,l0_list_bytes,"
               "l2_active_bytes,l1_active_bytes,root_active_bytes,"
               "peak_working_bytes,hot_entry_bytes,packed_vector_bytes,fingerprint,"
               "l2_to_l1_tiled_used,l2_to_l1_pair_records,l2_to_l1_tile_bits,"
               "l2_to_l1_tiled_pair_probes,l2_to_l1_tiled_nonempty_windows,"
               "l2_to_l1_tiled_auxiliary_bytes,l2_to_l1_tiled_setup_ns,"
               "l2_to_l1_tiled_scan_ns,"
               "l1_to_l0_tiled_used,l1_to_l0_pair_records,l1_to_l0_quotient_bits,"
               "l1_to_l0_prefilter_bits,l1_to_l0_low_prefilter_candidates,"
               "l1_to_l0_full_quotient_rejects,l1_to_l0_tile_bits,"
               "l1_to_l0_tiled_pair_probes,l1_to_l0_tiled_nonempty_windows,"
               "l1_to_l0_tiled_auxiliary_bytes,l1_to_l0_tiled_setup_ns,"
               "l1_to_l0_tiled_scan_ns,"
               "l1_to_l0_root_policy,l1_to_l0_valid_roots,"
               "l1_to_l0_early_stopped,l1_to_l0_output_peak_bytes,"
               "l1_to_l0_output_live_bytes,l1_to_l0_working_peak_bytes,"
               "l1_to_l0_first_witness_ceiling_bytes,"
               "attempts_used,terminal_attempt_index,terminal_attempt_seed,"
               "terminal_attempt_status,sum_attempt_ns,mean_attempt_ns,"
               "median_attempt_ns,total_root_pair_candidates\n";
  const char* empty = "";
  std::cout << status_name(first.status) << ',' << o.n << ',' << first.out.r1 << ','
            << first.out.r2 << ',' << first.out.level3_size << ',' << first.out.level3_size
            << ",\"" << join_sizes(t.level2_sizes, 9) << "\",\"" << join_sizes(t.level1_sizes, 3)
            << "\"," << t.level0_size << ',' << median(l3) << ',' << median(binary) << ','
            << median(middle) << ',' << median(root) << ',' << median(verification) << ','
            << median(totals) << ','
            << t.l3_pairs << ',' << t.l3_modular << ',' << t.l3_structural_rejects << ','
            << t.l3_distribution_rejects << ',' << t.l3_survivors << ',' << l2_total << ','
            << t.l2_pairs << ',' << t.l2_modular << ',' << t.l2_structural_rejects << ','
            << t.l2_distribution_rejects << ',' << t.l2_survivors << ',' << l1_total << ','
            << t.root_pairs << ',' << t.root_modular << ',' << t.root_structural_rejects << ','
            << t.root_distribution_rejects << ',' << t.valid_roots << ',' << t.level0_size << ',';
  for (int i = 0; i < 8; ++i) std::cout << empty << ',';       // l3_list_bytes .. root_active_bytes
  std::cout << first.out.device_bytes_held << ',' << empty << ',' << empty << ','
            << first.out.fingerprint << ','
            << 0 << ',' << 0 << ',';                               // tiled_used, pair_records
  for (int i = 0; i < 6; ++i) std::cout << empty << ',';       // l2_to_l1 tiled internals
  std::cout << 0 << ',' << 0 << ',' << t.root_quotient_bits << ',' << t.root_prefilter_bits << ','
            << t.root_low_prefilter << ',' << t.root_full_quotient_rejects << ',';
  for (int i = 0; i < 6; ++i) std::cout << empty << ',';       // l1_to_l0 tiled internals
  std::cout << t.root_policy << ',' << t.valid_roots << ',' << t.root_early_stopped << ',';
  for (int i = 0; i < 4; ++i) std::cout << empty << ',';       // root output bytes
  std::cout << executed << ',' << t.attempt << ',' << t.attempt_seed << ',' << status_name(t.status)
            << ',' << sum_ns << ',' << sum_ns / executed << ',' << median(per_attempt) << ','
            << root_pairs << '\n';
  if (o.require_found && first.status != TERGPU_FOUND) {
    std::cerr << "--require-found: terminal status was " << status_name(first.status)
              << ", not Found\n";
    return EXIT_FAILURE;
  }
  return EXIT_SUCCESS;
}

}  // namespace

int main(int argc, char** argv) {
  Options o;
  if (parse_options(argc, argv, &o) != 0) return EXIT_FAILURE;
  if (o.unsupported) {
    std::cerr << o.unsupported_what
              << " selects a reference path the device attempt does not implement "
                 "(it runs FiniteSanity / FullTer / Random targets)\n";
    return 2;
  }
  std::string command;
  for (int i = 0; i < argc; ++i) {
    if (i) command += ' ';
    command += argv[i];
  }
  if (o.preflight) return run_preflight(o);
  if (o.mode == Mode::SuccessCurve) {
    print_metadata(o, command, 0);
    return run_success_curve(o);
  }
  return run_timed(o, command);
}
