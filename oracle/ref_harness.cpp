// Reference harness -- test infrastructure, never part of the product.
//
// Drives the reference's own compiled code (built from its sources by
// oracle/Makefile) so tests can pin the oracle restatement and the GPU backend
// against it, and so bench.py can time the reference's CPU backends on the same
// host.  Every line of output is one JSON object.
//
//   terref solve N SEED ATTEMPTS KIND POLICY AUDIT [CONFIG_SEED [MODES]]
//       solve_full_ter (src/full_ter.cpp:3867) on authentic_instance (KIND=auth)
//       or build_instance(n, 10, seed) (KIND=build); per-attempt level sizes,
//       root accounting and the witness.  CONFIG_SEED (default SEED, "-" keeps
//       it) seeds the targets; MODES "guided", "fixture=<limit>" and
//       "cancelled" (comma-separated) select GuidedPlanted targets, FixtureTer
//       level 3 and a cancellation flag already set when the solve starts.
//   terref capture N SEED ATTEMPT KIND OUT
//       root_snapshot::capture_to_file (ter2_root/frozen/ter_root_snapshot.cpp:124).
//   terref snaproot SNAP BACKEND CELLS PROJ
//       load_snapshot_workload + build_family_keys + build_root_index, the cell
//       selection CELLS (apply_cells), then one backend into an authority sink.
//   terref snaptime SNAP BACKEND PROJ CELLS REPS FIRST STRIDE
//       load_snapshot_workload once (untimed), then REPS timed passes of one
//       backend; pass r runs the cells perm:((FIRST + r * STRIDE) mod 4096):CELLS
//       (successive windows of the reference's shuffled cell order) into a fresh
//       authority sink; one JSON row per pass.
//   terref synth BITS SEED SIZE POOL OUT
//       ter2_root/tests/ter_synthetic_root.hpp make_root; writes the three key
//       lists to OUT and prints the brute-force oracle digest.
//   terref keysroot KEYS BACKEND CELLS REPS PROJ
//       one backend over key lists read from KEYS (list 2 holds d), sink without
//       authority; REPS timed repetitions.
//   terref plant SNAP COUNT SEED
//       the whole-root runner's positive construction
//       (ter2_root/campaign/ter_arwlf_whole_root_main.cpp:240-247): PlantedTargets
//       on the anchor microproblem (select_microproblems(index, 1)); prints the
//       appended D keys and the expected final outputs.
//   terref report SNAP POLICY
//       report_full_ter_root (src/full_ter.cpp:3722) on the capture held by SNAP
//       (POLICY = first | count | canon), plus count_full_ter_root (:3861).
// BACKEND: arwlf | k2wide | k2 | dispatch | hash | gpu | brute

#include "ter_a64_chqr.hpp"
#include "ter_arwlf.hpp"
#include "ter_arwlf_campaign.hpp"
#include "ter_gpu_root.hpp"
#include "ter_hash_join_root.hpp"
#include "ter_root_generalization_workload.hpp"
#include "ter_root_queue_kernels.hpp"
#include "ter_root_snapshot.hpp"
#include "ter_synthetic_root.hpp"

#include "ter/full_ter.hpp"
#include "ter/instance.hpp"
#include "ter/limitations.hpp"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

namespace {

namespace rg = ter::root_generalization;
namespace mr8 = ter::microreport8;
namespace a64 = ter::a64;
namespace aw = ter::arwlf;
namespace rs = ter::root_snapshot;
namespace sr = ter::synthetic_root;
namespace hj = ter::hash_join_root;
namespace gr = ter::gpu_root;

using Clock = std::chrono::steady_clock;

std::string hex64(std::uint64_t v) {
  char buf[32];
  std::snprintf(buf, sizeof buf, "\"0x%016llx\"", static_cast<unsigned long long>(v));
  return buf;
}

ter::Instance make_instance(std::uint32_t n, std::uint64_t seed, const std::string& kind) {
  if (kind == "auth") { return rg::authentic_instance(n, seed); }
  auto built = ter::build_instance(n, ter::limits::benchmark::kFullTerFixtureModulusBits, seed);
  return built.status == ter::Status::Completed ? built.value : ter::Instance{};
}

std::string digest_json(const rg::OutputDigest& d) {
  std::ostringstream o;
  o << "\"triples\":" << d.triples << ",\"triple_sum\":" << hex64(d.triple_sum)
    << ",\"triple_xor\":" << hex64(d.triple_xor) << ",\"triple_sum2\":" << hex64(d.triple_sum2)
    << ",\"full_q\":" << d.full_q << ",\"residue\":" << d.residue
    << ",\"residue_sum\":" << hex64(d.residue_sum) << ",\"structural\":" << d.structural;
  return o.str();
}

std::string witnesses_json(std::vector<std::array<ter::EntryId, 3>> w) {
  std::sort(w.begin(), w.end());
  std::ostringstream o;
  o << "[";
  for (std::size_t i = 0; i < w.size(); ++i) {
    o << (i ? "," : "") << "[" << w[i][0] << "," << w[i][1] << "," << w[i][2] << "]";
  }
  o << "]";
  return o.str();
}

int cmd_solve(int argc, char** argv) {
  if (argc < 8) { return 2; }
  const auto n = static_cast<std::uint32_t>(std::strtoul(argv[2], nullptr, 0));
  const std::uint64_t seed = std::strtoull(argv[3], nullptr, 0);
  const auto attempts = static_cast<std::uint32_t>(std::strtoul(argv[4], nullptr, 0));
  const std::string kind = argv[5];
  const std::string policy = argv[6];
  const bool audit = std::string(argv[7]) == "1";
  const ter::Instance instance = make_instance(n, seed, kind);
  // optional: the config seed when it differs from the instance seed ("-" keeps
  // it), and the modes "guided", "fixture=<limit>" or "guided,fixture=<limit>"
  const std::uint64_t config_seed =
      argc > 8 && std::string(argv[8]) != "-" ? std::strtoull(argv[8], nullptr, 0) : seed;
  ter::FullTerConfig config = rg::authentic_config(config_seed);
  const std::string modes = argc > 9 ? argv[9] : "";
  if (modes.find("guided") != std::string::npos) {
    config.target_mode = ter::TerTargetMode::GuidedPlanted;
  }
  if (const auto at = modes.find("fixture="); at != std::string::npos) {
    config.execution_mode = ter::TerExecutionMode::FixtureTer;
    config.fixture_level3_limit = std::strtoull(modes.c_str() + at + 8, nullptr, 0);
  }
  config.attempt_limit = attempts;
  config.audit = audit;
  config.root_output_policy = policy == "canon" ? ter::RootOutputPolicy::FullCanonicalOutput
                                                : ter::RootOutputPolicy::FirstWitness;
  std::atomic_bool cancelled{true};
  if (modes.find("cancelled") != std::string::npos) { config.cancellation = &cancelled; }
  const auto start = Clock::now();
  const ter::FullTerResult result = ter::solve_full_ter(instance, config);
  const double ms = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
  const auto& t = result.telemetry;
  for (const auto& a : t.attempts) {
    std::cout << "{\"attempt\":" << a.attempt << ",\"seed\":" << a.seed
              << ",\"status\":" << static_cast<int>(a.status) << ",\"level2\":[";
    for (std::size_t i = 0; i < 9; ++i) { std::cout << (i ? "," : "") << a.level2_sizes[i]; }
    std::cout << "],\"level1\":[" << a.level1_sizes[0] << "," << a.level1_sizes[1] << ","
              << a.level1_sizes[2] << "],\"level0\":" << a.level0_size
              << ",\"l3_modular\":" << a.level3_to_level2.modular_candidates
              << ",\"l2_modular\":" << a.level2_to_level1.modular_candidates
              << ",\"root_prefilter\":" << a.level1_to_level0.low_prefilter_candidates
              << ",\"root_quotient_rejects\":" << a.level1_to_level0.full_quotient_rejects
              << ",\"root_modular\":" << a.level1_to_level0.modular_candidates
              << ",\"valid_roots\":" << a.level1_to_level0.valid_root_count
              << ",\"prefilter_bits\":" << a.level1_to_level0.prefilter_bits
              << ",\"root_ns\":" << a.level1_to_level0.elapsed_ns
              << ",\"total_ns\":" << a.total_ns;
    const auto stage = [](const char* name, const ter::FullTerStageTelemetry& s) {
      std::ostringstream o;
      o << ",\"" << name << "\":{\"pairs\":" << s.pair_candidates
        << ",\"modular\":" << s.modular_candidates << ",\"structural\":" << s.structural_rejects
        << ",\"distribution\":" << s.distribution_rejects
        << ",\"survivors\":" << s.survivors_before_dedup
        << ",\"deduplicated\":" << s.survivors_after_dedup
        << ",\"pair_records\":" << s.pair_records << ",\"quotient_bits\":" << s.quotient_bits
        << ",\"prefilter_bits\":" << s.prefilter_bits
        << ",\"low_prefilter\":" << s.low_prefilter_candidates
        << ",\"full_quotient_rejects\":" << s.full_quotient_rejects
        << ",\"valid_roots\":" << s.valid_root_count
        << ",\"policy\":" << static_cast<unsigned>(s.effective_root_output_policy)
        << ",\"early_stopped\":" << (s.early_stopped ? 1 : 0)
        << ",\"fingerprint\":" << hex64(s.output_fingerprint) << "}";
      return o.str();
    };
    std::cout << stage("binary", a.level3_to_level2) << stage("middle", a.level2_to_level1)
              << stage("root", a.level1_to_level0) << "}\n";
  }
  std::cout << "{\"status\":" << static_cast<int>(result.status) << ",\"r1\":" << t.parameters.r1
            << ",\"r2\":" << t.parameters.r2 << ",\"l3\":[" << t.physical_level3_sizes[0] << ","
            << t.physical_level3_sizes[1] << "],\"fingerprint\":" << hex64(t.fingerprint)
            << ",\"ms\":" << ms << ",\"witness\":\"";
  for (const auto d : result.witness) { std::cout << static_cast<int>(d); }
  std::cout << "\",\"message\":\"" << result.message << "\"}\n";
  return 0;
}

int cmd_capture(int argc, char** argv) {
  if (argc < 7) { return 2; }
  const auto n = static_cast<std::uint32_t>(std::strtoul(argv[2], nullptr, 0));
  const std::uint64_t seed = std::strtoull(argv[3], nullptr, 0);
  const auto attempt = static_cast<std::uint32_t>(std::strtoul(argv[4], nullptr, 0));
  const ter::Instance instance = make_instance(n, seed, argv[5]);
  ter::FullTerConfig config = rg::authentic_config(seed);
  config.attempt_limit = attempt + 1U;  // the stream refuses attempts outside the budget
  const auto start = Clock::now();
  const rs::CaptureOutcome outcome = rs::capture_to_file(instance, config, attempt, argv[6],
                                                         std::uint64_t{4} << 20, "reference");
  const double ms = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
  std::cout << "{\"written\":" << (outcome.written ? "true" : "false")
            << ",\"status\":" << static_cast<int>(outcome.stream.status)
            << ",\"level1\":[" << outcome.stream.level1_sizes[0] << ","
            << outcome.stream.level1_sizes[1] << "," << outcome.stream.level1_sizes[2]
            << "],\"level2\":[";
  for (std::size_t i = 0; i < 9; ++i) { std::cout << (i ? "," : "") << outcome.stream.level2_sizes[i]; }
  std::cout << "],\"file_bytes\":" << outcome.file_bytes << ",\"ms\":" << ms << "}\n";
  return outcome.written ? 0 : 1;
}

// One backend pass into `sink`; returns backend telemetry as JSON fields.
std::string run_backend(const std::string& backend, const mr8::Dataset& data, rg::RootIndex& index,
                        const a64::FamilyKeys& keys, rg::RootSink& sink, std::uint32_t proj,
                        double* ms) {
  std::ostringstream o;
  const auto start = Clock::now();
  if (backend == "arwlf") {
    aw::Config config;
    if (proj != 0U) { config.check_bits = proj - 19U; }
    aw::Telemetry t;
    const aw::Status st = aw::run_arwlf(data, index, keys, config, sink, &t);
    *ms = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
    o << "\"backend_status\":\"" << aw::status_label(st) << "\",\"logical_pairs\":" << t.logical_pairs
      << ",\"filter_survivors\":" << t.filter_survivors << ",\"projected_hits\":" << t.projected_hits
      << ",\"projected_bits\":" << 19U + t.check_bits << ",\"fast_hits\":" << t.fast_hits
      << ",\"full_hits\":" << t.full_hits;
  } else if (backend == "k2wide") {
    a64::Telemetry t;
    a64::run_k2_wide(data, index, keys, sink, &t, false);
    *ms = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
    o << "\"backend_status\":\"Completed\",\"logical_pairs\":" << t.logical_pairs
      << ",\"projected_hits\":" << t.projected_hits << ",\"fast_hits\":" << t.fast_hits
      << ",\"full_hits\":" << t.full_hits;
  } else if (backend == "k2") {
    rg::run_k2(data, sink);
    *ms = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
    o << "\"backend_status\":\"Completed\"";
  } else if (backend == "dispatch") {
    // the reference's probe-and-choose dispatcher (QUEUE_DENSE / ARWLF /
    // K2_WIDE), with radix tables kept for the process as its runner keeps them
    static rg::RadixTables tables;
    if (tables.sources.empty()) tables.allocate();
    const aw::Dispatch d = aw::dispatch_and_run(data, index, keys, &tables, sink);
    *ms = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
    o << "\"backend_status\":\"Completed\",\"chosen\":\"" << aw::backend_label(d.chosen)
      << "\",\"ran\":\"" << aw::backend_label(d.ran) << "\",\"probe_ms\":" << d.probe_ms;
  } else if (backend == "hash") {
    hj::Telemetry t;
    const hj::Status st = hj::run_hash_join(data, index, keys, hj::Config{}, sink, &t);
    *ms = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
    o << "\"backend_status\":\"" << hj::status_label(st) << "\",\"logical_pairs\":" << t.logical_pairs
      << ",\"full_hits\":" << t.full_hits;
  } else if (backend == "gpu") {
    gr::Config config;
    config.projected_bits = proj;
    gr::Telemetry t;
    const gr::Status st = gr::run_gpu_root(data, index, keys, config, sink, &t);
    *ms = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
    o << "\"backend_status\":\"" << gr::status_label(st) << "\",\"logical_pairs\":" << t.logical_pairs
      << ",\"filter_survivors\":" << t.filter_survivors << ",\"projected_hits\":" << t.projected_hits
      << ",\"projected_bits\":" << proj << ",\"fast_hits\":" << t.fast_hits
      << ",\"full_hits\":" << t.full_hits << ",\"join_ms\":" << t.join_ms
      << ",\"family_bits\":" << t.family_bits << ",\"filter_bits\":" << t.filter_bits;
  } else {
    *ms = 0.0;
    o << "\"backend_status\":\"unknown backend\"";
  }
  return o.str();
}

// CELLS selects the microproblems (index s * 64 + t) a backend runs:
//   a count N       the reference's declared subsample, select_microproblems(N)
//                   (ter_root_queue_kernels.cpp:111-132); N >= 4096 keeps all;
//   mod:P:I:M       the first M cells c with c % P == I (disjoint slices);
//   perm:S:C        positions [S, S + C) of the reference's own shuffled order,
//                   i.e. select_microproblems(S + C) minus select_microproblems(S):
//                   successive windows are disjoint and spread over all families.
void apply_cells(rg::RootIndex& index, const std::string& spec) {
  if (spec.rfind("mod:", 0) == 0) {
    unsigned p = 1, i = 0, m = 4096;
    std::sscanf(spec.c_str(), "mod:%u:%u:%u", &p, &i, &m);
    index.selected.fill(0U);
    index.selected_count = 0U;
    for (std::uint32_t c = 0; c < 4096U && index.selected_count < m; ++c) {
      if (p != 0U && c % p == i) {
        index.selected[c] = 1U;
        ++index.selected_count;
      }
    }
  } else if (spec.rfind("perm:", 0) == 0) {
    unsigned s = 0, c = 0;
    std::sscanf(spec.c_str(), "perm:%u:%u", &s, &c);
    s = std::min(s, 4096U);
    c = std::min(c, 4096U - s);
    rg::select_microproblems(index, s);
    const auto before = index.selected;
    rg::select_microproblems(index, s + c);
    index.selected_count = 0U;
    for (std::uint32_t cell = 0; cell < 4096U; ++cell) {
      index.selected[cell] = (index.selected[cell] != 0U && before[cell] == 0U) ? 1U : 0U;
      index.selected_count += index.selected[cell];
    }
  } else {
    const auto cells = static_cast<std::uint32_t>(std::strtoul(spec.c_str(), nullptr, 0));
    if (cells < 4096U) { rg::select_microproblems(index, cells); }
  }
}

int cmd_snaproot(int argc, char** argv) {
  if (argc < 6) { return 2; }
  const std::string path = argv[2];
  const std::string backend = argv[3];
  const std::string cells_arg = argv[4];
  const auto proj = static_cast<std::uint32_t>(std::strtoul(argv[5], nullptr, 0));
  const auto workload = rg::load_snapshot_workload(path, true);
  if (workload->status != rg::WorkloadStatus::Completed) {
    std::cout << "{\"error\":\"" << rg::status_label(workload->status) << ": "
              << workload->status_detail << "\"}\n";
    return 1;
  }
  const a64::FamilyKeys keys = a64::build_family_keys(*workload);
  const mr8::Dataset& data = *workload->data;
  rg::RootIndex index;
  rg::build_root_index(data, index);
  apply_cells(index, cells_arg);
  std::vector<std::array<ter::EntryId, 3>> witnesses;
  rg::RootSink sink;
  sink.data = &data;
  sink.index = &index;
  sink.authority = &workload->authority;
  sink.witnesses = &witnesses;
  sink.reset();
  double ms = 0.0;
  const std::string extra = run_backend(backend, data, index, keys, sink, proj, &ms);
  std::uint64_t pairs = 0U;
  for (std::uint32_t s = 0; s < 64U; ++s)
    for (std::uint32_t t = 0; t < 64U; ++t)
      if (index.active(s, t)) pairs += data.q_family[s].size() * data.x_family[t].size();
  std::cout << "{\"backend\":\"" << backend << "\",\"n\":" << workload->n
            << ",\"sizes\":[" << workload->a_size << "," << workload->b_size << "," << workload->c_size
            << "],\"quotient_bits\":" << workload->quotient_bits << ",\"cells\":" << index.selected_count
            << ",\"pairs\":" << pairs << ",\"ms\":" << ms << "," << digest_json(sink.digest) << ","
            << extra << ",\"witnesses\":" << witnesses_json(witnesses) << "}\n";
  return 0;
}

int cmd_snaptime(int argc, char** argv) {
  if (argc < 9) { return 2; }
  const std::string path = argv[2];
  const std::string backend = argv[3];
  const auto proj = static_cast<std::uint32_t>(std::strtoul(argv[4], nullptr, 0));
  const auto cells = static_cast<std::uint32_t>(std::strtoul(argv[5], nullptr, 0));
  const int reps = std::max(1, std::atoi(argv[6]));
  const auto first = static_cast<std::uint32_t>(std::strtoul(argv[7], nullptr, 0));
  const auto stride = static_cast<std::uint32_t>(std::strtoul(argv[8], nullptr, 0));
  const auto load_start = Clock::now();
  const auto workload = rg::load_snapshot_workload(path, true);
  if (workload->status != rg::WorkloadStatus::Completed) {
    std::cout << "{\"error\":\"" << rg::status_label(workload->status) << ": "
              << workload->status_detail << "\"}\n";
    return 1;
  }
  const a64::FamilyKeys keys = a64::build_family_keys(*workload);
  const mr8::Dataset& data = *workload->data;
  rg::RootIndex index;
  rg::build_root_index(data, index);
  const double load_ms = std::chrono::duration<double, std::milli>(Clock::now() - load_start).count();
  for (int rep = 0; rep < reps; ++rep) {
    const std::uint32_t at = (first + static_cast<std::uint32_t>(rep) * stride) % 4096U;
    const std::uint32_t take = std::min(cells, 4096U - at);
    apply_cells(index, "perm:" + std::to_string(at) + ":" + std::to_string(take));
    std::vector<std::array<ter::EntryId, 3>> witnesses;
    rg::RootSink sink;
    sink.data = &data;
    sink.index = &index;
    sink.authority = &workload->authority;
    sink.witnesses = &witnesses;
    sink.reset();
    double ms = 0.0;
    const std::string extra = run_backend(backend, data, index, keys, sink, proj, &ms);
    std::uint64_t pairs = 0U;
    for (std::uint32_t s = 0; s < 64U; ++s)
      for (std::uint32_t t = 0; t < 64U; ++t)
        if (index.active(s, t)) pairs += data.q_family[s].size() * data.x_family[t].size();
    std::cout << "{\"backend\":\"" << backend << "\",\"rep\":" << rep << ",\"first_cell\":" << at
              << ",\"cell_ids\":[";
    bool any = false;
    for (std::uint32_t c = 0; c < 4096U; ++c) {
      if (index.selected[c] == 0U) continue;
      std::cout << (any ? "," : "") << c;
      any = true;
    }
    std::cout << "],\"cells\":" << index.selected_count << ",\"pairs\":" << pairs
              << ",\"load_ms\":" << load_ms << ",\"ms\":" << ms << "," << digest_json(sink.digest)
              << "," << extra << "}\n" << std::flush;
  }
  return 0;
}

bool write_keys(const std::string& path, const sr::Synthetic& root) {
  std::ofstream f(path, std::ios::binary);
  const char magic[8] = {'T', 'E', 'R', 'K', 'E', 'Y', 'S', '1'};
  f.write(magic, 8);
  const std::uint32_t head[2] = {root.bits, 0U};
  f.write(reinterpret_cast<const char*>(head), sizeof head);
  for (std::size_t l = 0; l < 3; ++l) {
    const std::uint64_t count = root.lists[l].size();
    f.write(reinterpret_cast<const char*>(&count), 8);
  }
  for (std::size_t l = 0; l < 3; ++l) {
    for (const auto& v : root.lists[l]) { f.write(reinterpret_cast<const char*>(&v.lo), 8); }
    for (const auto& v : root.lists[l]) {
      const auto h = static_cast<std::uint8_t>(v.hi);
      f.write(reinterpret_cast<const char*>(&h), 1);
    }
    const std::size_t pad = (8U - root.lists[l].size() % 8U) % 8U;
    const char zeros[8] = {};
    f.write(zeros, static_cast<std::streamsize>(pad));
  }
  return static_cast<bool>(f);
}

bool read_keys(const std::string& path, sr::Synthetic& root) {
  std::ifstream f(path, std::ios::binary);
  char magic[8];
  f.read(magic, 8);
  if (!f || std::memcmp(magic, "TERKEYS1", 8) != 0) { return false; }
  std::uint32_t head[2];
  f.read(reinterpret_cast<char*>(head), sizeof head);
  root.bits = head[0];
  std::uint64_t counts[3];
  f.read(reinterpret_cast<char*>(counts), sizeof counts);
  for (std::size_t l = 0; l < 3; ++l) {
    std::vector<std::uint64_t> lo(counts[l]);
    std::vector<std::uint8_t> hi(counts[l]);
    f.read(reinterpret_cast<char*>(lo.data()), static_cast<std::streamsize>(8U * counts[l]));
    f.read(reinterpret_cast<char*>(hi.data()), static_cast<std::streamsize>(counts[l]));
    f.ignore(static_cast<std::streamsize>((8U - counts[l] % 8U) % 8U));
    root.lists[l].resize(counts[l]);
    for (std::size_t i = 0; i < counts[l]; ++i) { root.lists[l][i] = sr::Value{lo[i], hi[i]}; }
  }
  return static_cast<bool>(f);
}

int cmd_synth(int argc, char** argv) {
  if (argc < 7) { return 2; }
  const auto bits = static_cast<std::uint32_t>(std::strtoul(argv[2], nullptr, 0));
  const std::uint64_t seed = std::strtoull(argv[3], nullptr, 0);
  const auto size = static_cast<std::size_t>(std::strtoull(argv[4], nullptr, 0));
  const auto pool = static_cast<std::uint32_t>(std::strtoul(argv[5], nullptr, 0));
  sr::Synthetic root = sr::make_root(bits, seed, size, pool);
  const rg::OutputDigest expected = sr::oracle(root);
  if (!write_keys(argv[6], root)) { return 1; }
  std::cout << "{\"bits\":" << bits << ",\"sizes\":[" << root.lists[0].size() << ","
            << root.lists[1].size() << "," << root.lists[2].size() << "]," << digest_json(expected)
            << "}\n";
  return 0;
}

int cmd_keysroot(int argc, char** argv) {
  if (argc < 7) { return 2; }
  sr::Synthetic root;
  if (!read_keys(argv[2], root)) {
    std::cout << "{\"error\":\"cannot read keys\"}\n";
    return 1;
  }
  const std::string backend = argv[3];
  const std::string cells_arg = argv[4];
  const int reps = std::max(1, std::atoi(argv[5]));
  const auto proj = static_cast<std::uint32_t>(std::strtoul(argv[6], nullptr, 0));
  const auto build_start = Clock::now();
  sr::finish(root);
  const double build_ms = std::chrono::duration<double, std::milli>(Clock::now() - build_start).count();
  apply_cells(root.index, cells_arg);
  std::uint64_t pairs = 0U;
  for (std::uint32_t s = 0; s < 64U; ++s)
    for (std::uint32_t t = 0; t < 64U; ++t)
      if (root.index.active(s, t)) pairs += root.data->q_family[s].size() * root.data->x_family[t].size();
  for (int rep = 0; rep < reps; ++rep) {
    rg::RootSink sink = sr::make_sink(root);
    double ms = 0.0;
    std::string extra;
    if (backend == "brute") {
      const auto start = Clock::now();
      sink.digest = sr::oracle(root);
      ms = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
      extra = "\"backend_status\":\"Completed\"";
    } else {
      extra = run_backend(backend, *root.data, root.index, root.keys, sink, proj, &ms);
    }
    std::cout << "{\"backend\":\"" << backend << "\",\"rep\":" << rep << ",\"bits\":" << root.bits
              << ",\"cells\":" << root.index.selected_count << ",\"pairs\":" << pairs
              << ",\"build_ms\":" << build_ms << ",\"ms\":" << ms << "," << digest_json(sink.digest)
              << "," << extra << "}\n" << std::flush;
  }
  return 0;
}

int cmd_plant(int argc, char** argv) {
  if (argc < 5) { return 2; }
  const auto count = static_cast<std::uint32_t>(std::strtoul(argv[3], nullptr, 0));
  const std::uint64_t seed = std::strtoull(argv[4], nullptr, 0);
  auto workload = rg::load_snapshot_workload(argv[2], true);
  if (workload->status != rg::WorkloadStatus::Completed || !workload->authority.ok) {
    std::cout << "{\"error\":\"" << rg::status_label(workload->status) << "\"}\n";
    return 1;
  }
  std::uint32_t anchor = 4096U;
  {
    rg::RootIndex probe;
    rg::build_root_index(*workload->data, probe);
    rg::select_microproblems(probe, 1U);
    for (std::uint32_t cell = 0U; cell < 4096U; ++cell) {
      anchor = probe.selected[cell] != 0U ? cell : anchor;
    }
  }
  const std::size_t before = workload->key_lo[2].size();
  const ter::arwlf_campaign::PlantedTargets planted(
      *workload, anchor,
      ter::arwlf_campaign::Plant{ter::arwlf_campaign::PlantKind::Positive, count, seed});
  std::cout << "{\"anchor_cell\":" << anchor << ",\"first_planted\":" << planted.first_planted()
            << ",\"d_lo\":[";
  for (std::size_t i = before; i < workload->key_lo[2].size(); ++i) {
    std::cout << (i > before ? "," : "") << "\"" << workload->key_lo[2][i] << "\"";
  }
  std::cout << "],\"d_hi\":[";
  for (std::size_t i = before; i < workload->key_hi[2].size(); ++i) {
    std::cout << (i > before ? "," : "") << static_cast<int>(workload->key_hi[2][i]);
  }
  std::cout << "],\"expected\":[";
  for (std::size_t i = 0; i < planted.expected().size(); ++i) {
    const auto& w = planted.expected()[i];
    std::cout << (i ? "," : "") << "[" << w[0] << "," << w[1] << "," << w[2] << "]";
  }
  std::cout << "]}\n";
  return 0;
}

int cmd_report(int argc, char** argv) {
  if (argc < 4) { return 2; }
  rs::Snapshot snap;
  std::string error;
  if (!rs::load(argv[2], snap, error)) {
    std::cout << "{\"error\":\"" << error << "\"}\n";
    return 1;
  }
  const std::string policy_name = argv[3];
  const ter::RootOutputPolicy policy =
      policy_name == "count" ? ter::RootOutputPolicy::CountOnly
      : policy_name == "canon" ? ter::RootOutputPolicy::FullCanonicalOutput
                               : ter::RootOutputPolicy::FirstWitness;
  const std::uint32_t n = snap.header.n;
  ter::FullTerRootCapture capture;
  const auto params = ter::derive_full_ter_parameters(ter::ShapeFamily::FiniteSanity, n, n);
  capture.status = params.status;
  capture.parameters = params.value;
  capture.seed = snap.header.seed;
  capture.execution_mode = ter::TerExecutionMode::FullTer;
  for (std::size_t l = 0; l < 3; ++l) {
    const std::uint64_t count = snap.header.entries[l];
    capture.children[l].resize(count);
    capture.residues_words_le[l].resize(count);
    for (std::uint64_t i = 0; i < count; ++i) {
      auto& digits = capture.children[l][i];
      digits.resize(n);
      for (std::uint32_t c = 0; c < n; ++c) {
        digits[c] = static_cast<std::int8_t>(snap.digit(l, i, c));
      }
      const auto res = snap.residue(l, i);
      capture.residues_words_le[l][i].assign(res.begin(), res.end());
    }
    const auto ct = snap.child_target(l);
    capture.child_targets_words_le[l].assign(ct.begin(), ct.end());
  }
  const auto rt = snap.root_target();
  capture.root_target_words_le.assign(rt.begin(), rt.end());
  ter::FullTerConfig config = rg::authentic_config(snap.header.seed);
  config.memory_limit_bytes = std::uint64_t{64} << 30;
  const auto start = Clock::now();
  const auto report = ter::report_full_ter_root(capture, config, policy);
  const double ms = std::chrono::duration<double, std::milli>(Clock::now() - start).count();
  const auto count = ter::count_full_ter_root(capture, config);
  std::cout << "{\"status\":" << static_cast<int>(report.status)
            << ",\"policy\":" << static_cast<int>(report.effective_root_output_policy)
            << ",\"valid_root_count\":" << report.valid_root_count
            << ",\"retained_root_count\":" << report.retained_root_count
            << ",\"count_status\":" << static_cast<int>(count.status)
            << ",\"count_valid_root_count\":" << count.valid_root_count
            << ",\"modular\":" << report.telemetry.modular_candidates
            << ",\"ms\":" << ms << ",\"message\":\"" << report.message << "\"}\n";
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) {
    std::cerr << "usage: terref solve|capture|snaproot|snaptime|synth|keysroot|plant|report ...\n";
    return 2;
  }
  const std::string cmd = argv[1];
  int rc = 2;
  if (cmd == "solve") { rc = cmd_solve(argc, argv); }
  else if (cmd == "capture") { rc = cmd_capture(argc, argv); }
  else if (cmd == "snaproot") { rc = cmd_snaproot(argc, argv); }
  else if (cmd == "snaptime") { rc = cmd_snaptime(argc, argv); }
  else if (cmd == "synth") { rc = cmd_synth(argc, argv); }
  else if (cmd == "keysroot") { rc = cmd_keysroot(argc, argv); }
  else if (cmd == "report") { rc = cmd_report(argc, argv); }
  else if (cmd == "plant") { rc = cmd_plant(argc, argv); }
  if (rc == 2) { std::cerr << "bad arguments for " << cmd << "\n"; }
  return rc;
}
