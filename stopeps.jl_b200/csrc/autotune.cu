// Autotuner: launch-shape choices picked by timing the candidates on the
// first call with a new shape, then reused by every engine on that device.
//
// A tuned operation asks lookup(key); on a miss it times each candidate on
// its real operands with CUDA events on the engine's stream (a warm-up run
// and a timed run each, host-synchronised), calls store() with the winner and
// the timings, and then runs the winner.  The table is process-wide and keyed
// by device, operation and shape, so every engine of the process (the batch
// workers included) uses the same choice once it is made; report_json()
// lists the table.  Tuning is off unless an engine's `autotune` flag is set:
// a choice changes the order of floating-point sums, so results can differ
// at rounding level between a tuned and an untuned run (not between engines
// of one tuned run).
#include "engine.h"
#include <mutex>
#include <sstream>

namespace sps {
namespace tune {

namespace {
struct Entry {
  int choice;
  std::vector<std::pair<int, float>> timings;
};
std::mutex g_mu;
std::map<std::string, Entry> g_table;
}  // namespace

std::string key(Engine& E, const char* op, std::initializer_list<long long> shape) {
  std::ostringstream s;
  s << E.device << ":" << op;
  for (long long v : shape) s << ":" << v;
  return s.str();
}

bool lookup(const std::string& k, int* choice) {
  std::lock_guard<std::mutex> g(g_mu);
  auto it = g_table.find(k);
  if (it == g_table.end()) return false;
  *choice = it->second.choice;
  return true;
}

static void store(const std::string& k, int choice, const std::vector<std::pair<int, float>>& timings) {
  std::lock_guard<std::mutex> g(g_mu);
  g_table.emplace(k, Entry{choice, timings});   // the first stored choice wins
}

int pick(Engine& E, const std::string& k, const std::vector<int>& candidates, const std::function<void(int)>& run) {
  int c = 0;
  if (lookup(k, &c)) return c;
  cudaEvent_t a, b;
  SPS_CUDA(cudaEventCreate(&a));
  SPS_CUDA(cudaEventCreate(&b));
  std::vector<std::pair<int, float>> t;
  int best = candidates.front();
  float best_ms = 1e30f;
  for (int cand : candidates) {
    run(cand);   // warm-up (attributes, caches)
    SPS_CUDA(cudaEventRecord(a, E.stream));
    run(cand);
    SPS_CUDA(cudaEventRecord(b, E.stream));
    SPS_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    SPS_CUDA(cudaEventElapsedTime(&ms, a, b));
    t.emplace_back(cand, ms);
    if (ms < best_ms) {
      best_ms = ms;
      best = cand;
    }
  }
  SPS_CUDA(cudaEventDestroy(a));
  SPS_CUDA(cudaEventDestroy(b));
  store(k, best, t);
  lookup(k, &best);   // a concurrent tuner may have stored first
  return best;
}

std::string report_json() {
  std::lock_guard<std::mutex> g(g_mu);
  std::ostringstream s;
  s << "{";
  bool first = true;
  for (auto& kv : g_table) {
    s << (first ? "" : ", ") << "\"" << kv.first << "\": {\"choice\": " << kv.second.choice << ", \"ms\": {";
    bool f2 = true;
    for (auto& t : kv.second.timings) {
      s << (f2 ? "" : ", ") << "\"" << t.first << "\": " << t.second;
      f2 = false;
    }
    s << "}}";
    first = false;
  }
  s << "}";
  return s.str();
}

void clear() {
  std::lock_guard<std::mutex> g(g_mu);
  g_table.clear();
}

}  // namespace tune
}  // namespace sps
