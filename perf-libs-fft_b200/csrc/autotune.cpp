// Plan-time autotuning for the planner rigor levels, with wisdom.
//
// The reference's MEASURE / PATIENT / EXHAUSTIVE planners time candidate
// decompositions within a budget and keep the fastest, remembering the
// choice per problem (src/plfft.cpp:149-184, src/planner/benchmarker.hpp:
// 33-93, src/planner/wisdom.hpp:23-37).  Here the candidates are device
// schedules for the same problem: for C2C (make_c2c_candidates) launch
// shapes, kernel families, four-step shapes; for R2C, C2R and the R2R kinds
// (make_real_candidates) the fused kernel's launch shapes and the real-wrap
// schedule.  Each is run on scratch device buffers
// with the plan's layout and timed with CUDA events: one warm-up, then
// rounds of k executions (k calibrated so a round lasts >= 50 us), 3 to 7
// rounds, median per execution.  The default schedule is timed first and a
// challenger replaces it only if it is at least 2% faster.  Budget of timed
// work per plan: 0.1 s (MEASURE), 0.5 s (PATIENT), 2 s (EXHAUSTIVE).
//
// Wisdom maps a problem key (kind, n, batch layout, direction, scale flag,
// precision, device name) to the description of the winning schedule.  It
// lives in the process; with PLFFT_B200_WISDOM=<file> it is loaded from and
// appended to that file, and plfft_cuda_wisdom_export/import/forget manage
// it explicitly.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

#include "plan.hpp"

namespace plfft_b200 {

namespace {

std::mutex g_wisdom_mu;
std::map<std::string, std::string> g_wisdom;
bool g_wisdom_loaded = false;

void load_env_wisdom_locked() {
  if (g_wisdom_loaded) return;
  g_wisdom_loaded = true;
  const char* path = std::getenv("PLFFT_B200_WISDOM");
  if (!path) return;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    const size_t tab = line.find('\t');
    if (tab != std::string::npos) g_wisdom[line.substr(0, tab)] = line.substr(tab + 1);
  }
}

void remember(const std::string& key, const std::string& choice) {
  std::lock_guard<std::mutex> lock(g_wisdom_mu);
  load_env_wisdom_locked();
  g_wisdom[key] = choice;
  if (const char* path = std::getenv("PLFFT_B200_WISDOM")) {
    std::ofstream f(path, std::ios::app);
    f << key << '\t' << choice << '\n';
  }
}

bool recall(const std::string& key, std::string& choice) {
  std::lock_guard<std::mutex> lock(g_wisdom_mu);
  load_env_wisdom_locked();
  auto it = g_wisdom.find(key);
  if (it == g_wisdom.end()) return false;
  choice = it->second;
  return true;
}

std::string device_name() {
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceProp p{};
  if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return "unknown";
  return p.name;
}

int64_t span(int64_t howmany, int64_t dist, int64_t n, int64_t stride) {
  return (howmany - 1) * (howmany > 1 ? dist : 0) + (n - 1) * stride + 1;
}

// median seconds per execution of `node`, or a negative value on error
double time_node(const Node& node, const void* in, void* out, void* ws, cudaStream_t st, double budget_left) {
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return -1;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return -1;
  }
  double result = -1;
  std::vector<double> rounds;
  int k = 1;
  if (node.run(in, out, ws, st) == cudaSuccess && cudaStreamSynchronize(st) == cudaSuccess) {
    double spent = 0;
    while (rounds.size() < 7) {
      cudaEventRecord(e0, st);
      bool ok = true;
      for (int i = 0; i < k && ok; ++i) ok = node.run(in, out, ws, st) == cudaSuccess;
      cudaEventRecord(e1, st);
      if (!ok || cudaEventSynchronize(e1) != cudaSuccess) {
        rounds.clear();
        break;
      }
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      spent += ms * 1e-3;
      if (ms < 0.05f && k < (1 << 16)) {  // calibrate: rounds of >= 50 us
        k *= 2;
        continue;
      }
      rounds.push_back(ms * 1e-3 / k);
      if (rounds.size() >= 3 && spent > budget_left) break;
    }
    if (!rounds.empty()) {
      std::sort(rounds.begin(), rounds.end());
      result = rounds[rounds.size() / 2];
    }
  }
  cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return result;
}

}  // namespace

bool wisdom_recall(const std::string& key, std::string& choice) { return recall(key, choice); }
void wisdom_remember(const std::string& key, const std::string& choice) { remember(key, choice); }
std::string wisdom_device() { return device_name(); }

std::string wisdom_key(const ConfigData& c) {
  static const char* kinds[] = {"c2c", "r2c", "c2r", "r2r"};
  std::ostringstream o;
  o << kinds[int(c.kind)] << " n=" << c.n << " hm=" << c.howmany << " is=" << c.istride << " id=" << c.idist
    << " os=" << c.ostride << " od=" << c.odist << " dir=" << c.payload << " scaled=" << (c.scale != 1.0)
    << " prec=" << c.precision << " dev=" << device_name();
  return o.str();
}

namespace {

// Times the candidates (default first) on scratch buffers of the plan's
// spans and keeps the fastest; the wisdom key remembers the choice.
std::unique_ptr<Node> tune(const ConfigData& c, std::vector<std::unique_ptr<Node>> cands, int64_t nin, int64_t nout,
                           size_t in_elem, size_t out_elem, std::string* note) {
  const double budget = c.rigor == PLFFT_MEASURE ? 0.1 : (c.rigor == PLFFT_PATIENT ? 0.5 : 2.0);
  const std::string key = wisdom_key(c);
  std::string known;
  if (recall(key, known)) {
    for (auto& cand : cands)
      if (cand->describe() == known) {
        if (note) *note = "wisdom";
        return std::move(cand);
      }
  }
  if (cands.size() == 1) return std::move(cands[0]);
  // scratch buffers with the plan's spans and the largest workspace
  size_t ws_bytes = 0;
  for (auto& cand : cands) ws_bytes = std::max(ws_bytes, cand->workspace());
  DevBuf din, dout, dws;
  const size_t ib = size_t(span(c.howmany, c.idist, nin, c.istride)) * in_elem;
  const size_t ob = size_t(span(c.howmany, c.odist, nout, c.ostride)) * out_elem;
  cudaStream_t st = nullptr;
  if (din.alloc(ib) != cudaSuccess || dout.alloc(ob) != cudaSuccess || dws.alloc(ws_bytes) != cudaSuccess ||
      cudaMemset(din.p, 0, ib) != cudaSuccess || cudaStreamCreate(&st) != cudaSuccess) {
    cudaGetLastError();
    if (st) cudaStreamDestroy(st);
    return std::move(cands[0]);  // no room to measure: keep the default schedule
  }
  const auto t0 = std::chrono::steady_clock::now();
  size_t best = 0;
  double best_t = -1;
  int timed = 0;
  for (size_t i = 0; i < cands.size(); ++i) {
    const double used = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (i > 1 && used > budget) break;  // the default and one challenger at least
    const double t = time_node(*cands[i], din.p, dout.p, dws.p, st, (budget - used) / double(cands.size() - i));
    ++timed;
    if (t <= 0) continue;  // failed to run: never chosen
    // the first schedule that ran is the incumbent; challengers need a 2% win
    if (best_t < 0 || t < best_t * 0.98) {
      best = i;
      best_t = t;
    }
  }
  cudaStreamDestroy(st);
  if (note) {
    std::ostringstream o;
    o << "autotuned " << timed << "/" << cands.size() << " candidates";
    *note = o.str();
  }
  remember(key, cands[best]->describe());
  return std::move(cands[best]);
}

int tune_level(const ConfigData& c) { return c.rigor == PLFFT_MEASURE ? 1 : (c.rigor == PLFFT_PATIENT ? 2 : 3); }

}  // namespace

std::unique_ptr<Node> autotune_c2c(const ConfigData& c, const Layout& lay, std::string* why, std::string* note) {
  auto cands = make_c2c_candidates(c.n, lay, c.payload, float(c.scale), c.precision, tune_level(c));
  if (cands.empty()) return make_c2c_node(c.n, lay, c.payload, float(c.scale), c.precision, why);
  return tune(c, std::move(cands), c.n, c.n, sizeof(float2), sizeof(float2), note);
}

std::unique_ptr<Node> autotune_real(const ConfigData& c, const Layout& lay, int fused_kind, int wrap_kind,
                                    std::string* why, std::string* note) {
  auto cands = make_real_candidates(fused_kind, wrap_kind, c.n, lay, float(c.scale), tune_level(c));
  if (cands.empty()) return make_realwrap_node(wrap_kind, c.n, lay, c.scale, why);
  const int64_t h = c.n / 2 + 1;
  const bool cin = c.kind == TKind::C2R, cout = c.kind == TKind::R2C;
  return tune(c, std::move(cands), cin ? h : c.n, cout ? h : c.n, cin ? sizeof(float2) : sizeof(float),
              cout ? sizeof(float2) : sizeof(float), note);
}

}  // namespace plfft_b200

// ---------------------------------------------------------------------------
// C-ABI: wisdom management (extension; the reference keeps its wisdom
// internal to the process)
// ---------------------------------------------------------------------------
#include "../../include/plfft_cuda.h"

extern "C" plfft_status_t plfft_cuda_wisdom_export(const char* path) {
  using namespace plfft_b200;
  if (!path) return PLFFT_NULL_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_wisdom_mu);
  load_env_wisdom_locked();
  std::ofstream f(path, std::ios::trunc);
  if (!f) return PLFFT_INVALID_ARGUMENT;
  for (auto& kv : g_wisdom) f << kv.first << '\t' << kv.second << '\n';
  return f ? PLFFT_OK : PLFFT_INVALID_ARGUMENT;
}

extern "C" plfft_status_t plfft_cuda_wisdom_import(const char* path) {
  using namespace plfft_b200;
  if (!path) return PLFFT_NULL_ARGUMENT;
  std::ifstream f(path);
  if (!f) return PLFFT_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(g_wisdom_mu);
  load_env_wisdom_locked();
  std::string line;
  while (std::getline(f, line)) {
    const size_t tab = line.find('\t');
    if (tab != std::string::npos) g_wisdom[line.substr(0, tab)] = line.substr(tab + 1);
  }
  return PLFFT_OK;
}

extern "C" void plfft_cuda_wisdom_forget(void) {
  using namespace plfft_b200;
  std::lock_guard<std::mutex> lock(g_wisdom_mu);
  g_wisdom.clear();
  g_wisdom_loaded = true;  // do not reload the environment file
}
