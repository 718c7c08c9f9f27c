// Run-time autotuner: picks a launch parameter (the split-K count of the
// chi0 contractions) for each problem shape by timing the candidates once on
// the caller's own data, then reuses the choice.  Choices are kept per
// process and, when a cache file is set, in a small JSON object
// {"shape key": choice, ...} that later runs read back.
#include <cstdio>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include "autotune.cuh"

namespace qsgw {

static int g_mode = 0;                     // 0 = heuristics, 1 = tune unseen shapes
static int g_suspend = 0;

TuneSuspend::TuneSuspend() { ++g_suspend; }
TuneSuspend::~TuneSuspend() { --g_suspend; }
static std::string g_path;
static std::map<std::string, int> g_cache;
static std::map<std::string, double> g_notes;   // error estimates of the slice-count trials (report only)

static void load_cache() {
  std::ifstream f(g_path);
  if (!f) return;
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string t = ss.str();
  size_t i = 0;
  while ((i = t.find('"', i)) != std::string::npos) {
    const size_t j = t.find('"', i + 1);
    if (j == std::string::npos) break;
    const std::string key = t.substr(i + 1, j - i - 1);
    size_t k = t.find(':', j);
    if (k == std::string::npos) break;
    g_cache[key] = std::atoi(t.c_str() + k + 1);
    i = t.find_first_of(",}", k);
    if (i == std::string::npos) break;
  }
}

static std::string cache_json() {
  std::string o = "{";
  bool first = true;
  for (const auto& kv : g_cache) {
    o += first ? "\"" : ", \"";
    o += kv.first + "\": " + std::to_string(kv.second);
    first = false;
  }
  return o + "}";
}

static std::string report_json() {
  std::string o = cache_json();
  if (g_notes.empty()) return o;
  o.pop_back();                                  // the closing brace
  char num[64];
  for (const auto& kv : g_notes) {
    std::snprintf(num, sizeof(num), "%.6e", kv.second);
    o += (o.size() > 1 ? ", \"" : "\"") + kv.first + "\": " + num;
  }
  return o + "}";
}

static void save_cache() {
  if (g_path.empty()) return;
  std::ofstream f(g_path, std::ios::trunc);
  if (f) f << cache_json() << "\n";
}

int tuned_choice(const std::string& key, const std::vector<int>& cands, int heuristic,
                 const std::function<int(int)>& run, cudaStream_t s, int* chosen, bool* tried) {
  *chosen = heuristic;
  *tried = false;
  auto it = g_cache.find(key);
  if (it != g_cache.end()) {
    *chosen = it->second;
    return QSGW_OK;
  }
  if (g_mode == 0 || g_suspend > 0 || ctx().capturing || cands.size() < 2) return QSGW_OK;
  cudaEvent_t e0, e1;
  QSGW_CUDA(cudaEventCreate(&e0));
  QSGW_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  int rc = QSGW_OK;
  *tried = true;
  for (int c : cands) {
    cudaEventRecord(e0, s);
    rc = run(c);
    if (rc) break;
    cudaEventRecord(e1, s);
    if ((rc = check_cuda(cudaEventSynchronize(e1), "autotune sync"))) break;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) { best = ms; *chosen = c; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  g_cache[key] = *chosen;
  save_cache();
  return QSGW_OK;
}

bool tuned_lookup(const std::string& key, int* v) {
  auto it = g_cache.find(key);
  if (it == g_cache.end()) return false;
  *v = it->second;
  return true;
}

int tuned_slices(const std::string& key, const std::vector<int>& cands, int top, double tol,
                 const std::function<int(int, double*)>& err, int fallback, int* chosen) {
  *chosen = fallback;
  auto it = g_cache.find(key);
  if (it != g_cache.end()) {
    *chosen = it->second;
    return QSGW_OK;
  }
  if (g_suspend > 0 || ctx().capturing) return QSGW_OK;
  *chosen = top;
  for (int c : cands) {
    double e = 0.0;
    const int rc = err(c, &e);
    if (rc) return rc;
    g_notes[key + " err@" + std::to_string(c)] = e;
    if (e <= tol) {
      *chosen = c;
      break;
    }
  }
  g_cache[key] = *chosen;
  save_cache();
  return QSGW_OK;
}

}  // namespace qsgw

using namespace qsgw;

extern "C" int qsgw_set_autotune(int mode, const char* cache_path) {
  int rc = require_init();
  if (rc) return rc;
  QSGW_ARG(mode == 0 || mode == 1, "set_autotune: mode %d (0 or 1)", mode);
  g_mode = mode;
  g_path = cache_path ? cache_path : "";
  if (!g_path.empty()) load_cache();
  return QSGW_OK;
}

extern "C" int qsgw_autotune_report(char* buf, int len) {
  if (!buf || len <= 0) return QSGW_ERR_ARG;
  const std::string j = report_json();
  std::snprintf(buf, static_cast<size_t>(len), "%s", j.c_str());
  return static_cast<int>(j.size()) < len ? QSGW_OK : QSGW_ERR_ARG;
}
