// Kernel-configuration choice: a forced configuration (ssblasSetKernelConfig), else the tuning
// table written by the autotuner (ssblasex_b200/autotune.py), else the built-in default.
//
// The table is a JSON file with one entry per line:
//   {"path": <ssblasPath_t>, "bucket": "m<a>n<b>k<c>b<d>", "config": <index>},
// where a, b, c, d are ceil(log2(.)) of m, n, k and the batch count. It is read once, from
// $SSBLAS_TUNE_FILE if set, else from tune/ssblas_tune.json next to the shared library.
#include <dlfcn.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <map>
#include <mutex>
#include <string>

#include "internal.h"

namespace ssb {
namespace {

std::mutex g_tune_mutex;
bool g_loaded = false;
std::map<std::pair<int, std::string>, int> g_table;
constexpr int kKeys = 16;
int g_forced[kKeys] = {-1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1};

int clog2(long x) {
  int r = 0;
  while ((1L << r) < x && r < 62) ++r;
  return r;
}

std::string table_path() {
  if (const char* e = getenv("SSBLAS_TUNE_FILE")) return e;
  Dl_info info;
  if (dladdr((void*)&table_path, &info) && info.dli_fname) {
    std::string p(info.dli_fname);
    const size_t s = p.rfind('/');
    return (s == std::string::npos ? std::string(".") : p.substr(0, s)) + "/tune/ssblas_tune.json";
  }
  return "tune/ssblas_tune.json";
}

void load_table() {
  g_loaded = true;
  FILE* f = fopen(table_path().c_str(), "r");
  if (!f) return;
  char line[512];
  while (fgets(line, sizeof(line), f)) {
    int path = -1, cfg = -1;
    char bucket[128] = {0};
    const char* p = strstr(line, "\"path\"");
    if (!p) continue;
    if (sscanf(p, "\"path\": %d, \"bucket\": \"%127[^\"]\", \"config\": %d", &path, bucket, &cfg) == 3 && path >= 0 &&
        cfg >= 0)
      g_table[{path, std::string(bucket)}] = cfg;
  }
  fclose(f);
}

}  // namespace

std::string size_bucket(long m, long n, long k, long batch) {
  char b[64];
  snprintf(b, sizeof(b), "m%dn%dk%db%d", clog2(m), clog2(n), clog2(k), clog2(batch));
  return b;
}

int choose_config(int path, long m, long n, long k, long batch, int fallback) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  if (path >= 0 && path < kKeys && g_forced[path] >= 0) return g_forced[path];
  if (!g_loaded) load_table();
  auto it = g_table.find({path, size_bucket(m, n, k, batch)});
  return it != g_table.end() ? it->second : fallback;
}

int forced_config(int path) {
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  return (path >= 0 && path < kKeys) ? g_forced[path] : -1;
}

}  // namespace ssb

extern "C" ssblasStatus_t ssblasSetKernelConfig(int path, int config) {
  if (path < 0 || path >= ssb::kKeys || config < -1 || config > 64) return SSBLAS_STATUS_INVALID_VALUE;
  std::lock_guard<std::mutex> lock(ssb::g_tune_mutex);
  ssb::g_forced[path] = config;
  return SSBLAS_STATUS_SUCCESS;
}

extern "C" ssblasStatus_t ssblasReloadTuning(void) {
  std::lock_guard<std::mutex> lock(ssb::g_tune_mutex);
  ssb::g_table.clear();
  ssb::load_table();
  return SSBLAS_STATUS_SUCCESS;
}
