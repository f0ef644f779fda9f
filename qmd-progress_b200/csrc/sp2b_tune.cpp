// Launch-configuration autotuner: the decision table, its file, and the timing loop.
#include "sp2b_tune.h"

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>

#include "sp2b.h"

namespace sp2b {

namespace {

struct Table {
  std::mutex mu;
  bool loaded = false;
  std::map<std::string, int> choice;
  std::map<std::string, std::vector<float>> ms;
};

Table& table() {
  static Table t;
  return t;
}

const char* tune_file() {
  const char* f = std::getenv("SP2B_TUNE_FILE");
  return (f && f[0]) ? f : nullptr;
}

// Reads SP2B_TUNE_FILE once; later lines for the same key win.  Caller holds t.mu.
void load_locked(Table& t) {
  if (t.loaded) return;
  t.loaded = true;
  const char* path = tune_file();
  if (!path) return;
  FILE* f = std::fopen(path, "r");
  if (!f) return;
  char line[4096];
  while (std::fgets(line, sizeof(line), f)) {
    std::istringstream in(line);
    std::string key;
    int c = -1;
    if (!(in >> key >> c) || key.empty() || key[0] == '#' || c < 0) continue;
    std::vector<float> v;
    float x;
    while (in >> x) v.push_back(x);
    t.choice[key] = c;
    t.ms[key] = v;
  }
  std::fclose(f);
}

}  // namespace

int device_sms() {
  static std::atomic<int> sms[64];   // per device, 0 until first queried
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 148;
  if (dev >= 0 && dev < 64 && sms[dev].load(std::memory_order_relaxed) > 0)
    return sms[dev].load(std::memory_order_relaxed);
  int v = 0;
  if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
    return 148;
  if (dev >= 0 && dev < 64) sms[dev].store(v, std::memory_order_relaxed);
  return v;
}

bool tune_enabled() {
  const char* e = std::getenv("SP2B_TUNE");
  return !(e && e[0] == '0');
}

bool tune_lookup(const std::string& key, int* choice) {
  Table& t = table();
  std::lock_guard<std::mutex> lk(t.mu);
  load_locked(t);
  auto it = t.choice.find(key);
  if (it == t.choice.end()) return false;
  *choice = it->second;
  return true;
}

void tune_store(const std::string& key, int choice, const std::vector<float>& ms) {
  Table& t = table();
  std::lock_guard<std::mutex> lk(t.mu);
  load_locked(t);
  t.choice[key] = choice;
  t.ms[key] = ms;
  const char* path = tune_file();
  if (!path) return;
  if (FILE* f = std::fopen(path, "a")) {
    std::fprintf(f, "%s %d", key.c_str(), choice);
    for (float x : ms) std::fprintf(f, " %.4f", x);
    std::fprintf(f, "\n");
    std::fclose(f);
  }
}

int tune_measure(int ncand, int reps, cudaStream_t st, const std::function<int(int)>& run,
                 std::vector<float>* ms, int* best) {
  ms->assign(ncand, 0.0f);
  *best = 0;
  if (ncand <= 1) return SP2B_OK;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    return SP2B_CUDA_ERROR;
  }
  int rc = SP2B_OK;
  std::vector<float> t;
  for (int c = 0; c < ncand && rc == SP2B_OK; ++c) {
    if ((rc = run(c)) != SP2B_OK) break;   // untimed: layouts, graphs, caches
    t.clear();
    for (int r = 0; r < std::max(reps, 1) && rc == SP2B_OK; ++r) {
      if (cudaEventRecord(e0, st) != cudaSuccess) rc = SP2B_CUDA_ERROR;
      if (rc == SP2B_OK) rc = run(c);
      if (rc == SP2B_OK && (cudaEventRecord(e1, st) != cudaSuccess ||
                            cudaEventSynchronize(e1) != cudaSuccess))
        rc = SP2B_CUDA_ERROR;
      float x = 0.0f;
      if (rc == SP2B_OK && cudaEventElapsedTime(&x, e0, e1) != cudaSuccess) rc = SP2B_CUDA_ERROR;
      t.push_back(x);
    }
    if (rc != SP2B_OK) break;
    std::sort(t.begin(), t.end());
    (*ms)[c] = t[t.size() / 2];
    if ((*ms)[c] < (*ms)[*best]) *best = c;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

}  // namespace sp2b

using namespace sp2b;

extern "C" int sp2b_tune_get(const char* key, int* choice, float* ms, int max_ms, int* nms) {
  if (!key || !choice) return SP2B_BAD_ARG;
  Table& t = table();
  std::lock_guard<std::mutex> lk(t.mu);
  load_locked(t);
  auto it = t.choice.find(key);
  if (it == t.choice.end()) return SP2B_BAD_ARG;
  *choice = it->second;
  const std::vector<float>& v = t.ms[key];
  if (nms) *nms = (int)v.size();
  if (ms)
    for (int i = 0; i < std::min(max_ms, (int)v.size()); ++i) ms[i] = v[i];
  return SP2B_OK;
}

extern "C" int sp2b_tune_set(const char* key, int choice) {
  if (!key || !key[0] || choice < 0 || std::strpbrk(key, " \t\n")) return SP2B_BAD_ARG;
  tune_store(key, choice, {});
  return SP2B_OK;
}

extern "C" int sp2b_tune_keys(char* buf, int cap) {
  Table& t = table();
  std::lock_guard<std::mutex> lk(t.mu);
  load_locked(t);
  std::string s;
  for (const auto& kv : t.choice) {
    s += kv.first;
    s += '\n';
  }
  if (buf && cap > 0) {
    const int m = std::min(cap - 1, (int)s.size());
    std::memcpy(buf, s.data(), m);
    buf[m] = '\0';
  }
  return (int)s.size() + 1;
}

extern "C" int sp2b_tune_clear(void) {
  Table& t = table();
  std::lock_guard<std::mutex> lk(t.mu);
  t.choice.clear();
  t.ms.clear();
  t.loaded = true;   // a cleared table does not re-read the file
  return SP2B_OK;
}
