// Autotuner cache: the kernel variants a plan measured fastest, per problem
// key (kind, orbital sizes, precision, slices, dtype).  Process-wide and
// thread-safe; optionally persisted as text lines "key: v0 v1 ..." in the
// file named by LIBPT_TUNE_FILE (read once, appended on every new entry).
// LIBPT_AUTOTUNE=0 turns measuring off (plans then use fixed heuristics);
// LIBPT_TUNE_VERBOSE=1 prints every measured candidate.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "tune.h"

namespace ptb {

namespace {

std::mutex g_mu;
std::map<std::string, std::vector<int>> g_cache;
bool g_loaded = false;

const char *tune_file() {
  const char *f = std::getenv("LIBPT_TUNE_FILE");
  return f && *f ? f : nullptr;
}

void load_locked() {
  if (g_loaded) return;
  g_loaded = true;
  const char *f = tune_file();
  if (!f) return;
  FILE *fp = std::fopen(f, "r");
  if (!fp) return;
  char line[512];
  while (std::fgets(line, sizeof(line), fp)) {
    const char *colon = std::strchr(line, ':');
    if (!colon) continue;
    std::string key(line, colon - line);
    std::istringstream in(colon + 1);
    std::vector<int> v;
    int x;
    while (in >> x) v.push_back(x);
    if (!v.empty()) g_cache[key] = v;
  }
  std::fclose(fp);
}

}  // namespace

std::string tune_key(int kind, int oa, int va, int ob, int vb, int precision,
                     int slices, int dtype) {
  std::ostringstream k;
  k << "k" << kind << " o" << oa << "," << ob << " v" << va << "," << vb
    << " p" << precision << " s" << slices << " d" << dtype;
  return k.str();
}

bool tune_enabled() {
  const char *e = std::getenv("LIBPT_AUTOTUNE");
  return !(e && std::strcmp(e, "0") == 0);
}

bool tune_verbose() {
  const char *e = std::getenv("LIBPT_TUNE_VERBOSE");
  return e && std::strcmp(e, "1") == 0;
}

bool tune_lookup(const std::string &key, std::vector<int> *choice) {
  std::lock_guard<std::mutex> g(g_mu);
  load_locked();
  auto it = g_cache.find(key);
  if (it == g_cache.end()) return false;
  *choice = it->second;
  return true;
}

void tune_store(const std::string &key, const std::vector<int> &choice) {
  std::lock_guard<std::mutex> g(g_mu);
  load_locked();
  g_cache[key] = choice;
  const char *f = tune_file();
  if (!f) return;
  FILE *fp = std::fopen(f, "a");
  if (!fp) return;
  std::fprintf(fp, "%s:", key.c_str());
  for (int x : choice) std::fprintf(fp, " %d", x);
  std::fprintf(fp, "\n");
  std::fclose(fp);
}

void tune_clear() {
  std::lock_guard<std::mutex> g(g_mu);
  g_cache.clear();
  g_loaded = true;   // an explicit clear also forgets the file's entries
}

}  // namespace ptb
