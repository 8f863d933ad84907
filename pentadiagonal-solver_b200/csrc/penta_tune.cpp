// penta_tune.cpp -- the process-wide tuning table.
//
// An autotuner (pentadsolver_autotune_solve / _plan in penta_api.cpp, or a
// file written by an earlier run) records, per solve shape class, the kernel
// choice that measured fastest.  The class key is
//
//   <GPU name>|<solve or plan>|<f64 or f32>|<x or yz>|n<N>|l<L>
//
// with N the line length and L the number of lines (a plan: its longest line
// and all its lines), each rounded up to a power of two.  The automatic
// selection consults the table for shapes that neither the environment
// selectors nor the handle fix; plan creation with ctas = 0 takes its CTA
// count from it.  On first use the table is read from the file named by
// PENTA_TUNING_CACHE, when that variable is set.
//
// File format: one entry per line, tab-separated
//   key  spec  algo  lanes  ctas  ms
// where spec is a pentadsolver_set_tuning string ("auto", "tmem=3,4",
// "no-tmem", "no-tma"), algo a family name ("thomas-pcr", "naive", ...),
// lanes the PCR lanes (0 automatic), ctas a plan's CTA count (0 for
// solves) and ms the measured time.  Lines starting with '#' are comments.
#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "penta_internal.hpp"

namespace penta {
namespace {

std::mutex g_mu;
std::unordered_map<std::string, TuneChoice> g_table;
std::atomic<size_t> g_size{0};
bool g_env_loaded = false;

long long bucket(long long v) {
  long long b = 1;
  while (b < v) b <<= 1;
  return b;
}

bool parse_line(const std::string &line, std::string &key, TuneChoice &c) {
  if (line.empty() || line[0] == '#') return false;
  std::vector<std::string> f;
  std::string cur;
  for (char ch : line) {
    if (ch == '\t') {
      f.push_back(cur);
      cur.clear();
    } else if (ch != '\r' && ch != '\n') {
      cur.push_back(ch);
    }
  }
  f.push_back(cur);
  if (f.size() != 6 || f[0].empty()) return false;
  char *end = nullptr;
  const long lanes = std::strtol(f[3].c_str(), &end, 10);
  if (*end != '\0' || lanes < 0 || lanes > 32) return false;
  const long ctas = std::strtol(f[4].c_str(), &end, 10);
  if (*end != '\0' || ctas < 0 || ctas > 1 << 20) return false;
  const double ms = std::strtod(f[5].c_str(), &end);
  if (*end != '\0') return false;
  key = f[0];
  c.spec = f[1] == "auto" ? "" : f[1];
  c.algo = f[2];
  c.lanes = (int)lanes;
  c.ctas = (int)ctas;
  c.ms = ms;
  return true;
}

bool load_locked(const char *path) {
  std::ifstream in(path);
  if (!in) return false;
  std::string line, key;
  while (std::getline(in, line)) {
    TuneChoice c;
    if (parse_line(line, key, c)) g_table[key] = c;
  }
  g_size.store(g_table.size());
  return true;
}

void ensure_env_loaded_locked() {
  if (g_env_loaded) return;
  g_env_loaded = true;
  const char *p = std::getenv("PENTA_TUNING_CACHE");
  if (p != nullptr && p[0] != '\0') load_locked(p);
}

}  // namespace

std::string tune_key(const std::string &gpu, const char *kind, size_t elem, int dir,
                     long long n, long long lines) {
  std::ostringstream o;
  o << gpu << '|' << kind << '|' << (elem == 8 ? "f64" : "f32") << '|' << (dir == 0 ? "x" : "yz")
    << "|n" << bucket(n) << "|l" << bucket(lines);
  return o.str();
}

bool tune_lookup(const std::string &key, TuneChoice &out) {
  std::lock_guard<std::mutex> lock(g_mu);
  ensure_env_loaded_locked();
  if (g_size.load() == 0) return false;
  auto it = g_table.find(key);
  if (it == g_table.end()) return false;
  out = it->second;
  return true;
}

bool tune_table_empty() {
  std::lock_guard<std::mutex> lock(g_mu);
  ensure_env_loaded_locked();
  return g_table.empty();
}

void tune_store(const std::string &key, const TuneChoice &c) {
  std::lock_guard<std::mutex> lock(g_mu);
  ensure_env_loaded_locked();
  g_table[key] = c;
  g_size.store(g_table.size());
}

bool tune_load(const char *path) {
  std::lock_guard<std::mutex> lock(g_mu);
  ensure_env_loaded_locked();
  return load_locked(path);
}

bool tune_save(const char *path) {
  std::vector<std::pair<std::string, TuneChoice>> rows;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    ensure_env_loaded_locked();
    rows.assign(g_table.begin(), g_table.end());
  }
  std::sort(rows.begin(), rows.end(),
            [](const auto &a, const auto &b) { return a.first < b.first; });
  std::ofstream out(path, std::ios::trunc);
  if (!out) return false;
  out << "# pentadsolver tuning table: key\tspec\talgo\tlanes\tctas\tms\n";
  for (const auto &r : rows) {
    char ms[32];
    std::snprintf(ms, sizeof ms, "%.6g", r.second.ms);
    out << r.first << '\t' << (r.second.spec.empty() ? "auto" : r.second.spec) << '\t'
        << (r.second.algo.empty() ? "auto" : r.second.algo) << '\t' << r.second.lanes << '\t'
        << r.second.ctas << '\t' << ms << '\n';
  }
  return (bool)out;
}

void tune_clear() {
  std::lock_guard<std::mutex> lock(g_mu);
  g_env_loaded = true;  // an explicit clear also drops the environment's file
  g_table.clear();
  g_size.store(0);
}

std::string tune_format(const TuneChoice &c) {
  char ms[32];
  std::snprintf(ms, sizeof ms, "%.6g", c.ms);
  return (c.spec.empty() ? std::string("auto") : c.spec) + "\t" +
         (c.algo.empty() ? std::string("auto") : c.algo) + "\t" + std::to_string(c.lanes) +
         "\t" + std::to_string(c.ctas) + "\t" + ms;
}

}  // namespace penta
