// Autotuner of the energy pipeline's run-time tiles and splits (Tuning in
// tree.hpp): for one tree it times each candidate value of one parameter at
// a time (coordinate descent, the other parameters held) with CUDA events on
// the tree's stream and keeps the fastest. Results are cached per (digits,
// precision, floor(log2 N)) in a JSON table: tuning.json beside the library,
// or the file named by HPDMK_TUNING. Trees look the table up at
// construction (the same size bucket, else the nearest bucket of the same
// digits and precision, else the defaults).
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "tree.hpp"

namespace pdmk {
namespace {

using Key = std::tuple<int, int, int>;  // digits, precision, floor(log2 N)

std::mutex g_mu;
std::map<Key, Tuning> g_table;
bool g_loaded = false;

int size_bucket(long n) { return n <= 1 ? 0 : int(std::floor(std::log2(double(n)))); }

std::string default_path() {
  if (const char* e = std::getenv("HPDMK_TUNING")) return e;
  Dl_info info{};
  if (dladdr(reinterpret_cast<const void*>(&default_path), &info) && info.dli_fname) {
    std::string f = info.dli_fname;
    const size_t slash = f.rfind('/');
    return (slash == std::string::npos ? std::string(".") : f.substr(0, slash)) + "/tuning.json";
  }
  return "tuning.json";
}

// the integer value of "name": in one flat JSON object's text; false when absent
bool field(const std::string& obj, const char* name, int& out) {
  const std::string k = std::string("\"") + name + "\"";
  size_t p = obj.find(k);
  if (p == std::string::npos) return false;
  p = obj.find(':', p + k.size());
  if (p == std::string::npos) return false;
  char* end = nullptr;
  const long v = std::strtol(obj.c_str() + p + 1, &end, 10);
  if (end == obj.c_str() + p + 1) return false;
  out = int(v);
  return true;
}

// Reads a table written by save(): a JSON array of flat objects with integer
// fields. Entries missing a key field are skipped; missing tuning fields keep
// their defaults.
void load_file(const std::string& path, std::map<Key, Tuning>& table) {
  std::ifstream in(path);
  if (!in) return;
  std::stringstream ss;
  ss << in.rdbuf();
  const std::string s = ss.str();
  size_t p = 0;
  while ((p = s.find('{', p)) != std::string::npos) {
    const size_t e = s.find('}', p);
    if (e == std::string::npos) break;
    const std::string obj = s.substr(p, e - p + 1);
    p = e + 1;
    int d, pr, nb;
    if (!field(obj, "digits", d) || !field(obj, "precision", pr) || !field(obj, "n_log2", nb)) continue;
    Tuning t;
    field(obj, "ksplit", t.ksplit);
    field(obj, "ksplit_root", t.ksplit_root);
    field(obj, "inc_waves", t.inc_waves);
    field(obj, "res_ny_max", t.res_ny_max);
    table[Key{d, pr, nb}] = t;
  }
}

void ensure_loaded() {
  if (g_loaded) return;
  load_file(default_path(), g_table);
  g_loaded = true;
}

bool save(const std::string& path, const std::map<Key, Tuning>& table) {
  std::ofstream out(path);
  if (!out) return false;
  out << "[\n";
  size_t i = 0;
  for (const auto& kv : table) {
    const Tuning& t = kv.second;
    out << "  {\"digits\": " << std::get<0>(kv.first) << ", \"precision\": " << std::get<1>(kv.first)
        << ", \"n_log2\": " << std::get<2>(kv.first) << ", \"ksplit\": " << t.ksplit
        << ", \"ksplit_root\": " << t.ksplit_root << ", \"inc_waves\": " << t.inc_waves
        << ", \"res_ny_max\": " << t.res_ny_max << "}" << (++i < table.size() ? "," : "") << "\n";
  }
  out << "]\n";
  return bool(out);
}

// the entry of this kind: the same size bucket, else the nearest bucket of
// the same digits and precision, else the defaults
Tuning lookup_in(const std::map<Key, Tuning>& table, int digits, int precision, long n) {
  const int nb = size_bucket(n);
  auto it = table.find(Key{digits, precision, nb});
  if (it != table.end()) return it->second;
  int best = 1 << 30;
  Tuning out;
  for (const auto& kv : table)
    if (std::get<0>(kv.first) == digits && std::get<1>(kv.first) == precision) {
      const int dist = std::abs(std::get<2>(kv.first) - nb);
      if (dist < best) {
        best = dist;
        out = kv.second;
      }
    }
  return out;
}

}  // namespace

// the cached choice for a tree of this kind (defaults when the table has none)
Tuning lookup_tuning(int digits, int precision, long n) {
  std::lock_guard<std::mutex> g(g_mu);
  ensure_loaded();
  return lookup_in(g_table, digits, precision, n);
}

// the lookup on the table in one file (host only; used by the tests)
Tuning lookup_tuning_file(const std::string& path, int digits, int precision, long n) {
  std::map<Key, Tuning> table;
  load_file(path, table);
  return lookup_in(table, digits, precision, n);
}

// Searches the tree's tuning and records it in the table and at `path` (the
// default table when null or empty). out[0..3]: the chosen ksplit,
// ksplit_root, inc_waves, res_ny_max; times[0..2] (may be null): the
// outgoing, incoming and near-field milliseconds with them.
void autotune_tree(DmkTree& t, const char* path, int reps, int* out, double* times) {
  reps = std::max(1, reps);
  Tuning cur = t.tuning();
  t.form_outgoing_pw();  // warm-up: the pipeline's set-up and the kernels' first launches
  t.form_incoming_pw();
  auto search = [&](int Tuning::*field_ptr, const std::vector<int>& values, int phase) {
    double best = 1e300;
    int best_v = cur.*field_ptr;
    for (int v : values) {
      Tuning c = cur;
      c.*field_ptr = v;
      t.set_tuning(c);
      if (t.tuning().*field_ptr != v) continue;  // outside the supported range
      t.time_phase(phase, 1);                    // this value's first run
      const double ms = t.time_phase(phase, reps);
      if (ms < best) {
        best = ms;
        best_v = v;
      }
    }
    cur.*field_ptr = best_v;
    t.set_tuning(cur);
    return best;
  };
  search(&Tuning::ksplit, {1024, 2048, 4096, 8192, 16384}, 0);
  const double t_out = search(&Tuning::ksplit_root, {1024, 2048, 4096, 8192, 16384}, 0);
  const double t_inc = search(&Tuning::inc_waves, {1, 2, 4, 8, 16}, 1);
  const double t_res = search(&Tuning::res_ny_max, {1, 2, 4, 8}, 2);
  // leave the tree's expansions formed with the chosen values
  t.form_outgoing_pw();
  t.form_incoming_pw();
  const Tuning& ch = t.tuning();
  if (out) {
    out[0] = ch.ksplit;
    out[1] = ch.ksplit_root;
    out[2] = ch.inc_waves;
    out[3] = ch.res_ny_max;
  }
  if (times) {
    times[0] = t_out;
    times[1] = t_inc;
    times[2] = t_res;
  }
  std::lock_guard<std::mutex> g(g_mu);
  ensure_loaded();
  const std::string p = (path && *path) ? std::string(path) : default_path();
  std::map<Key, Tuning> table;
  load_file(p, table);  // keep the file's other entries
  const Key key{t.digits(), t.precision(), size_bucket(t.n_particles())};
  table[key] = ch;
  g_table[key] = ch;
  if (!save(p, table)) throw std::runtime_error("autotune: cannot write the tuning table " + p);
}

}  // namespace pdmk
