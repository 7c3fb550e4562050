// tuning.cu — the per-shape tuning table (see tuning.hpp).
//
// File format: one record per line, whitespace-separated key=value pairs,
//   join kind=<0|1> build=<log2 rows> dense=<0|1> lf=<load factor> part=<-1|0|1> bits=<1..8>
//   join_agg kind=<0|1> build=<log2 rows> block=<threads> blocks=<per SM> rows=<in flight> table=<log2 slots>
//   agg rows=<log2 rows> block=<threads>
// Lines starting with '#' are comments.
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <tuple>

#include "tuning.hpp"

namespace prism {

namespace {

struct Table {
  std::mutex mu;
  bool loaded_env = false;
  std::map<std::pair<int, int>, JoinTuning> join;
  std::map<std::pair<int, int>, AggTuning> join_agg;
  std::map<int, AggTuning> agg;
};

Table& table() {
  static Table* t = new Table();  // never destroyed: read by calls until exit
  return *t;
}

int log2_bucket(int64_t n) {
  int b = 0;
  while (b < 62 && ((int64_t)1 << (b + 1)) <= std::max<int64_t>(n, 1)) ++b;
  return b;
}

void parse_line(Table& T, const std::string& line) {
  std::istringstream in(line);
  std::string kind;
  if (!(in >> kind) || kind.empty() || kind[0] == '#') return;
  std::map<std::string, std::string> kv;
  std::string tok;
  while (in >> tok) {
    const size_t eq = tok.find('=');
    if (eq == std::string::npos) fail(PRISM_ERR_INVALID_ARGUMENT, "tuning file: '" + tok + "' is not key=value");
    kv[tok.substr(0, eq)] = tok.substr(eq + 1);
  }
  auto geti = [&](const char* k) -> int {
    auto it = kv.find(k);
    if (it == kv.end()) fail(PRISM_ERR_INVALID_ARGUMENT, std::string("tuning file: missing ") + k + " in: " + line);
    return std::atoi(it->second.c_str());
  };
  if (kind == "join") {
    JoinTuning t;
    t.dense = geti("dense") != 0;
    t.load_factor = std::atof(kv.count("lf") ? kv["lf"].c_str() : "0.5");
    t.partition = geti("part");
    t.partition_bits = geti("bits");
    if (t.load_factor < 0.1 || t.load_factor > 0.9 || t.partition < -1 || t.partition > 1 || t.partition_bits < 1 ||
        t.partition_bits > 8)
      fail(PRISM_ERR_INVALID_ARGUMENT, "tuning file: join value out of range in: " + line);
    T.join[{geti("kind"), geti("build")}] = t;
  } else if (kind == "join_agg") {
    AggTuning t;
    t.join_block = geti("block");
    t.join_min_blocks = geti("blocks");
    t.join_rows = geti("rows");
    t.join_table_log2 = geti("table");
    const int b = t.join_block, r = t.join_rows;
    if (!(b == 128 || b == 256 || b == 512 || b == 1024) || t.join_min_blocks < 1 || t.join_min_blocks > 8 ||
        !(r == 1 || r == 2 || r == 4 || r == 8) || t.join_table_log2 < 8 || t.join_table_log2 > 12)
      fail(PRISM_ERR_INVALID_ARGUMENT, "tuning file: join_agg value out of range in: " + line);
    T.join_agg[{geti("kind"), geti("build")}] = t;
  } else if (kind == "agg") {
    AggTuning t;
    t.hash_block = geti("block");
    if (!(t.hash_block == 256 || t.hash_block == 512 || t.hash_block == 1024))
      fail(PRISM_ERR_INVALID_ARGUMENT, "tuning file: agg block out of range in: " + line);
    T.agg[geti("rows")] = t;
  } else {
    fail(PRISM_ERR_INVALID_ARGUMENT, "tuning file: unknown record '" + kind + "'");
  }
}

void load_into(Table& T, const std::string& path) {
  std::ifstream f(path);
  if (!f) fail(PRISM_ERR_INVALID_ARGUMENT, "cannot read tuning file " + path);
  std::string line;
  while (std::getline(f, line)) parse_line(T, line);
}

// PRISM_TUNING_FILE, once, under T.mu
void ensure_env(Table& T) {
  if (T.loaded_env) return;
  T.loaded_env = true;
  const char* p = std::getenv("PRISM_TUNING_FILE");
  if (p && *p) {
    std::ifstream probe(p);
    if (probe) load_into(T, p);  // a file not written yet is an empty table
  }
}

}  // namespace

JoinShape join_shape(const Batch& build, const std::vector<int>& keys) {
  JoinShape s;
  s.key_kind = (keys.size() == 1 && keys[0] >= 0 && keys[0] < (int)build.cols.size() &&
                build.cols[keys[0]]->type == TY_I64)
                   ? 0
                   : 1;
  s.build_log2 = log2_bucket(build.rows);
  return s;
}

bool apply_join_tuning(const JoinShape& shape, JoinTuning& t) {
  Table& T = table();
  std::lock_guard<std::mutex> lk(T.mu);
  ensure_env(T);
  auto it = T.join.find({shape.key_kind, shape.build_log2});
  if (it == T.join.end()) return false;
  const JoinTuning& r = it->second;
  if (!(t.fixed & JoinTuning::FIX_DENSE)) t.dense = r.dense;
  if (!(t.fixed & JoinTuning::FIX_PARTITION)) {
    t.partition = r.partition;
    t.partition_bits = r.partition_bits;
  }
  if (!(t.fixed & JoinTuning::FIX_LOAD)) t.load_factor = r.load_factor;
  return true;
}

bool apply_join_agg_tuning(const JoinShape& shape, AggTuning& t) {
  Table& T = table();
  std::lock_guard<std::mutex> lk(T.mu);
  ensure_env(T);
  auto it = T.join_agg.find({shape.key_kind, shape.build_log2});
  if (it == T.join_agg.end() || (t.fixed & AggTuning::FIX_JOIN_SHAPE)) return false;
  t.join_block = it->second.join_block;
  t.join_min_blocks = it->second.join_min_blocks;
  t.join_rows = it->second.join_rows;
  t.join_table_log2 = it->second.join_table_log2;
  return true;
}

bool apply_agg_tuning(int64_t rows, AggTuning& t) {
  Table& T = table();
  std::lock_guard<std::mutex> lk(T.mu);
  ensure_env(T);
  auto it = T.agg.find(log2_bucket(rows));
  if (it == T.agg.end() || (t.fixed & AggTuning::FIX_HASH_BLOCK)) return false;
  t.hash_block = it->second.hash_block;
  return true;
}

void record_join_tuning(const JoinShape& shape, const JoinTuning& t) {
  Table& T = table();
  std::lock_guard<std::mutex> lk(T.mu);
  ensure_env(T);
  T.join[{shape.key_kind, shape.build_log2}] = t;
}

void record_join_agg_tuning(const JoinShape& shape, const AggTuning& t) {
  Table& T = table();
  std::lock_guard<std::mutex> lk(T.mu);
  ensure_env(T);
  T.join_agg[{shape.key_kind, shape.build_log2}] = t;
}

void record_agg_tuning(int64_t rows, const AggTuning& t) {
  Table& T = table();
  std::lock_guard<std::mutex> lk(T.mu);
  ensure_env(T);
  T.agg[log2_bucket(rows)] = t;
}

void tuning_clear() {
  Table& T = table();
  std::lock_guard<std::mutex> lk(T.mu);
  T.loaded_env = true;  // a cleared table stays empty (the file is not re-read)
  T.join.clear();
  T.join_agg.clear();
  T.agg.clear();
}

std::string tuning_dump() {
  Table& T = table();
  std::lock_guard<std::mutex> lk(T.mu);
  ensure_env(T);
  std::ostringstream o;
  o << "# prism-gpu tuning table: the fastest measured setting per shape class\n";
  for (auto& [k, t] : T.join)
    o << "join kind=" << k.first << " build=" << k.second << " dense=" << (t.dense ? 1 : 0) << " lf=" << t.load_factor
      << " part=" << t.partition << " bits=" << t.partition_bits << "\n";
  for (auto& [k, t] : T.join_agg)
    o << "join_agg kind=" << k.first << " build=" << k.second << " block=" << t.join_block
      << " blocks=" << t.join_min_blocks << " rows=" << t.join_rows << " table=" << t.join_table_log2 << "\n";
  for (auto& [k, t] : T.agg) o << "agg rows=" << k << " block=" << t.hash_block << "\n";
  return o.str();
}

void tuning_save(const std::string& path) {
  const std::string text = tuning_dump();
  std::ofstream f(path);
  if (!f) fail(PRISM_ERR_INVALID_ARGUMENT, "cannot write tuning file " + path);
  f << text;
  if (!f) fail(PRISM_ERR_INVALID_ARGUMENT, "cannot write tuning file " + path);
}

void tuning_load(const std::string& path) {
  Table& T = table();
  Table fresh;
  load_into(fresh, path);  // parse fully before replacing anything
  std::lock_guard<std::mutex> lk(T.mu);
  T.loaded_env = true;
  for (auto& [k, v] : fresh.join) T.join[k] = v;
  for (auto& [k, v] : fresh.join_agg) T.join_agg[k] = v;
  for (auto& [k, v] : fresh.agg) T.agg[k] = v;
}

}  // namespace prism
