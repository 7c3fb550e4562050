// oracle.cpp — TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the reference hot path, used as the parity checker for
// the GPU engine and as the timed CPU baseline. Each function cites the
// reference code it restates. The GPU product never links or calls this file.
//
// Reference algorithms restated here (paths relative to the reference tree):
//   native/prism-executor/src/hash_join.rs        HashTable::build/probe, assembly
//   native/prism-executor/src/hash_aggregate.rs   FxHash grouping, f64 accumulators
//   native/prism-executor/src/filter_project.rs   predicate / expression evaluation
//   native/prism-substrait/src/executor.rs        fused join -> aggregate
// Third-party behaviour the reference relies on (arrow-rs 57.3.0 cast, cmp,
// take, filter, numeric kernels; rayon 1.11.0 chunking) is restated from its
// published semantics; see the notes at each use.

#include "oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>

#include "oracle_arrow.hpp"

using namespace oracle;

namespace {

thread_local std::string g_err;

int guard(const std::function<void()>& fn) {
  try {
    fn();
    g_err.clear();
    return PRISM_OK;
  } catch (const Error& e) {
    g_err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    g_err = "out of host memory";
    return PRISM_ERR_NO_MEMORY;
  } catch (const std::exception& e) {
    g_err = e.what();
    return PRISM_ERR_INTERNAL;
  }
}

// Run fn(i) for i in [0, n) on up to n_threads threads (rayon stand-in).
void parallel_for(int64_t n, int n_threads, const std::function<void(int64_t)>& fn) {
  if (n_threads <= 1 || n <= 1) {
    for (int64_t i = 0; i < n; ++i) fn(i);
    return;
  }
  std::atomic<int64_t> next{0};
  std::vector<std::thread> ts;
  std::mutex em;
  Error first{0, ""};
  bool failed = false;
  int nt = (int)std::min<int64_t>(n_threads, n);
  for (int t = 0; t < nt; ++t) {
    ts.emplace_back([&]() {
      for (;;) {
        int64_t i = next.fetch_add(1);
        if (i >= n) return;
        try {
          fn(i);
        } catch (const Error& e) {
          std::lock_guard<std::mutex> lk(em);
          if (!failed) { failed = true; first = e; }
        }
      }
    });
  }
  for (auto& t : ts) t.join();
  if (failed) throw first;
}

std::vector<Batch> import_all(const ArrowArray* const* arrays, const ArrowSchema* schema, int n) {
  std::vector<Batch> out;
  for (int i = 0; i < n; ++i) out.push_back(import_batch(arrays[i], schema));
  return out;
}

const Col& col_at(const Batch& b, int idx) {
  if (idx < 0 || idx >= (int)b.cols.size())
    fail(PRISM_ERR_INVALID_ARGUMENT, "column index " + std::to_string(idx) + " out of range");
  return *b.cols[idx];
}

// ============================================================== hashing ====
// FxHasher (hash_aggregate.rs:24-75): state = state * K + word.
constexpr uint64_t FX_K = 0x517cc1b727220a95ULL;
struct Fx {
  uint64_t s = 0;
  void word(uint64_t w) { s = s * FX_K + w; }
  void bytes(const uint8_t* p, size_t n) {  // Hasher::write, 8-byte LE chunks
    for (size_t i = 0; i < n; i += 8) {
      uint64_t w = 0;
      std::memcpy(&w, p + i, std::min<size_t>(8, n - i));
      word(w);
    }
  }
  void str(std::string_view v) {  // impl Hash for str: write(bytes) + write_u8(0xff)
    bytes(reinterpret_cast<const uint8_t*>(v.data()), v.size());
    word(0xff);
  }
};

// Fallback identity for types the reference hashes through their Debug text
// (hash_aggregate.rs:502): a type tag word followed by the raw value. Any
// injective encoding gives the same grouping; this one is shared with the GPU.
constexpr uint64_t FALLBACK_TAG = 0x9E3779B97F4A7C15ULL;

// hash_array_value (hash_aggregate.rs:492-504) into an FxHasher.
void fx_value(Fx& h, const Col& c, int64_t row) {
  if (c.null_at(row)) { h.word(0); return; }  // 0u8.hash -> write_u8(0)
  switch (c.ty) {
    case T_I32: case T_I64: h.word((uint64_t)c.ival(row)); return;  // write_i32/i64
    case T_F64: h.word(c.fbits(row)); return;                       // to_bits().hash
    case T_UTF8: case T_DICT: h.str(c.sval(row)); return;           // str hash (dictionary: decoded)
    case T_DEC128: {
      __int128 v = c.dval(row);
      h.word(FALLBACK_TAG ^ (uint64_t)c.ty);
      h.word((uint64_t)v);
      h.word((uint64_t)(v >> 64));
      return;
    }
    case T_F32: {
      float f = reinterpret_cast<const float*>(c.vals)[c.off + row];
      uint32_t u;
      std::memcpy(&u, &f, 4);
      h.word(FALLBACK_TAG ^ (uint64_t)c.ty);
      h.word(u);
      return;
    }
    default:
      h.word(FALLBACK_TAG ^ (uint64_t)c.ty);
      h.word((uint64_t)c.ival(row));
      return;
  }
}

uint64_t hash_group_keys(const Batch& b, const std::vector<int>& keys, int64_t row) {
  Fx h;
  for (int k : keys) fx_value(h, *b.cols[k], row);
  return h.s;
}

// ======================================================== f64 exact sum ====
// Exact accumulation of doubles in 2^-1074 units, 32-bit limbs held in
// signed 64-bit counters (carry-save), then one correctly rounded conversion.
struct ExactSum {
  static constexpr int L = 72;  // 2304 bits
  int64_t limb[L] = {0};
  int64_t adds = 0;
  bool nan = false, pinf = false, ninf = false;
  void add(double v) {
    if (std::isnan(v)) { nan = true; return; }
    if (std::isinf(v)) { (v > 0 ? pinf : ninf) = true; return; }
    if (v == 0) return;
    uint64_t u;
    std::memcpy(&u, &v, 8);
    int e = (int)((u >> 52) & 0x7ff);
    uint64_t m = u & ((1ULL << 52) - 1);
    if (e) m |= (1ULL << 52); else e = 1;
    int pos = e - 1;  // bit position of m's LSB in 2^-1074 units
    int k = pos >> 5, sh = pos & 31;
    unsigned __int128 x = (unsigned __int128)m << sh;
    int64_t sgn = (u >> 63) ? -1 : 1;
    for (int j = 0; j < 3 && k + j < L; ++j) {
      int64_t part = (int64_t)(uint32_t)(x >> (32 * j));
      limb[k + j] += sgn * part;
    }
    if (++adds >= (1LL << 30)) normalize();
  }
  void normalize() {
    int64_t carry = 0;
    for (int i = 0; i < L; ++i) {
      int64_t v = limb[i] + carry;
      carry = v >> 32;  // arithmetic shift: floor division
      limb[i] = v & 0xffffffffLL;
    }
    limb[L - 1] += carry << 32;
    adds = 0;
  }
  double result() {
    if (nan || (pinf && ninf)) return std::numeric_limits<double>::quiet_NaN();
    if (pinf) return std::numeric_limits<double>::infinity();
    if (ninf) return -std::numeric_limits<double>::infinity();
    normalize();
    // sign: top limb holds the signed carry
    bool neg = limb[L - 1] < 0;
    uint32_t mag[L];
    if (neg) {  // two's complement negate over 32-bit limbs
      uint64_t c = 1;
      for (int i = 0; i < L; ++i) {
        uint64_t v = (uint64_t)(uint32_t)(~(uint32_t)limb[i]) + c;
        mag[i] = (uint32_t)v;
        c = v >> 32;
      }
    } else {
      for (int i = 0; i < L; ++i) mag[i] = (uint32_t)limb[i];
    }
    int top = -1;
    for (int i = L - 1; i >= 0; --i)
      if (mag[i]) { top = i * 32 + 31 - __builtin_clz(mag[i]); break; }
    if (top < 0) return 0.0;
    auto bit = [&](int p) -> uint64_t { return p < 0 ? 0 : (mag[p >> 5] >> (p & 31)) & 1; };
    double r;
    if (top <= 52) {  // exact, possibly subnormal
      uint64_t m = 0;
      for (int p = top; p >= 0; --p) m = (m << 1) | bit(p);
      r = std::ldexp((double)m, -1074);
    } else {
      uint64_t m = 0;
      for (int p = top; p >= top - 52; --p) m = (m << 1) | bit(p);
      int lo = top - 52;
      uint64_t rb = bit(lo - 1);
      bool sticky = false;
      for (int p = lo - 2; p >= 0 && !sticky; --p) sticky = bit(p);
      if (rb && (sticky || (m & 1))) ++m;
      r = std::ldexp((double)m, lo - 1074);
    }
    return neg ? -r : r;
  }
};

// ===================================================== column utilities ====
ColP take_col(const Col& c, const std::vector<int64_t>& idx, const std::string& name,
              bool nullable) {
  // arrow compute::take; idx < 0 means a null index. A null value at a valid
  // index keeps its raw slot for fixed-width and Boolean columns (take_native
  // and take_bits copy the values buffer whatever its validity) and is empty
  // for Utf8 (take_bytes appends no bytes for it).
  Builder b = builder_like(c, name, nullable);
  b.reserve((int64_t)idx.size());
  for (int64_t i : idx) {
    if (i < 0) { b.push_null(); continue; }
    if (i >= c.len) fail(PRISM_ERR_ARROW, "Out-of-bounds index " + std::to_string(i));
    if (c.null_at(i) && c.ty != T_UTF8) b.push_slot(c, i);
    else b.push_from(c, i);
  }
  return b.finish();
}

ColP filter_col(const Col& c, const std::vector<uint8_t>& keep) {
  Builder b = builder_like(c, c.name, c.nullable);
  for (int64_t i = 0; i < c.len; ++i)
    if (keep[i]) b.push_slot(c, i);
  return b.finish();
}

// cast of a column to Float64 as arrow_cast::cast does for the aggregate and
// arithmetic inputs (hash_aggregate.rs:227-245, filter_project.rs:236-238).
// Null slots: a Float64 column is not cast and keeps its raw slots; the
// Decimal128 -> Float64 cast maps every slot (unary), so raw slots are
// mapped too; integer, Float32 and Boolean casts (numeric_cast / unary_opt,
// cast_bool_to_numeric) write only valid rows into a zeroed buffer, so a
// null row reads 0.
struct F64Col {
  std::vector<double> v;
  std::vector<uint8_t> valid;  // 1 = valid
};
F64Col cast_f64(const Col& c, const char* what) {
  F64Col r;
  r.v.resize(c.len);
  r.valid.resize(c.len);
  switch (c.ty) {
    case T_I8: case T_I16: case T_I32: case T_I64: case T_U8: case T_U16: case T_U32:
    case T_U64: case T_F32: case T_F64: case T_BOOL: case T_DEC128:
      for (int64_t i = 0; i < c.len; ++i) {
        r.valid[i] = !c.null_at(i);
        r.v[i] = (r.valid[i] || c.ty == T_F64 || c.ty == T_DEC128) ? c.fval(i) : 0.0;
      }
      return r;
    case T_NULL:
      for (int64_t i = 0; i < c.len; ++i) { r.v[i] = 0; r.valid[i] = 0; }
      return r;
    default:
      fail(PRISM_ERR_ARROW, std::string("Cast error: cannot cast column '") + c.name +
                                "' to Float64 for " + what);
  }
}

// ================================================================= join ====
// HashTable (hash_join.rs:77-201).
constexpr int HASH_PARTITIONS = 64;
constexpr uint64_t HASH_PART_MASK = HASH_PARTITIONS - 1;

inline uint64_t hash_i64_fast(int64_t v) { return (uint64_t)v * FX_K; }  // hash_join.rs:371-373

// General-path row hash. The reference uses SipHash-1-3 (DefaultHasher) here
// (hash_join.rs:378-392) only to bucket rows; matches are then verified with
// keys_equal, so any hash that is equal for equal keys yields the same match
// set. Null rows hash a marker only (the reference hashes 0u8 for them).
uint64_t mix64(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return x;
}
uint64_t general_row_hash(const Batch& b, const std::vector<int>& keys, int64_t row) {
  uint64_t h = 0x2545F4914F6CDD1DULL;
  for (int k : keys) {
    const Col& c = *b.cols[k];
    uint64_t w;
    if (c.null_at(row)) w = 0x6a09e667f3bcc909ULL;
    else if (c.ty == T_UTF8 || c.ty == T_DICT) {
      auto s = c.sval(row);
      Fx f;
      f.str(s);
      w = f.s;
    } else if (c.ty == T_F64) w = c.fbits(row);
    else if (c.ty == T_DEC128) { __int128 v = c.dval(row); w = (uint64_t)v ^ mix64((uint64_t)(v >> 64)); }
    else if (c.ty == T_F32) { float f = reinterpret_cast<const float*>(c.vals)[c.off + row]; uint32_t u; std::memcpy(&u, &f, 4); w = u; }
    else w = (uint64_t)c.ival(row);
    h = mix64(h ^ w) + 0x9E3779B97F4A7C15ULL;
  }
  return h;
}

// keys_equal (hash_join.rs:628-670) combined with the hash precondition:
// a null row only ever meets a null row (its hash is the null marker), and
// raw values must be equal (null bits are otherwise ignored). Float64 needs
// equal bits (the hash uses to_bits) and `==` (so NaN never matches).
bool keys_equal(const Batch& a, const std::vector<int>& ka, int64_t ra, const Batch& b,
                const std::vector<int>& kb, int64_t rb) {
  for (size_t i = 0; i < ka.size(); ++i) {
    const Col& x = *a.cols[ka[i]];
    const Col& y = *b.cols[kb[i]];
    bool nx = x.null_at(ra), ny = y.null_at(rb);
    if (nx != ny) return false;
    switch (x.ty) {
      case T_UTF8: case T_DICT:
        if (x.sval(ra) != y.sval(rb)) return false;
        break;
      case T_F64: {
        double dx = x.fval(ra), dy = y.fval(rb);
        if (!(dx == dy) || x.fbits(ra) != y.fbits(rb)) return false;
        break;
      }
      case T_F32: {
        float fx = reinterpret_cast<const float*>(x.vals)[x.off + ra];
        float fy = reinterpret_cast<const float*>(y.vals)[y.off + rb];
        uint32_t ux, uy;
        std::memcpy(&ux, &fx, 4);
        std::memcpy(&uy, &fy, 4);
        if (!(fx == fy) || ux != uy) return false;
        break;
      }
      case T_DEC128:
        if (x.dval(ra) != y.dval(rb)) return false;
        break;
      case T_NULL:
        break;
      default:
        if (x.ival(ra) != y.ival(rb)) return false;
    }
  }
  return true;
}

struct FlatMap {  // open addressing u64 -> row list (stands in for hashbrown)
  std::vector<uint64_t> keys;
  std::vector<uint8_t> used;
  std::vector<std::vector<uint32_t>> vals;
  uint64_t mask = 0;
  void init(size_t n) {
    size_t cap = 16;
    while (cap < n * 2) cap <<= 1;
    keys.assign(cap, 0);
    used.assign(cap, 0);
    vals.resize(cap);
    mask = cap - 1;
  }
  static uint64_t spread(uint64_t h) { return mix64(h); }
  std::vector<uint32_t>& entry(uint64_t h) {
    uint64_t s = spread(h) & mask;
    while (used[s] && keys[s] != h) s = (s + 1) & mask;
    if (!used[s]) { used[s] = 1; keys[s] = h; }
    return vals[s];
  }
  const std::vector<uint32_t>* get(uint64_t h) const {
    uint64_t s = spread(h) & mask;
    while (used[s]) {
      if (keys[s] == h) return &vals[s];
      s = (s + 1) & mask;
    }
    return nullptr;
  }
};

struct HashTable {
  std::vector<FlatMap> parts;
  const Batch* build = nullptr;
  std::vector<int> key_cols;
  bool skip_key_check = false;
};

void check_key_types(const Batch& probe, const std::vector<int>& pk, const Batch& build,
                     const std::vector<int>& bk) {
  if (pk.size() != bk.size() || pk.empty())
    fail(PRISM_ERR_INVALID_ARGUMENT, "probe and build key lists must be non-empty and equal length");
  for (size_t i = 0; i < pk.size(); ++i) {
    const Col& a = col_at(probe, pk[i]);
    const Col& b = col_at(build, bk[i]);
    bool sa = a.ty == T_UTF8 || a.ty == T_DICT, sb = b.ty == T_UTF8 || b.ty == T_DICT;
    if (a.ty != b.ty && !(sa && sb))
      fail(PRISM_ERR_SCHEMA_MISMATCH, "join key types differ between probe and build");
  }
}

// HashTable::build (hash_join.rs:87-141)
HashTable build_table(const Batch& build, const std::vector<int>& keys, int n_threads) {
  HashTable t;
  t.build = &build;
  t.key_cols = keys;
  for (int k : keys) col_at(build, k);
  int64_t n = build.rows;
  t.skip_key_check = keys.size() == 1 && build.cols[keys[0]]->ty == T_I64;
  // Step 1: hash every row (parallel)
  std::vector<uint64_t> hashes(n);
  int64_t nchunk = std::max<int64_t>(1, std::min<int64_t>(n_threads * 4, (n + 65535) / 65536));
  parallel_for(nchunk, n_threads, [&](int64_t c) {
    int64_t lo = n * c / nchunk, hi = n * (c + 1) / nchunk;
    if (t.skip_key_check) {
      const Col& kc = *build.cols[keys[0]];
      const int64_t* v = reinterpret_cast<const int64_t*>(kc.vals) + kc.off;
      for (int64_t i = lo; i < hi; ++i) hashes[i] = hash_i64_fast(v[i]);
    } else {
      for (int64_t i = lo; i < hi; ++i) hashes[i] = general_row_hash(build, keys, i);
    }
  });
  // Step 2: serial scatter into 64 partitions, row order preserved
  std::vector<std::vector<std::pair<uint64_t, uint32_t>>> part_rows(HASH_PARTITIONS);
  for (auto& p : part_rows) p.reserve(n / HASH_PARTITIONS + 1);
  for (int64_t i = 0; i < n; ++i)
    part_rows[hashes[i] & HASH_PART_MASK].push_back({hashes[i], (uint32_t)i});
  // Step 3: per-partition maps (parallel); rows appended in ascending order
  t.parts.resize(HASH_PARTITIONS);
  parallel_for(HASH_PARTITIONS, n_threads, [&](int64_t p) {
    FlatMap& m = t.parts[p];
    m.init(part_rows[p].size());
    for (auto& e : part_rows[p]) m.entry(e.first).push_back(e.second);
  });
  return t;
}

// HashTable::probe (hash_join.rs:143-200)
void probe_table(const HashTable& t, const Batch& probe, const std::vector<int>& keys,
                 std::vector<uint32_t>& pi, std::vector<uint32_t>& bi) {
  int64_t n = probe.rows;
  pi.clear();
  bi.clear();
  pi.reserve(n);
  bi.reserve(n);
  for (int k : keys) col_at(probe, k);
  if (t.skip_key_check && keys.size() == 1 && probe.cols[keys[0]]->ty == T_I64) {
    const Col& kc = *probe.cols[keys[0]];
    const int64_t* v = reinterpret_cast<const int64_t*>(kc.vals) + kc.off;
    for (int64_t r = 0; r < n; ++r) {
      uint64_t h = hash_i64_fast(v[r]);
      const auto* rows = t.parts[h & HASH_PART_MASK].get(h);
      if (rows)
        for (uint32_t b : *rows) { pi.push_back((uint32_t)r); bi.push_back(b); }
    }
    return;
  }
  for (int64_t r = 0; r < n; ++r) {
    uint64_t h = general_row_hash(probe, keys, r);
    const auto* rows = t.parts[h & HASH_PART_MASK].get(h);
    if (!rows) continue;
    for (uint32_t b : *rows)
      if (keys_equal(probe, keys, r, *t.build, t.key_cols, b)) {
        pi.push_back((uint32_t)r);
        bi.push_back(b);
      }
  }
}

std::string right_name(const Batch& probe, const std::string& nm) {
  for (auto& c : probe.cols)
    if (c->name == nm) return nm + "_right";
  return nm;
}

// assemble_joined_batch and its nullable variants (hash_join.rs:424-625)
Batch assemble(const Batch& probe, const std::vector<int64_t>& pidx, const Batch& build,
               const std::vector<int64_t>& bidx, int mode /*0 inner, 1 nullable probe, 2 both*/) {
  Batch out;
  out.rows = (int64_t)pidx.size();
  for (auto& c : probe.cols)
    out.cols.push_back(take_col(*c, pidx, c->name, mode == 0 ? c->nullable : true));
  for (auto& c : build.cols) {
    std::string nm = right_name(probe, c->name);
    bool nullable = c->nullable;
    if (mode == 2 && nm != c->name) nullable = true;
    out.cols.push_back(take_col(*c, bidx, nm, nullable));
  }
  return out;
}

Batch semi_anti(const Batch& probe, const std::vector<uint32_t>& pi, bool anti) {
  std::vector<uint8_t> m(probe.rows, 0);
  for (uint32_t p : pi) m[p] = 1;
  if (anti)
    for (auto& x : m) x = !x;
  Batch out;
  for (auto& c : probe.cols) out.cols.push_back(filter_col(*c, m));
  out.rows = 0;
  for (auto x : m) out.rows += x;
  return out;
}

std::vector<int64_t> widen(const std::vector<uint32_t>& v) { return std::vector<int64_t>(v.begin(), v.end()); }

// left_join_indices (hash_join.rs:455-483): unmatched probe rows pair with
// build index 0 (a non-null index, so they carry build row 0's values).
void left_indices(int64_t probe_rows, const std::vector<uint32_t>& pi,
                  const std::vector<uint32_t>& bi, std::vector<int64_t>& po,
                  std::vector<int64_t>& bo) {
  std::vector<uint8_t> matched(probe_rows, 0);
  po.assign(pi.begin(), pi.end());
  bo.assign(bi.begin(), bi.end());
  for (uint32_t p : pi) matched[p] = 1;
  for (int64_t r = 0; r < probe_rows; ++r)
    if (!matched[r]) { po.push_back(r); bo.push_back(0); }
}

Batch join_one(const Batch& probe, const Batch& build, const HashTable& t,
               const prism_join_config& cfg, const std::vector<int>& pk, bool chunked) {
  std::vector<uint32_t> pi, bi;
  probe_table(t, probe, pk, pi, bi);
  switch (cfg.join_type) {
    case PRISM_JOIN_INNER:
      return assemble(probe, widen(pi), build, widen(bi), 0);
    case PRISM_JOIN_LEFT: {
      std::vector<int64_t> po, bo;
      left_indices(probe.rows, pi, bi, po, bo);
      return assemble(probe, po, build, bo, 0);
    }
    case PRISM_JOIN_LEFT_SEMI: return semi_anti(probe, pi, false);
    case PRISM_JOIN_LEFT_ANTI: return semi_anti(probe, pi, true);
    case PRISM_JOIN_RIGHT: {
      if (chunked) return assemble(probe, widen(pi), build, widen(bi), 0);
      // right_join_indices (hash_join.rs:495-523)
      std::vector<int64_t> po(pi.begin(), pi.end()), bo(bi.begin(), bi.end());
      std::vector<uint8_t> bm(build.rows, 0);
      for (uint32_t b : bi) bm[b] = 1;
      for (int64_t r = 0; r < build.rows; ++r)
        if (!bm[r]) { po.push_back(-1); bo.push_back(r); }
      return assemble(probe, po, build, bo, 1);
    }
    case PRISM_JOIN_FULL: {
      if (chunked) return assemble(probe, widen(pi), build, widen(bi), 0);
      // full_join_indices (hash_join.rs:526-566)
      std::vector<int64_t> po(pi.begin(), pi.end()), bo(bi.begin(), bi.end());
      std::vector<uint8_t> pm(probe.rows, 0), bm(build.rows, 0);
      for (size_t i = 0; i < pi.size(); ++i) { pm[pi[i]] = 1; bm[bi[i]] = 1; }
      for (int64_t r = 0; r < probe.rows; ++r)
        if (!pm[r]) { po.push_back(r); bo.push_back(-1); }
      for (int64_t r = 0; r < build.rows; ++r)
        if (!bm[r]) { po.push_back(-1); bo.push_back(r); }
      return assemble(probe, po, build, bo, 2);
    }
    default:
      fail(PRISM_ERR_INVALID_ARGUMENT, "unknown join type");
  }
}

// ============================================================ aggregate ====
struct Acc {  // GroupAccumulator (hash_aggregate.rs:104-171)
  double sum = 0;
  uint64_t count = 0;
  double mn = std::numeric_limits<double>::infinity();
  double mx = -std::numeric_limits<double>::infinity();
  std::unique_ptr<std::unordered_set<std::string>> distinct;
  ExactSum* exact = nullptr;  // unused in reference mode
  __int128 dsum = 0;          // exact decimal sum (EXACT mode only)
  void accumulate(double v) {
    sum += v;
    count += 1;
    if (v < mn) mn = v;
    if (v > mx) mx = v;
  }
  void merge(const Acc& o) {
    sum += o.sum;
    count += o.count;
    if (o.mn < mn) mn = o.mn;
    if (o.mx > mx) mx = o.mx;
    dsum += o.dsum;
    if (distinct && o.distinct)
      for (auto& v : *o.distinct) distinct->insert(v);
  }
  double result(int func) const {
    switch (func) {
      case PRISM_AGG_SUM: return sum;
      case PRISM_AGG_COUNT: return (double)count;
      case PRISM_AGG_AVG: return count > 0 ? sum / (double)count : 0.0;
      case PRISM_AGG_MIN: return count > 0 ? mn : 0.0;
      case PRISM_AGG_MAX: return count > 0 ? mx : 0.0;
      case PRISM_AGG_COUNT_DISTINCT: return distinct ? (double)distinct->size() : 0.0;
    }
    return 0;
  }
};

// distinct_value (hash_aggregate.rs:457-481); encoded as tag + bytes.
bool distinct_value(const Col& c, int64_t row, std::string& out) {
  if (c.null_at(row)) return false;
  out.clear();
  switch (c.ty) {
    case T_I32: { int32_t v = (int32_t)c.ival(row); out = "i"; out.append((const char*)&v, 4); break; }
    case T_I64: { int64_t v = c.ival(row); out = "l"; out.append((const char*)&v, 8); break; }
    case T_F64: {
      double v = c.fval(row);
      uint64_t bits;
      if (v == 0.0) bits = 0;
      else if (std::isnan(v)) bits = 0x7ff8000000000000ULL;
      else std::memcpy(&bits, &v, 8);
      out = "g";
      out.append((const char*)&bits, 8);
      break;
    }
    case T_UTF8: case T_DICT: { out = "u"; auto s = c.sval(row); out.append(s.data(), s.size()); break; }
    case T_BOOL: out = c.ival(row) ? "b1" : "b0"; break;
    case T_DATE32: { int32_t v = (int32_t)c.ival(row); out = "d"; out.append((const char*)&v, 4); break; }
    case T_DEC128: { __int128 v = c.dval(row); out = "x"; out.append((const char*)&v, 16); break; }
    default: { int64_t v = c.ival(row); out = "f" + std::to_string((int)c.ty); out.append((const char*)&v, 8); }
  }
  return true;
}

struct GroupEntry {
  int64_t bi, ri;
  std::vector<Acc> accs;
};
struct Partial {
  std::unordered_map<uint64_t, GroupEntry> groups;
  std::vector<uint64_t> order;
};

bool is_dec_sum_exact(const Col& c, int func, bool exact_dec) {
  return exact_dec && c.ty == T_DEC128 && (func == PRISM_AGG_SUM || func == PRISM_AGG_AVG);
}

std::vector<Acc> new_accs(const prism_agg_config& cfg) {
  std::vector<Acc> a(cfg.n_aggs);
  for (int i = 0; i < cfg.n_aggs; ++i)
    if (cfg.aggs[i].func == PRISM_AGG_COUNT_DISTINCT)
      a[i].distinct = std::make_unique<std::unordered_set<std::string>>();
  return a;
}

Batch empty_result(const std::vector<ColP>& schema_cols, bool have_schema,
                   const prism_agg_config& cfg) {
  // build_empty_result (hash_aggregate.rs:506-527)
  Batch out;
  out.rows = 0;
  std::vector<ColP> fields = schema_cols;
  if (!have_schema) {  // hash_aggregate.rs:189-198: schema of the aggregate fields only
    fields.clear();
    for (int i = 0; i < cfg.n_aggs; ++i) {
      auto c = std::make_shared<Col>();
      int f = cfg.aggs[i].func;
      c->ty = (f == PRISM_AGG_COUNT || f == PRISM_AGG_COUNT_DISTINCT) ? T_I64 : T_F64;
      c->name = cfg.aggs[i].output_name ? cfg.aggs[i].output_name : "";
      fields.push_back(c);
    }
  }
  for (int g = 0; g < cfg.n_group_by; ++g) {
    int idx = cfg.group_by[g];
    if (idx < 0 || idx >= (int)fields.size()) fail(PRISM_ERR_INVALID_ARGUMENT, "group-by column out of range");
    Builder b = builder_like(*fields[idx], fields[idx]->name, fields[idx]->nullable);
    out.cols.push_back(b.finish());
  }
  for (int i = 0; i < cfg.n_aggs; ++i) {
    int f = cfg.aggs[i].func;
    Builder b((f == PRISM_AGG_COUNT || f == PRISM_AGG_COUNT_DISTINCT) ? T_I64 : T_F64,
              cfg.aggs[i].output_name ? cfg.aggs[i].output_name : "", true);
    out.cols.push_back(b.finish());
  }
  return out;
}

// global_aggregate_batches (hash_aggregate.rs:343-447)
Batch global_aggregate(const std::vector<Batch>& batches, const prism_agg_config& cfg) {
  Batch out;
  out.rows = 1;
  for (int a = 0; a < cfg.n_aggs; ++a) {
    const prism_agg_expr& ag = cfg.aggs[a];
    int f = ag.func;
    double result = 0;
    if (f == PRISM_AGG_COUNT) {
      uint64_t total = 0;
      for (auto& b : batches) {
        if (ag.column >= (int)b.cols.size()) total += b.rows;  // COUNT(*) on zero-column batch
        else {
          const Col& c = col_at(b, ag.column);
          uint64_t nn = 0;
          for (int64_t i = 0; i < c.len; ++i) nn += c.null_at(i) ? 0 : 1;
          total += nn;
        }
      }
      result = (double)total;
    } else if (f == PRISM_AGG_COUNT_DISTINCT) {
      std::unordered_set<std::string> s;
      std::string v;
      for (auto& b : batches) {
        const Col& c = col_at(b, ag.column);
        for (int64_t i = 0; i < c.len; ++i)
          if (distinct_value(c, i, v)) s.insert(v);
      }
      result = (double)s.size();
    } else {
      // arrow_agg::sum/min/max per batch over non-null values; the reference's
      // arrow kernel sums in SIMD lanes, an order this restatement does not
      // reproduce (sequential here), so SUM/AVG parity is to tolerance.
      std::vector<double> psum, pmin, pmax;
      uint64_t cnt = 0;
      for (auto& b : batches) {
        if (b.rows == 0) continue;
        const Col& c = col_at(b, ag.column);
        F64Col v = cast_f64(c, "aggregate");
        double s = 0;
        bool any = false;
        double mn = std::numeric_limits<double>::infinity(), mx = -mn;
        for (int64_t i = 0; i < c.len; ++i) {
          if (!v.valid[i]) continue;
          any = true;
          s += v.v[i];
          ++cnt;
          if (!std::isnan(v.v[i])) { mn = std::min(mn, v.v[i]); mx = std::max(mx, v.v[i]); }
        }
        psum.push_back(any ? s : 0.0);
        if (any) { pmin.push_back(mn); pmax.push_back(mx); }
      }
      if (f == PRISM_AGG_SUM || f == PRISM_AGG_AVG) {
        double t = 0;
        for (double x : psum) t += x;
        result = f == PRISM_AGG_SUM ? t : (cnt > 0 ? t / (double)cnt : 0.0);
      } else if (f == PRISM_AGG_MIN) {
        double m = std::numeric_limits<double>::infinity();
        for (double x : pmin) m = std::fmin(m, x);
        result = std::isinf(m) && m > 0 ? 0.0 : m;
      } else if (f == PRISM_AGG_MAX) {
        double m = -std::numeric_limits<double>::infinity();
        for (double x : pmax) m = std::fmax(m, x);
        result = std::isinf(m) && m < 0 ? 0.0 : m;
      } else {
        fail(PRISM_ERR_UNSUPPORTED_AGGREGATION, "unknown aggregate function");
      }
    }
    bool is_int = f == PRISM_AGG_COUNT || f == PRISM_AGG_COUNT_DISTINCT;
    Builder bb(is_int ? T_I64 : T_F64, ag.output_name ? ag.output_name : "", true);
    if (is_int) bb.push_i64((int64_t)result);
    else bb.push_f64(result);
    out.cols.push_back(bb.finish());
  }
  return out;
}

// hash_aggregate_batches (hash_aggregate.rs:182-339). exact_dec: Decimal128
// SUM/AVG inputs accumulate exactly in 128-bit (EXACT arithmetic mode).
Batch aggregate_batches(const std::vector<Batch>& batches, const std::vector<ColP>& schema_cols,
                        const prism_agg_config& cfg, int n_threads, bool exact_dec) {
  for (int i = 0; i < cfg.n_aggs; ++i)
    if (cfg.aggs[i].func < 0 || cfg.aggs[i].func > PRISM_AGG_COUNT_DISTINCT)
      fail(PRISM_ERR_UNSUPPORTED_AGGREGATION, "unknown aggregate function");
  bool any_rows = false;
  for (auto& b : batches) any_rows |= b.rows > 0;
  if (cfg.n_group_by == 0 && any_rows && !exact_dec) return global_aggregate(batches, cfg);
  if (!any_rows) return empty_result(schema_cols, !batches.empty(), cfg);

  std::vector<int> gb(cfg.group_by, cfg.group_by + cfg.n_group_by);
  std::vector<std::pair<int64_t, const Batch*>> non_empty;
  for (size_t i = 0; i < batches.size(); ++i)
    if (batches[i].rows > 0) non_empty.push_back({(int64_t)i, &batches[i]});
  const Batch& ref = *non_empty[0].second;
  for (int g : gb) col_at(ref, g);
  for (int i = 0; i < cfg.n_aggs; ++i) col_at(ref, cfg.aggs[i].column);

  int64_t chunk = std::max<int64_t>(1, (int64_t)non_empty.size() / std::max(1, n_threads));
  int64_t n_chunks = ((int64_t)non_empty.size() + chunk - 1) / chunk;
  std::vector<Partial> partials(n_chunks);
  parallel_for(n_chunks, n_threads, [&](int64_t ci) {
    Partial& P = partials[ci];
    int64_t lo = ci * chunk, hi = std::min<int64_t>((int64_t)non_empty.size(), lo + chunk);
    for (int64_t k = lo; k < hi; ++k) {
      int64_t batch_idx = non_empty[k].first;
      const Batch& b = *non_empty[k].second;
      std::vector<F64Col> vals(cfg.n_aggs);
      for (int a = 0; a < cfg.n_aggs; ++a) {
        int f = cfg.aggs[a].func;
        const Col& c = col_at(b, cfg.aggs[a].column);
        if (f == PRISM_AGG_COUNT_DISTINCT) continue;
        if (f == PRISM_AGG_COUNT && (c.ty == T_UTF8 || c.ty == T_DICT || c.ty == T_DATE32)) {
          vals[a].v.assign(c.len, 0.0);  // values unused by COUNT
          continue;
        }
        if (c.ty == T_UTF8 || c.ty == T_DICT || c.ty == T_DATE32)
          fail(PRISM_ERR_UNSUPPORTED_AGGREGATION,
               "numeric aggregate over a non-numeric column '" + c.name + "'");
        vals[a] = cast_f64(c, "aggregate");
      }
      std::string dv;
      for (int64_t row = 0; row < b.rows; ++row) {
        uint64_t gh = hash_group_keys(b, gb, row);
        auto it = P.groups.find(gh);
        if (it == P.groups.end()) {
          P.order.push_back(gh);
          it = P.groups.emplace(gh, GroupEntry{batch_idx, row, new_accs(cfg)}).first;
        }
        auto& accs = it->second.accs;
        for (int a = 0; a < cfg.n_aggs; ++a) {
          int f = cfg.aggs[a].func;
          const Col& c = *b.cols[cfg.aggs[a].column];
          if (f == PRISM_AGG_COUNT_DISTINCT) {
            if (distinct_value(c, row, dv)) accs[a].distinct->insert(dv);
            continue;
          }
          accs[a].accumulate(vals[a].v[row]);
          if (is_dec_sum_exact(c, f, exact_dec)) accs[a].dsum += c.dval(row);
        }
      }
    }
  });
  // merge partial maps in chunk order (hash_aggregate.rs:276-296)
  std::unordered_map<uint64_t, GroupEntry> groups;
  std::vector<uint64_t> order;
  for (auto& P : partials) {
    for (uint64_t gh : P.order) {
      auto& src = P.groups.at(gh);
      auto it = groups.find(gh);
      if (it == groups.end()) {
        order.push_back(gh);
        it = groups.emplace(gh, GroupEntry{src.bi, src.ri, new_accs(cfg)}).first;
      }
      for (int a = 0; a < cfg.n_aggs; ++a) it->second.accs[a].merge(src.accs[a]);
    }
  }
  // output (hash_aggregate.rs:298-338)
  Batch out;
  out.rows = (int64_t)order.size();
  for (int g : gb) {
    const Col& rc = *ref.cols[g];
    if (rc.ty == T_DICT) {
      // first-row values, re-encoded against one dictionary of the distinct
      // decoded values in output order
      Builder dv(T_UTF8, "", true);
      std::map<std::string, int64_t> seen;
      Builder ib(T_DICT, rc.name, rc.nullable);
      ib.idx_ty = rc.idx_ty;
      for (uint64_t gh : order) {
        auto& e = groups.at(gh);
        const Col& c = *batches[e.bi].cols[g];
        if (c.null_at(e.ri)) { ib.push_null(); continue; }
        std::string s(c.sval(e.ri));
        auto it = seen.find(s);
        if (it == seen.end()) {
          it = seen.emplace(s, (int64_t)seen.size()).first;
          dv.push_str(s);
        }
        ib.push_i64(it->second);
      }
      ib.dict = dv.finish();
      out.cols.push_back(ib.finish());
      continue;
    }
    Builder b = builder_like(rc, rc.name, rc.nullable);
    for (uint64_t gh : order) {
      auto& e = groups.at(gh);
      b.push_from(*batches[e.bi].cols[g], e.ri);
    }
    out.cols.push_back(b.finish());
  }
  for (int a = 0; a < cfg.n_aggs; ++a) {
    int f = cfg.aggs[a].func;
    const Col& src = *ref.cols[cfg.aggs[a].column];
    std::string nm = cfg.aggs[a].output_name ? cfg.aggs[a].output_name : "";
    if (is_dec_sum_exact(src, f, exact_dec) && f == PRISM_AGG_SUM) {
      Builder b(T_DEC128, nm, true);
      b.prec = 38;
      b.scale = src.scale;
      for (uint64_t gh : order) b.push_i128(groups.at(gh).accs[a].dsum);
      out.cols.push_back(b.finish());
      continue;
    }
    bool is_int = f == PRISM_AGG_COUNT || f == PRISM_AGG_COUNT_DISTINCT;
    Builder b(is_int ? T_I64 : T_F64, nm, true);
    for (uint64_t gh : order) {
      const Acc& acc = groups.at(gh).accs[a];
      if (is_dec_sum_exact(src, f, exact_dec)) {  // exact AVG: ((double)sum / 10^s) / count
        double p = 1.0;
        for (int k = 0; k < src.scale; ++k) p *= 10.0;
        b.push_f64(acc.count ? ((double)acc.dsum / p) / (double)acc.count : 0.0);
        continue;
      }
      double r = acc.result(f);
      if (is_int) b.push_i64((int64_t)r);
      else b.push_f64(r);
    }
    out.cols.push_back(b.finish());
  }
  return out;
}

// ====================================================== filter/project ====
struct BoolCol {
  std::vector<uint8_t> val, valid;
};

// total-order key of a double (IEEE 754 totalOrder), as arrow-ord compares floats
int64_t total_key(double d) {
  int64_t i;
  std::memcpy(&i, &d, 8);
  i ^= (int64_t)(((uint64_t)(i >> 63)) >> 1);
  return i;
}

template <class T>
bool cmp_op(int op, const T& a, const T& b) {
  switch (op) {
    case PRISM_PRED_EQ: return a == b;
    case PRISM_PRED_NE: return a != b;
    case PRISM_PRED_LT: return a < b;
    case PRISM_PRED_LE: return a <= b;
    case PRISM_PRED_GT: return a > b;
    case PRISM_PRED_GE: return a >= b;
  }
  return false;
}

// SQL LIKE over bytes: '%' any run, '_' one character (one UTF-8 code point),
// '\\' escapes the next character (arrow-string like semantics).
bool like_match(std::string_view s, std::string_view p, bool ci) {
  auto lower = [&](unsigned char c) -> unsigned char { return ci && c >= 'A' && c <= 'Z' ? c + 32 : c; };
  auto cplen = [](unsigned char c) -> size_t {
    if (c < 0x80) return 1;
    if ((c >> 5) == 6) return 2;
    if ((c >> 4) == 14) return 3;
    return 4;
  };
  // iterative matcher with backtracking on the last '%'
  size_t si = 0, pi = 0, star_p = std::string_view::npos, star_s = 0;
  while (si < s.size()) {
    if (pi < p.size()) {
      unsigned char pc = p[pi];
      if (pc == '%') { star_p = ++pi; star_s = si; continue; }
      if (pc == '_') { si += cplen((unsigned char)s[si]); ++pi; continue; }
      if (pc == '\\' && pi + 1 < p.size()) {
        if (lower((unsigned char)s[si]) == lower((unsigned char)p[pi + 1])) { ++si; pi += 2; continue; }
      } else if (lower((unsigned char)s[si]) == lower(pc)) { ++si; ++pi; continue; }
    }
    if (star_p != std::string_view::npos) {
      star_s += cplen((unsigned char)s[star_s]);
      si = star_s;
      pi = star_p;
      continue;
    }
    return false;
  }
  while (pi < p.size() && p[pi] == '%') ++pi;
  return pi == p.size();
}

BoolCol eval_pred_range(const Batch& b, const prism_pred_node* nodes, int n) {
  std::vector<BoolCol> st;
  int64_t R = b.rows;
  for (int k = 0; k < n; ++k) {
    const prism_pred_node& nd = nodes[k];
    BoolCol r;
    r.val.assign(R, 0);
    r.valid.assign(R, 1);
    switch (nd.op) {
      case PRISM_PRED_LITERAL:
        std::fill(r.val.begin(), r.val.end(), nd.value.i64 ? 1 : 0);
        break;
      case PRISM_PRED_EQ: case PRISM_PRED_NE: case PRISM_PRED_LT: case PRISM_PRED_LE:
      case PRISM_PRED_GT: case PRISM_PRED_GE: {
        // compare_column (filter_project.rs:346-392): supported type pairs only
        const Col& c = col_at(b, nd.column);
        int st_ = nd.value.type;
        bool ok = (c.ty == T_I32 && st_ == PRISM_SCALAR_INT32) ||
                  (c.ty == T_I64 && st_ == PRISM_SCALAR_INT64) ||
                  (c.ty == T_F64 && st_ == PRISM_SCALAR_FLOAT64) ||
                  (c.ty == T_UTF8 && st_ == PRISM_SCALAR_UTF8) ||
                  (c.ty == T_DATE32 && (st_ == PRISM_SCALAR_DATE32 || st_ == PRISM_SCALAR_INT32));
        if (!ok) fail(PRISM_ERR_INVALID_ARGUMENT, "Cannot compare column type with scalar");
        std::string_view lit(nd.value.str ? nd.value.str : "", (size_t)nd.value.str_len);
        for (int64_t i = 0; i < R; ++i) {
          r.valid[i] = !c.null_at(i);
          bool v;
          if (c.ty == T_F64) v = cmp_op(nd.op, total_key(c.fval(i)), total_key(nd.value.f64));
          else if (c.ty == T_UTF8) v = cmp_op(nd.op, c.sval(i), lit);
          else v = cmp_op(nd.op, c.ival(i), nd.value.i64);
          r.val[i] = v;
        }
        break;
      }
      case PRISM_PRED_IS_NULL: case PRISM_PRED_IS_NOT_NULL: {
        const Col& c = col_at(b, nd.column);
        for (int64_t i = 0; i < R; ++i) r.val[i] = (c.null_at(i) == (nd.op == PRISM_PRED_IS_NULL));
        break;
      }
      case PRISM_PRED_LIKE: case PRISM_PRED_ILIKE: {
        const Col& c = col_at(b, nd.column);
        if (c.ty != T_UTF8) fail(PRISM_ERR_INVALID_ARGUMENT, "LIKE requires Utf8 column");
        std::string_view pat(nd.value.str ? nd.value.str : "", (size_t)nd.value.str_len);
        for (int64_t i = 0; i < R; ++i) {
          r.valid[i] = !c.null_at(i);
          r.val[i] = like_match(c.sval(i), pat, nd.op == PRISM_PRED_ILIKE);
        }
        break;
      }
      case PRISM_PRED_AND: case PRISM_PRED_OR: {
        // arrow compute::and / or: null if either side is null
        if (st.size() < 2) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed predicate");
        BoolCol rr = std::move(st.back()); st.pop_back();
        BoolCol ll = std::move(st.back()); st.pop_back();
        for (int64_t i = 0; i < R; ++i) {
          r.valid[i] = ll.valid[i] && rr.valid[i];
          r.val[i] = nd.op == PRISM_PRED_AND ? (ll.val[i] && rr.val[i]) : (ll.val[i] || rr.val[i]);
        }
        break;
      }
      case PRISM_PRED_NOT: {
        if (st.empty()) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed predicate");
        BoolCol x = std::move(st.back()); st.pop_back();
        for (int64_t i = 0; i < R; ++i) { r.valid[i] = x.valid[i]; r.val[i] = !x.val[i]; }
        break;
      }
      default:
        fail(PRISM_ERR_INVALID_ARGUMENT, "unknown predicate op");
    }
    st.push_back(std::move(r));
  }
  if (st.size() != 1) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed predicate");
  return std::move(st.back());
}

ColP bool_to_col(const BoolCol& m, const std::string& name) {
  Builder b(T_BOOL, name, true);
  for (size_t i = 0; i < m.val.size(); ++i) {
    if (!m.valid[i]) b.push_null();
    else b.push_i64(m.val[i]);
  }
  return b.finish();
}

std::vector<uint8_t> keep_of(const BoolCol& m) {
  std::vector<uint8_t> k(m.val.size());
  for (size_t i = 0; i < k.size(); ++i) k[i] = m.val[i] && m.valid[i];
  return k;
}

Batch filter_by(const Batch& b, const std::vector<uint8_t>& keep) {
  Batch out;
  out.rows = 0;
  for (auto x : keep) out.rows += x;
  for (auto& c : b.cols) out.cols.push_back(filter_col(*c, keep));
  return out;
}

Batch project(const Batch& b, const int32_t* cols, int n) {
  Batch out;
  out.rows = b.rows;
  for (int i = 0; i < n; ++i) out.cols.push_back(b.cols.at(col_at(b, cols[i]).len >= 0 ? cols[i] : 0));
  return out;
}

ColP literal_col(const prism_scalar& s, int64_t n) {
  switch (s.type) {
    case PRISM_SCALAR_FLOAT64: { Builder b(T_F64, "", true); for (int64_t i = 0; i < n; ++i) b.push_f64(s.f64); return b.finish(); }
    case PRISM_SCALAR_INT64: { Builder b(T_I64, "", true); for (int64_t i = 0; i < n; ++i) b.push_i64(s.i64); return b.finish(); }
    case PRISM_SCALAR_INT32: { Builder b(T_I32, "", true); for (int64_t i = 0; i < n; ++i) b.push_i64(s.i64); return b.finish(); }
    case PRISM_SCALAR_DATE32: { Builder b(T_DATE32, "", true); for (int64_t i = 0; i < n; ++i) b.push_i64(s.i64); return b.finish(); }
    case PRISM_SCALAR_BOOLEAN: { Builder b(T_BOOL, "", true); for (int64_t i = 0; i < n; ++i) b.push_i64(s.i64 ? 1 : 0); return b.finish(); }
    case PRISM_SCALAR_UTF8: {
      Builder b(T_UTF8, "", true);
      std::string_view v(s.str ? s.str : "", (size_t)s.str_len);
      for (int64_t i = 0; i < n; ++i) b.push_str(v);
      return b.finish();
    }
  }
  fail(PRISM_ERR_INVALID_ARGUMENT, "unknown scalar type");
}

// Cast for IfThen branch alignment (filter_project.rs:296-302): identical
// types pass through; numeric <-> numeric follow arrow's safe cast (float to
// integer truncates toward zero, out of range becomes null).
ColP cast_to(const ColP& c, const Col& target) {
  if (c->ty == target.ty && c->scale == target.scale) return c;
  bool num_src = is_int_like(c->ty) || c->ty == T_F64 || c->ty == T_F32 || c->ty == T_BOOL || c->ty == T_DEC128;
  bool num_dst = (is_int_like(target.ty) && target.ty != T_DATE32) || target.ty == T_F64;
  if (c->ty == T_NULL) {
    Builder b = builder_like(target, "", true);
    for (int64_t i = 0; i < c->len; ++i) b.push_null();
    return b.finish();
  }
  if (!num_src || !num_dst || c->ty == T_DATE32)
    fail(PRISM_ERR_ARROW, "Cast error: unsupported cast in IfThen branch");
  Builder b = builder_like(target, "", true);
  for (int64_t i = 0; i < c->len; ++i) {
    if (c->null_at(i)) { b.push_null(); continue; }
    if (target.ty == T_F64) { b.push_f64(c->fval(i)); continue; }
    double d = c->fval(i);
    if (c->ty == T_F64 || c->ty == T_F32 || c->ty == T_DEC128) {
      double t = std::trunc(d);
      if (!(t >= -9.223372036854775808e18 && t < 9.223372036854775808e18)) { b.push_null(); continue; }
      b.push_i64((int64_t)t);
    } else {
      b.push_i64(c->ival(i));
    }
  }
  return b.finish();
}

__int128 pow10_i128(int s) {
  __int128 p = 1;
  for (int i = 0; i < s; ++i) p *= 10;
  return p;
}

bool exactable(const Col& c) {
  return (is_int_like(c.ty) && c.ty != T_DATE32) || c.ty == T_DEC128 || c.ty == T_BOOL;
}
// exact value of row i; a null row of an integer column reads 0 and a
// Decimal128 keeps its raw slot, as the Float64 cast above treats them
__int128 exact_val(const Col& c, int64_t i) {
  if (c.ty == T_DEC128) return c.dval(i);
  if (c.null_at(i)) return 0;
  if (c.ty == T_U64) return (__int128)(uint64_t)c.ival(i);
  return (__int128)c.ival(i);
}

ColP eval_expr(const Batch& b, const prism_expr& e, int mode);

ColP eval_expr_range(const Batch& b, const prism_expr& e, int begin, int end, int mode) {
  std::vector<ColP> st;
  int64_t R = b.rows;
  for (int k = begin; k < end; ++k) {
    const prism_expr_node& nd = e.nodes[k];
    switch (nd.op) {
      case PRISM_EXPR_COLUMN:
        st.push_back(b.cols.at(col_at(b, nd.column).len >= 0 ? nd.column : 0));
        break;
      case PRISM_EXPR_LITERAL:
        st.push_back(literal_col(nd.literal, R));
        break;
      case PRISM_EXPR_ADD: case PRISM_EXPR_SUB: case PRISM_EXPR_MUL: case PRISM_EXPR_DIV: {
        if (st.size() < 2) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed expression");
        ColP r = st.back(); st.pop_back();
        ColP l = st.back(); st.pop_back();
        if (mode == PRISM_ARITH_EXACT && nd.op != PRISM_EXPR_DIV && exactable(*l) && exactable(*r)) {
          int sl = l->ty == T_DEC128 ? l->scale : 0, sr = r->ty == T_DEC128 ? r->scale : 0;
          int so = nd.op == PRISM_EXPR_MUL ? sl + sr : std::max(sl, sr);
          if (so > 38) fail(PRISM_ERR_EXECUTION, "decimal scale exceeds 38");
          Builder ob(T_DEC128, "", true);
          ob.prec = 38;
          ob.scale = so;
          __int128 fl = pow10_i128(so - sl), fr = pow10_i128(so - sr);
          for (int64_t i = 0; i < R; ++i) {
            // null rows carry the wrapped (mod 2^128) result of the raw
            // slots and never raise
            bool valid = !l->null_at(i) && !r->null_at(i);
            __int128 a = exact_val(*l, i), c = exact_val(*r, i), out;
            bool ovf = false;
            if (nd.op == PRISM_EXPR_MUL) ovf = __builtin_mul_overflow(a, c, &out);
            else {
              __int128 aa, cc;
              ovf = __builtin_mul_overflow(a, fl, &aa);
              ovf = __builtin_mul_overflow(c, fr, &cc) || ovf;
              ovf = (nd.op == PRISM_EXPR_ADD ? __builtin_add_overflow(aa, cc, &out)
                                             : __builtin_sub_overflow(aa, cc, &out)) || ovf;
            }
            if (!valid) { ob.push_raw_null(&out, 16); continue; }
            if (ovf) fail(PRISM_ERR_EXECUTION, "decimal overflow in exact arithmetic");
            ob.push_i128(out);
          }
          st.push_back(ob.finish());
          break;
        }
        // filter_project.rs:233-247: cast both to Float64, IEEE arithmetic
        F64Col lv = cast_f64(*l, "arithmetic"), rv = cast_f64(*r, "arithmetic");
        Builder ob(T_F64, "", true);
        // arrow-arith applies float ops to every slot (binary), so a null
        // row holds the result of its raw operand slots
        for (int64_t i = 0; i < R; ++i) {
          double a = lv.v[i], c = rv.v[i], o = 0;
          switch (nd.op) {
            case PRISM_EXPR_ADD: o = a + c; break;
            case PRISM_EXPR_SUB: o = a - c; break;
            case PRISM_EXPR_MUL: o = a * c; break;
            case PRISM_EXPR_DIV: o = a / c; break;
          }
          if (!lv.valid[i] || !rv.valid[i]) ob.push_raw_null(&o, 8);
          else ob.push_f64(o);
        }
        st.push_back(ob.finish());
        break;
      }
      case PRISM_EXPR_NEG: {
        if (st.empty()) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed expression");
        ColP x = st.back(); st.pop_back();
        if (mode == PRISM_ARITH_EXACT && exactable(*x)) {
          Builder ob(T_DEC128, "", true);
          ob.prec = 38;
          ob.scale = x->ty == T_DEC128 ? x->scale : 0;
          for (int64_t i = 0; i < R; ++i) {
            __int128 v = (__int128)((unsigned __int128)0 - (unsigned __int128)exact_val(*x, i));
            if (x->null_at(i)) ob.push_raw_null(&v, 16);
            else ob.push_i128(v);
          }
          st.push_back(ob.finish());
          break;
        }
        F64Col v = cast_f64(*x, "negation");
        Builder ob(T_F64, "", true);
        for (int64_t i = 0; i < R; ++i) {
          double o = -v.v[i];
          if (!v.valid[i]) ob.push_raw_null(&o, 8);
          else ob.push_f64(o);
        }
        st.push_back(ob.finish());
        break;
      }
      case PRISM_EXPR_IF_THEN: {
        int nc = nd.n_clauses;
        int need = nc + (nd.has_else ? 1 : 0);
        if ((int)st.size() < need) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed expression");
        std::vector<ColP> branches(st.end() - need, st.end() - (nd.has_else ? 1 : 0));
        ColP else_c = nd.has_else ? st.back() : nullptr;
        st.resize(st.size() - need);
        if (nc == 0) {
          if (!else_c) fail(PRISM_ERR_INVALID_ARGUMENT,
                            "IfThen expression requires at least one clause or an else branch");
          st.push_back(else_c);
          break;
        }
        const Col& target = *branches[0];
        ColP result;
        if (else_c) result = cast_to(else_c, target);
        else {
          Builder nb = builder_like(target, "", true);
          for (int64_t i = 0; i < R; ++i) nb.push_null();
          result = nb.finish();
        }
        for (int ci = nc - 1; ci >= 0; --ci) {
          const prism_expr_clause& cl = e.clauses[nd.clause_begin + ci];
          BoolCol m = eval_pred_range(b, e.preds + cl.pred_begin, cl.pred_len);
          ColP br = cast_to(branches[ci], target);
          Builder zb = builder_like(target, "", true);
          for (int64_t i = 0; i < R; ++i) {
            if (m.valid[i] && m.val[i]) zb.push_slot(*br, i);
            else zb.push_slot(*result, i);
          }
          result = zb.finish();
        }
        st.push_back(result);
        break;
      }
      default:
        fail(PRISM_ERR_INVALID_ARGUMENT, "unknown expression op");
    }
  }
  if (st.size() != 1) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed expression");
  return st.back();
}

ColP eval_expr(const Batch& b, const prism_expr& e, int mode) {
  return eval_expr_range(b, e, 0, e.n_nodes, mode);
}

Batch project_exprs(const Batch& b, const int32_t* cols, int n_cols, const prism_expr* exprs,
                    int n_exprs, int mode) {
  Batch out;
  out.rows = b.rows;
  for (int i = 0; i < n_cols; ++i) {
    col_at(b, cols[i]);
    out.cols.push_back(b.cols[cols[i]]);
  }
  for (int i = 0; i < n_exprs; ++i) {
    ColP c = eval_expr(b, exprs[i], mode);
    auto named = std::make_shared<Col>(*c);
    named->name = "expr_" + std::to_string(i);
    named->nullable = true;
    out.cols.push_back(named);
  }
  return out;
}

std::vector<ColP> schema_cols_of(const ArrowSchema* s) {
  // zero-row view of a schema, for empty results
  std::vector<ColP> cols;
  if (!s) return cols;
  for (int64_t i = 0; i < s->n_children; ++i) {
    auto c = std::make_shared<Col>();
    const ArrowSchema* ch = s->children[i];
    Ty t;
    int p = 38, sc = 0;
    if (!parse_format(ch->format, t, p, sc)) fail(PRISM_ERR_ARROW, "unsupported format");
    c->ty = ch->dictionary ? T_DICT : t;
    if (ch->dictionary) {
      c->idx_ty = t;
      c->dict = std::make_shared<Col>();
      Ty dt;
      parse_format(ch->dictionary->format, dt, p, sc);
      c->dict->ty = dt;
    }
    c->prec = p;
    c->scale = sc;
    c->name = ch->name ? ch->name : "";
    c->nullable = (ch->flags & ARROW_FLAG_NULLABLE) != 0;
    cols.push_back(c);
  }
  return cols;
}

// ================================================= fused join -> aggregate =
// executor.rs:333-458 with project_join_matches (:474-551),
// expand_worker_aggregates (:684-712), build_final_merge_config (:714-743),
// reconstruct_original_aggregate_batch (:745-812).
Batch join_aggregate(const std::vector<Batch>& probes, const Batch& build,
                     const std::vector<int>& pk, const std::vector<int>& bk, const int32_t* cols,
                     int n_cols, const prism_expr* exprs, int n_exprs,
                     const prism_agg_config& agg, int n_threads) {
  // worker aggregates: AVG -> SUM + COUNT
  std::vector<prism_agg_expr> worker;
  std::vector<std::vector<int>> mapping;
  std::vector<std::string> wnames;
  for (int i = 0; i < agg.n_aggs; ++i) {
    const prism_agg_expr& a = agg.aggs[i];
    if (a.func == PRISM_AGG_AVG) {
      mapping.push_back({(int)worker.size(), (int)worker.size() + 1});
      worker.push_back({a.column, PRISM_AGG_SUM, nullptr});
      worker.push_back({a.column, PRISM_AGG_COUNT, nullptr});
    } else {
      mapping.push_back({(int)worker.size()});
      worker.push_back({a.column, a.func, nullptr});
    }
  }
  for (size_t i = 0; i < worker.size(); ++i) wnames.push_back("agg_" + std::to_string(i));
  for (size_t i = 0; i < worker.size(); ++i) worker[i].output_name = wnames[i].c_str();
  prism_agg_config wcfg{agg.n_group_by, agg.group_by, (int32_t)worker.size(), worker.data()};

  if (probes.empty()) fail(PRISM_ERR_INVALID_ARGUMENT, "no probe batches");
  HashTable t = build_table(build, bk, n_threads);
  std::vector<std::vector<uint32_t>> mp(probes.size()), mb(probes.size());
  parallel_for((int64_t)probes.size(), n_threads,
               [&](int64_t i) { probe_table(t, probes[i], pk, mp[i], mb[i]); });

  std::vector<Batch> partials;
  int n_probe_cols = (int)probes[0].cols.size();
  Batch empty_projected;  // probe batch 0 joined with no rows
  for (size_t bi = 0; bi < probes.size(); ++bi) {
    if (mp[bi].empty() && bi != 0) continue;
    // project_join_matches: take referenced joined columns, evaluate exprs
    Batch joined;
    joined.rows = (int64_t)mp[bi].size();
    std::vector<int64_t> pidx = widen(mp[bi]), bidx = widen(mb[bi]);
    int total_cols = n_probe_cols + (int)build.cols.size();
    joined.cols.resize(total_cols);
    auto need = [&](int c) {
      if (c < 0 || c >= total_cols) fail(PRISM_ERR_INVALID_ARGUMENT, "joined column out of range");
      if (joined.cols[c]) return;
      if (c < n_probe_cols) {
        const Col& pc = *probes[bi].cols[c];
        joined.cols[c] = take_col(pc, pidx, pc.name, pc.nullable);
      } else {
        const Col& bc = *build.cols[c - n_probe_cols];
        joined.cols[c] = take_col(bc, bidx, right_name(probes[bi], bc.name), bc.nullable);
      }
    };
    for (int i = 0; i < n_cols; ++i) need(cols[i]);
    for (int e = 0; e < n_exprs; ++e) {
      for (int k = 0; k < exprs[e].n_nodes; ++k)
        if (exprs[e].nodes[k].op == PRISM_EXPR_COLUMN) need(exprs[e].nodes[k].column);
      for (int k = 0; k < exprs[e].n_preds; ++k) {
        int op = exprs[e].preds[k].op;
        if (op != PRISM_PRED_LITERAL && op != PRISM_PRED_AND && op != PRISM_PRED_OR && op != PRISM_PRED_NOT)
          need(exprs[e].preds[k].column);
      }
    }
    for (int c = 0; c < total_cols; ++c)
      if (!joined.cols[c]) {  // placeholder (never read)
        auto z = std::make_shared<Col>();
        z->ty = T_NULL;
        z->len = joined.rows;
        joined.cols[c] = z;
      }
    Batch projected = project_exprs(joined, cols, n_cols, exprs, n_exprs, PRISM_ARITH_F64);
    if (projected.rows == 0) {
      if (bi == 0) empty_projected = projected;
      continue;
    }
    partials.push_back(aggregate_batches({projected}, projected.cols, wcfg, 1, false));
  }
  // final merge config: SUM for SUM/COUNT/COUNT_DISTINCT, MIN, MAX
  std::vector<int32_t> mgb(agg.n_group_by);
  for (int i = 0; i < agg.n_group_by; ++i) mgb[i] = i;
  std::vector<prism_agg_expr> merge;
  for (size_t i = 0; i < worker.size(); ++i) {
    int f = worker[i].func;
    int mf = (f == PRISM_AGG_MIN || f == PRISM_AGG_MAX) ? f : PRISM_AGG_SUM;
    merge.push_back({agg.n_group_by + (int)i, mf, wnames[i].c_str()});
  }
  prism_agg_config mcfg{agg.n_group_by, mgb.data(), (int32_t)merge.size(), merge.data()};
  Batch merged;
  if (partials.empty()) {
    // no matches: the fused executor declines (executor.rs:444-446) and the
    // unfused plan aggregates the empty projected join output, which
    // hash_aggregate answers with its empty result (group and aggregate
    // fields, hash_aggregate.rs:188-203, 506-525)
    return aggregate_batches({empty_projected}, empty_projected.cols, agg, 1, false);
  }
  merged = aggregate_batches(partials, partials[0].cols, mcfg, n_threads, false);
  // reconstruct
  Batch out;
  out.rows = merged.rows;
  for (int i = 0; i < agg.n_group_by; ++i) out.cols.push_back(merged.cols[i]);
  for (int i = 0; i < agg.n_aggs; ++i) {
    const prism_agg_expr& a = agg.aggs[i];
    const Col& src = *merged.cols[agg.n_group_by + mapping[i][0]];
    std::string nm = a.output_name ? a.output_name : "";
    if (a.func == PRISM_AGG_COUNT || a.func == PRISM_AGG_COUNT_DISTINCT) {
      Builder b(T_I64, nm, true);
      for (int64_t r = 0; r < merged.rows; ++r) b.push_i64(src.null_at(r) ? 0 : (int64_t)src.fval(r));
      out.cols.push_back(b.finish());
    } else if (a.func == PRISM_AGG_AVG) {
      const Col& cnt = *merged.cols[agg.n_group_by + mapping[i][1]];
      Builder b(T_F64, nm, true);
      for (int64_t r = 0; r < merged.rows; ++r) {
        double s = src.null_at(r) ? 0 : src.fval(r), c = cnt.null_at(r) ? 0 : cnt.fval(r);
        b.push_f64(c > 0 ? s / c : 0.0);
      }
      out.cols.push_back(b.finish());
    } else {
      Builder b(T_F64, nm, true);
      for (int64_t r = 0; r < merged.rows; ++r) b.push_f64(src.null_at(r) ? 0 : src.fval(r));
      out.cols.push_back(b.finish());
    }
  }
  return out;
}

// ================================================================ sort ====
// sort_batch / sort_batch_limit (sort.rs:35-78): arrow-ord's
// lexsort_to_indices with each key's SortOptions, then take. Per key: two
// nulls are equal; a null sorts before a value with nulls_first, after it
// otherwise, whatever the direction; values compare ascending, reversed for
// descending. Value order (arrow-ord compare): integers numerically, floats
// by total_cmp (IEEE totalOrder), Boolean false < true, Utf8 (and a
// dictionary's decoded values) bytewise then by length, Decimal128
// numerically. The reference's sort is unstable (sort_unstable_by, with a
// partial sort under a limit); this restatement is stable, so ties keep the
// input order.
int64_t total_key64(double d) {
  int64_t i;
  std::memcpy(&i, &d, 8);
  return i ^ (int64_t)(((uint64_t)(i >> 63)) >> 1);
}
int32_t total_key32(float f) {
  int32_t i;
  std::memcpy(&i, &f, 4);
  return i ^ (int32_t)(((uint32_t)(i >> 31)) >> 1);
}

int sort_value_cmp(const Col& c, int64_t x, int64_t y) {
  auto sgn = [](auto a, auto b) { return a < b ? -1 : (b < a ? 1 : 0); };
  switch (c.ty) {
    case T_F64: return sgn(total_key64(reinterpret_cast<const double*>(c.vals)[c.off + x]),
                           total_key64(reinterpret_cast<const double*>(c.vals)[c.off + y]));
    case T_F32: return sgn(total_key32(reinterpret_cast<const float*>(c.vals)[c.off + x]),
                           total_key32(reinterpret_cast<const float*>(c.vals)[c.off + y]));
    case T_U64: return sgn((uint64_t)c.ival(x), (uint64_t)c.ival(y));
    case T_UTF8: case T_DICT: return sgn(c.sval(x), c.sval(y));
    case T_DEC128: return sgn(c.dval(x), c.dval(y));
    default: return sgn(c.ival(x), c.ival(y));
  }
}

Batch sort_batch(const Batch& b, const prism_sort_key* keys, int n_keys, int64_t limit) {
  for (int i = 0; i < n_keys; ++i) {
    if (keys[i].column < 0 || keys[i].column >= (int)b.cols.size())
      fail(PRISM_ERR_INVALID_ARGUMENT, "sort column out of range");
    if (b.cols[keys[i].column]->ty == T_NULL) fail(PRISM_ERR_INVALID_ARGUMENT, "sorting by a null-typed column");
  }
  if (b.rows == 0 || n_keys == 0) return b;
  std::vector<int64_t> idx(b.rows);
  for (int64_t i = 0; i < b.rows; ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](int64_t x, int64_t y) {
    for (int k = 0; k < n_keys; ++k) {
      const Col& c = *b.cols[keys[k].column];
      const bool nx = c.null_at(x), ny = c.null_at(y);
      if (nx || ny) {
        if (nx && ny) continue;
        return nx ? keys[k].nulls_first != 0 : keys[k].nulls_first == 0;
      }
      int r = sort_value_cmp(c, x, y);
      if (r == 0) continue;
      if (keys[k].descending) r = -r;
      return r < 0;
    }
    return false;
  });
  if (limit >= 0 && limit < b.rows) idx.resize((size_t)limit);
  Batch out;
  out.rows = (int64_t)idx.size();
  for (auto& c : b.cols) out.cols.push_back(take_col(*c, idx, c->name, c->nullable));
  return out;
}

}  // namespace

// ================================================================ C API ====
extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

int oracle_hash_join(const ArrowArray* probe, const ArrowSchema* probe_schema,
                     const ArrowArray* build, const ArrowSchema* build_schema,
                     const prism_join_config* config, int n_threads, ArrowArray* out,
                     ArrowSchema* out_schema) {
  return guard([&] {
    Batch p = import_batch(probe, probe_schema), b = import_batch(build, build_schema);
    std::vector<int> pk(config->probe_keys, config->probe_keys + config->n_keys);
    std::vector<int> bk(config->build_keys, config->build_keys + config->n_keys);
    check_key_types(p, pk, b, bk);
    HashTable t = build_table(b, bk, n_threads);
    if (config->join_type == PRISM_JOIN_LEFT && b.rows == 0 && p.rows > 0)
      fail(PRISM_ERR_JOIN, "left join of a non-empty probe side with an empty build side "
                           "(unmatched rows would take build row 0)");
    Batch r = join_one(p, b, t, *config, pk, false);
    export_batch(r, out, out_schema);
  });
}

int oracle_probe_matches_chunked(const ArrowArray* const* probes, const ArrowSchema* probe_schema,
                                 int n_probes, const ArrowArray* build,
                                 const ArrowSchema* build_schema, const int32_t* probe_keys,
                                 const int32_t* build_keys, int n_keys, int n_threads,
                                 ArrowArray* outs, ArrowSchema* out_schemas) {
  return guard([&] {
    auto ps = import_all(probes, probe_schema, n_probes);
    Batch b = import_batch(build, build_schema);
    std::vector<int> pk(probe_keys, probe_keys + n_keys), bk(build_keys, build_keys + n_keys);
    for (auto& p : ps) check_key_types(p, pk, b, bk);
    HashTable t = build_table(b, bk, n_threads);
    std::vector<std::vector<uint32_t>> mp(n_probes), mb(n_probes);
    parallel_for(n_probes, n_threads, [&](int64_t i) { probe_table(t, ps[i], pk, mp[i], mb[i]); });
    for (int i = 0; i < n_probes; ++i) {
      Batch r;
      r.rows = (int64_t)mp[i].size();
      Builder a(T_U32, "probe_idx", false), c(T_U32, "build_idx", false);
      for (size_t k = 0; k < mp[i].size(); ++k) { a.push_i64(mp[i][k]); c.push_i64(mb[i][k]); }
      r.cols = {a.finish(), c.finish()};
      export_batch(r, &outs[i], &out_schemas[i]);
    }
  });
}

int oracle_hash_join_probe_chunked(const ArrowArray* const* probes, const ArrowSchema* probe_schema,
                                   int n_probes, const ArrowArray* build,
                                   const ArrowSchema* build_schema, const prism_join_config* config,
                                   int n_threads, ArrowArray* outs, ArrowSchema* out_schemas,
                                   int* n_out) {
  return guard([&] {
    auto ps = import_all(probes, probe_schema, n_probes);
    Batch b = import_batch(build, build_schema);
    std::vector<int> pk(config->probe_keys, config->probe_keys + config->n_keys);
    std::vector<int> bk(config->build_keys, config->build_keys + config->n_keys);
    for (auto& p : ps) check_key_types(p, pk, b, bk);
    HashTable t = build_table(b, bk, n_threads);
    std::vector<Batch> res(n_probes);
    parallel_for(n_probes, n_threads, [&](int64_t i) {
      if (config->join_type == PRISM_JOIN_LEFT && b.rows == 0 && ps[i].rows > 0)
        fail(PRISM_ERR_JOIN, "left join with an empty build side");
      res[i] = join_one(ps[i], b, t, *config, pk, true);
    });
    int k = 0;
    for (int i = 0; i < n_probes; ++i)
      if (res[i].rows > 0) { export_batch(res[i], &outs[k], &out_schemas[k]); ++k; }
    *n_out = k;
  });
}

int64_t oracle_join_count_matches(const ArrowArray* const* probes, const ArrowSchema* probe_schema,
                                  int n_probes, const ArrowArray* build,
                                  const ArrowSchema* build_schema, const int32_t* probe_keys,
                                  const int32_t* build_keys, int n_keys, int n_threads,
                                  int materialize) {
  int64_t total = -1;
  int rc = guard([&] {
    auto ps = import_all(probes, probe_schema, n_probes);
    Batch b = import_batch(build, build_schema);
    std::vector<int> pk(probe_keys, probe_keys + n_keys), bk(build_keys, build_keys + n_keys);
    HashTable t = build_table(b, bk, n_threads);
    std::vector<int64_t> counts(n_probes, 0);
    parallel_for(n_probes, n_threads, [&](int64_t i) {
      std::vector<uint32_t> pi, bi;
      probe_table(t, ps[i], pk, pi, bi);
      counts[i] = (int64_t)pi.size();
      if (materialize >= 2 && b.cols.size() > 1) {  // take(build payload, build_idx)
        const Col& pay = *b.cols[1];
        std::vector<int64_t> g(bi.size());
        for (size_t k = 0; k < bi.size(); ++k) g[k] = pay.ival(bi[k]);
        counts[i] += (int64_t)(g.empty() ? 0 : (g[0] & 0));
      }
    });
    total = 0;
    for (auto c : counts) total += c;
  });
  return rc == PRISM_OK ? total : -(int64_t)rc;
}

int oracle_hash_aggregate_batches(const ArrowArray* const* batches, const ArrowSchema* schema,
                                  int n_batches, const prism_agg_config* config, int n_threads,
                                  ArrowArray* out, ArrowSchema* out_schema) {
  return guard([&] {
    auto bs = import_all(batches, schema, n_batches);
    Batch r = aggregate_batches(bs, schema_cols_of(schema), *config, n_threads, false);
    export_batch(r, out, out_schema);
  });
}

int oracle_evaluate_predicate(const ArrowArray* batch, const ArrowSchema* schema,
                              const prism_predicate* predicate, ArrowArray* out,
                              ArrowSchema* out_schema) {
  return guard([&] {
    Batch b = import_batch(batch, schema);
    BoolCol m = eval_pred_range(b, predicate->nodes, predicate->n_nodes);
    Batch r;
    r.rows = b.rows;
    r.cols = {bool_to_col(m, "mask")};
    export_batch(r, out, out_schema);
  });
}

int oracle_sort_batch(const ArrowArray* batch, const ArrowSchema* schema, const prism_sort_key* keys, int n_keys,
                      int64_t limit, ArrowArray* out, ArrowSchema* out_schema) {
  return guard([&] {
    Batch b = import_batch(batch, schema);
    export_batch(sort_batch(b, keys, n_keys, limit), out, out_schema);
  });
}

int oracle_filter_batch(const ArrowArray* batch, const ArrowSchema* schema, const ArrowArray* mask,
                        const ArrowSchema* mask_schema, ArrowArray* out, ArrowSchema* out_schema) {
  return guard([&] {
    Batch b = import_batch(batch, schema), m = import_batch(mask, mask_schema);
    if (m.cols.size() != 1 || m.cols[0]->ty != T_BOOL || m.rows != b.rows)
      fail(PRISM_ERR_INVALID_ARGUMENT, "mask must be one Boolean column of the batch's length");
    std::vector<uint8_t> keep(b.rows);
    for (int64_t i = 0; i < b.rows; ++i) keep[i] = !m.cols[0]->null_at(i) && m.cols[0]->ival(i);
    export_batch(filter_by(b, keep), out, out_schema);
  });
}

int oracle_project_batch(const ArrowArray* batch, const ArrowSchema* schema, const int32_t* cols,
                         int n_cols, ArrowArray* out, ArrowSchema* out_schema) {
  return guard([&] {
    Batch b = import_batch(batch, schema);
    export_batch(project(b, cols, n_cols), out, out_schema);
  });
}

int oracle_filter_and_project(const ArrowArray* batch, const ArrowSchema* schema,
                              const prism_predicate* predicate, const int32_t* cols, int n_cols,
                              ArrowArray* out, ArrowSchema* out_schema) {
  return guard([&] {
    Batch b = import_batch(batch, schema);
    Batch f = b;
    if (predicate) f = filter_by(b, keep_of(eval_pred_range(b, predicate->nodes, predicate->n_nodes)));
    export_batch(n_cols == 0 ? f : project(f, cols, n_cols), out, out_schema);
  });
}

int oracle_project_batch_with_exprs(const ArrowArray* batch, const ArrowSchema* schema,
                                    const int32_t* cols, int n_cols, const prism_expr* exprs,
                                    int n_exprs, int arith_mode, ArrowArray* out,
                                    ArrowSchema* out_schema) {
  return guard([&] {
    Batch b = import_batch(batch, schema);
    export_batch(project_exprs(b, cols, n_cols, exprs, n_exprs, arith_mode), out, out_schema);
  });
}

int oracle_filter_project_aggregate(const ArrowArray* const* batches, const ArrowSchema* schema,
                                    int n_batches, const prism_predicate* predicate,
                                    const int32_t* cols, int n_cols, const prism_expr* exprs,
                                    int n_exprs, int arith_mode, const prism_agg_config* agg,
                                    int n_threads, ArrowArray* out, ArrowSchema* out_schema) {
  return guard([&] {
    auto bs = import_all(batches, schema, n_batches);
    std::vector<Batch> projected(bs.size());
    parallel_for((int64_t)bs.size(), n_threads, [&](int64_t i) {
      Batch f = bs[i];
      if (predicate) f = filter_by(bs[i], keep_of(eval_pred_range(bs[i], predicate->nodes, predicate->n_nodes)));
      projected[i] = project_exprs(f, cols, n_cols, exprs, n_exprs, arith_mode);
    });
    std::vector<ColP> sc;
    if (!projected.empty()) sc = projected[0].cols;
    Batch r = aggregate_batches(projected, sc, *agg, n_threads, arith_mode == PRISM_ARITH_EXACT);
    export_batch(r, out, out_schema);
  });
}

int oracle_join_aggregate(const ArrowArray* const* probes, const ArrowSchema* probe_schema,
                          int n_probes, const ArrowArray* build, const ArrowSchema* build_schema,
                          const int32_t* probe_keys, const int32_t* build_keys, int n_keys,
                          const int32_t* cols, int n_cols, const prism_expr* exprs, int n_exprs,
                          const prism_agg_config* agg, int n_threads, ArrowArray* out,
                          ArrowSchema* out_schema) {
  return guard([&] {
    auto ps = import_all(probes, probe_schema, n_probes);
    Batch b = import_batch(build, build_schema);
    std::vector<int> pk(probe_keys, probe_keys + n_keys), bk(build_keys, build_keys + n_keys);
    for (auto& p : ps) check_key_types(p, pk, b, bk);
    Batch r = join_aggregate(ps, b, pk, bk, cols, n_cols, exprs, n_exprs, *agg, n_threads);
    export_batch(r, out, out_schema);
  });
}

double oracle_exact_sum_f64(const double* values, int64_t n) {
  ExactSum s;
  for (int64_t i = 0; i < n; ++i) s.add(values[i]);
  return s.result();
}

}  // extern "C"
