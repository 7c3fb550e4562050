// jit.cu — run-time generation and NVRTC compilation of per-query kernels.
//
// Generated code mirrors the interpreters of eval.cuh node for node:
//   predicates  eval_pred  (native/prism-executor/src/filter_project.rs:65-123, 346-404)
//   expressions eval_expr  (filter_project.rs:216-294)
// with the column types, null-freedom and program shape fixed at generation
// time. Literal values are read from the device programs once per thread
// (E::load), so queries that differ only in literals share one compiled
// kernel. NVRTC is loaded with dlopen on first use; kernels are loaded
// through the runtime's library API (cudaLibraryLoadData).
#include "jit.hpp"

#include <dlfcn.h>
#include <nvrtc.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <condition_variable>
#include <mutex>
#include <sstream>
#include <unordered_map>
#include <vector>

#include "agg_device.cuh"
#include "plan.hpp"

namespace prism {

// embedded device headers (generated by build.py from csrc/)
extern const int kJitHeaderCount;
extern const char* const kJitHeaderNames[];
extern const char* const kJitHeaderTexts[];

namespace {

struct Nvrtc {
  decltype(&nvrtcCreateProgram) create = nullptr;
  decltype(&nvrtcCompileProgram) compile = nullptr;
  decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
  decltype(&nvrtcGetProgramLog) log = nullptr;
  decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
  decltype(&nvrtcGetCUBIN) cubin = nullptr;
  decltype(&nvrtcDestroyProgram) destroy = nullptr;
  bool ok = false;
};

Nvrtc load_nvrtc() {
  Nvrtc n;
  const char* env = std::getenv("PRISM_JIT");
  if (env && std::strcmp(env, "0") == 0) return n;
  void* h = dlopen("libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
  if (!h) h = dlopen("/usr/local/cuda/lib64/libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
  if (!h) return n;
  n.create = reinterpret_cast<decltype(n.create)>(dlsym(h, "nvrtcCreateProgram"));
  n.compile = reinterpret_cast<decltype(n.compile)>(dlsym(h, "nvrtcCompileProgram"));
  n.log_size = reinterpret_cast<decltype(n.log_size)>(dlsym(h, "nvrtcGetProgramLogSize"));
  n.log = reinterpret_cast<decltype(n.log)>(dlsym(h, "nvrtcGetProgramLog"));
  n.cubin_size = reinterpret_cast<decltype(n.cubin_size)>(dlsym(h, "nvrtcGetCUBINSize"));
  n.cubin = reinterpret_cast<decltype(n.cubin)>(dlsym(h, "nvrtcGetCUBIN"));
  n.destroy = reinterpret_cast<decltype(n.destroy)>(dlsym(h, "nvrtcDestroyProgram"));
  n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy;
  return n;
}

Nvrtc& nvrtc() {
  static Nvrtc n = load_nvrtc();
  return n;
}

struct Entry {
  cudaLibrary_t lib = nullptr;
  std::unordered_map<std::string, cudaKernel_t> kernels;
  bool ready = false;  // false while one thread compiles it (others wait on g_cv)
};

std::mutex g_mu;
std::condition_variable g_cv;
std::unordered_map<std::string, Entry> g_cache;
int64_t g_compiles = 0;
double g_compile_ms = 0;

// ------------------------------------------------------------ generator --

const char* cmp_op(int c) {
  switch (c) {
    case C_EQ: return "==";
    case C_NE: return "!=";
    case C_LT: return "<";
    case C_LE: return "<=";
    case C_GT: return ">";
    default: return ">=";
  }
}

// Magnitude bounds of 128-bit values (exact, saturating): an add, subtract
// or multiply whose operand bounds keep |result| <= 2^127 - 1 cannot
// overflow and needs no check.
struct Mag {
  unsigned __int128 m = 0;
  bool unknown = true;
};
const unsigned __int128 I128_MAX = ((unsigned __int128)1 << 127) - 1;

Mag mag_of(unsigned __int128 m) {
  Mag r;
  r.m = m;
  r.unknown = false;
  return r;
}

// |value| bound of a column read by dcol_i128
Mag type_mag(int t) {
  switch (t) {
    case TY_BOOL: return mag_of(1);
    case TY_I8: return mag_of(128);
    case TY_U8: return mag_of(255);
    case TY_I16: return mag_of(1 << 15);
    case TY_U16: return mag_of(65535);
    case TY_I32: case TY_DATE32: return mag_of((unsigned __int128)1 << 31);
    case TY_U32: return mag_of(((unsigned __int128)1 << 32) - 1);
    case TY_I64: return mag_of((unsigned __int128)1 << 63);
    case TY_U64: return mag_of(((unsigned __int128)1 << 64) - 1);
    default: return Mag{};
  }
}

Mag mag_add(Mag a, Mag b) {
  if (a.unknown || b.unknown) return Mag{};
  unsigned __int128 s = a.m + b.m;
  if (s < a.m) return Mag{};
  return mag_of(s);
}

Mag mag_mul(Mag a, Mag b) {
  if ((!a.unknown && a.m == 0) || (!b.unknown && b.m == 0)) return mag_of(0);
  if (a.unknown || b.unknown) return Mag{};
  if (a.m > ~(unsigned __int128)0 / b.m) return Mag{};
  return mag_of(a.m * b.m);
}

Mag mag_max(Mag a, Mag b) {
  if (a.unknown || b.unknown) return Mag{};
  return mag_of(a.m > b.m ? a.m : b.m);
}

bool mag_fits(Mag a) { return !a.unknown && a.m <= I128_MAX; }

std::string hex64(uint64_t u) {
  char buf[32];
  std::snprintf(buf, sizeof buf, "0x%016llxULL", (unsigned long long)u);
  return buf;
}

struct Gen {
  const Program& pg;
  const Batch& b;
  std::ostringstream consts;  // Consts fields
  std::ostringstream load;    // E::load statements
  std::unordered_map<std::string, bool> have;
  std::ostringstream out;     // current function body
  int id = 0;
  bool ok = true;
  // program slot of the build column whose value the join table's slot
  // entries carry (read from the entry for a single-row slot), or -1
  int inl_slot = -1;

  Gen(const Program& p, const Batch& bb) : pg(p), b(bb) {}

  std::string fresh(const char* p) { return p + std::to_string(id++); }

  // every program the plan compiler emits is covered: a miss is an engine bug
  [[noreturn]] void gen_fail(const char* why) { fail(PRISM_ERR_INTERNAL, std::string("kernel generator: ") + why); }

  void konst(const std::string& decl_type, const std::string& name, const std::string& init) {
    if (have.count(name)) return;
    have[name] = true;
    consts << "    " << decl_type << " " << name << ";\n";
    load << "    K." << name << " = " << init << ";\n";
  }

  // Fixed-width columns (numbers, Boolean, dictionary indices, decimals)
  // are fetched for a row up front into a Row of raw register words (one
  // load each, no control flow, so the loads of several rows overlap); the
  // typed views below read them from there with the same dcol_* helpers the
  // interpreter uses (index 0 of the view, a constant type so the type
  // switches fold). Utf8 columns are read in place at the row index.
  int col_type(int slot) const { return b.cols[pg.cols[slot]]->type; }
  bool fetched(int slot) const { return width_of(col_type(slot) == TY_DICT ? TY_I32 : col_type(slot)) > 0 || col_type(slot) == TY_BOOL || col_type(slot) == TY_DICT; }
  bool nullable(int slot) const { return b.cols[pg.cols[slot]]->validity != nullptr; }
  // the row index a column is read at: build-side columns of a fused join
  // at the matched build row `bidx`, every other column at `idx`
  std::vector<char> bside;
  std::string rix(int slot) const { return slot < (int)bside.size() && bside[slot] ? "bidx" : "idx"; }
  std::string ix(int slot) const { return fetched(slot) ? "0" : rix(slot); }

  void declare_cols() {
    for (size_t s = 0; s < pg.cols.size(); ++s) {
      const Column& c = *b.cols[pg.cols[s]];
      int t = c.type == TY_BOOL ? TY_U8 : c.type;  // a fetched Boolean is one byte 0 / 1
      out << "    DCol c" << s << " = cols[" << s << "];\n";
      out << "    c" << s << ".type = " << t << "; c" << s << ".index_type = " << c.index_type << "; c" << s
          << ".scale = " << c.scale << ";";
      if (fetched((int)s)) out << " c" << s << ".values = &row.r" << s << "[0]; c" << s << ".validity = nullptr;";
      else if (!c.validity) out << " c" << s << ".validity = nullptr;";
      out << "\n";
    }
  }

  std::string col(int slot) {
    if (slot < 0 || slot >= (int)pg.cols.size()) gen_fail("column slot out of range");
    return "c" + std::to_string(slot);
  }

  // validity of the row in column `slot`
  std::string V(int slot) const {
    if (fetched(slot)) return nullable(slot) ? "row.m" + std::to_string(slot) : std::string("true");
    return "dcol_valid(c" + std::to_string(slot) + ", " + rix(slot) + ")";
  }
  // plain reader: fn(view, index)
  std::string rd(const char* fn, int slot) const {
    return std::string(fn) + "(c" + std::to_string(slot) + ", " + ix(slot) + ")";
  }
  // the dcol_*_cast readers: a null row of a column other than Float64 and
  // Decimal128 reads 0 (as arrow's casts leave it)
  std::string rd_cast(const char* fn, const char* zero, int slot) const {
    int t = col_type(slot);
    if (t == TY_F64 || t == TY_DEC128 || !nullable(slot)) return rd(fn, slot);
    return "(" + V(slot) + " ? " + rd(fn, slot) + " : " + zero + ")";
  }

  // struct Row and fetch(): raw words of every fixed-width program column
  std::string row_struct() const {
    std::ostringstream o;
    o << "  struct Row {\n";
    bool any = false;
    for (size_t s = 0; s < pg.cols.size(); ++s) {
      if (!fetched((int)s)) continue;
      any = true;
      const Column& c = *b.cols[pg.cols[s]];
      int t = c.type == TY_DICT ? c.index_type : c.type;
      // one 32-bit register for columns of up to 4 bytes (read from its low bytes)
      if (t == TY_DEC128) o << "    unsigned long long r" << s << "[2];\n";
      else if (width_of(t) == 8) o << "    unsigned long long r" << s << "[1];\n";
      else o << "    unsigned int r" << s << "[1];\n";
      if (nullable((int)s)) o << "    bool m" << s << ";\n";
    }
    if (!any) o << "    int unused;\n";
    o << "  };\n  static __device__ __forceinline__ Row fetch(const DCol* cols, idx_t idx, idx_t bidx, "
         "unsigned long long inl = 0, bool use_inl = false) {\n    Row w;\n";
    for (size_t s = 0; s < pg.cols.size(); ++s) {
      if (!fetched((int)s)) continue;
      const Column& c = *b.cols[pg.cols[s]];
      int t = c.type == TY_DICT ? c.index_type : c.type;
      std::string src = "cols[" + std::to_string(s) + "].values";
      const std::string at = rix((int)s);
      if ((int)s == inl_slot && !c.validity && (width_of(t) == 4 || width_of(t) == 8) && t != TY_BOOL) {
        const char* ty = width_of(t) == 4 ? "uint32_t" : "unsigned long long";
        o << "    w.r" << s << "[0] = use_inl ? (" << ty << ")inl : static_cast<const " << ty << "*>(" << src << ")["
          << at << "];\n";
        continue;
      }
      switch (t == TY_BOOL ? 0 : width_of(t)) {
        case 0:
          o << "    w.r" << s << "[0] = (static_cast<const uint8_t*>(" << src << ")[" << at << " >> 3] >> (" << at << " & 7)) & 1;\n";
          break;
        case 1: o << "    w.r" << s << "[0] = static_cast<const uint8_t*>(" << src << ")[" << at << "];\n"; break;
        case 2: o << "    w.r" << s << "[0] = static_cast<const uint16_t*>(" << src << ")[" << at << "];\n"; break;
        case 4: o << "    w.r" << s << "[0] = static_cast<const uint32_t*>(" << src << ")[" << at << "];\n"; break;
        case 8: o << "    w.r" << s << "[0] = static_cast<const unsigned long long*>(" << src << ")[" << at << "];\n"; break;
        default:
          o << "    w.r" << s << "[0] = static_cast<const unsigned long long*>(" << src << ")[2 * " << at << "];\n";
          o << "    w.r" << s << "[1] = static_cast<const unsigned long long*>(" << src << ")[2 * " << at << " + 1];\n";
      }
      if (c.validity)
        o << "    w.m" << s << " = (cols[" << s << "].validity[" << at << " >> 3] >> (" << at << " & 7)) & 1;\n";
    }
    o << "    return w;\n  }\n";
    return o.str();
  }

  // predicate nodes [begin, begin + len): emits statements, returns the
  // names of the value bit and the validity bit
  std::pair<std::string, std::string> pred(int begin, int len) {
    std::vector<std::pair<std::string, std::string>> st;
    const std::pair<std::string, std::string> bad{"false", "false"};
    for (int k = begin; k < begin + len; ++k) {
      const PNode& nd = pg.pnodes[k];
      std::string v = fresh("pv"), a = fresh("pa"), K = std::to_string(k);
      switch (nd.op) {
        case P_LIT:
          konst("bool", "pl" + K, "a.pn[" + K + "].i != 0");
          out << "    bool " << v << " = K.pl" << K << ", " << a << " = true;\n";
          break;
        case P_CMP_INT: {
          std::string c = col(nd.col);
          konst("int64_t", "pi" + K, "a.pn[" + K + "].i");
          out << "    bool " << a << " = " << V(nd.col) << ";\n";
          out << "    bool " << v << " = " << rd("dcol_ival", nd.col) << " " << cmp_op(nd.cmp) << " K.pi" << K << ";\n";
          break;
        }
        case P_CMP_F64: {
          std::string c = col(nd.col);
          konst("int64_t", "pf" + K, "total_key(a.pn[" + K + "].f)");
          out << "    bool " << a << " = " << V(nd.col) << ";\n";
          out << "    bool " << v << " = total_key(static_cast<const double*>(" << c << ".values)[" << ix(nd.col) << "]) "
              << cmp_op(nd.cmp) << " K.pf" << K << ";\n";
          break;
        }
        case P_CMP_STR: case P_LIKE: {
          std::string c = col(nd.col);
          konst("const uint8_t*", "ps" + K, "a.pn[" + K + "].s");
          konst("int32_t", "pn" + K, "a.pn[" + K + "].slen");
          std::string p = fresh("sp"), n = fresh("sn");
          out << "    bool " << a << " = " << V(nd.col) << ";\n";
          out << "    const uint8_t* " << p << "; int32_t " << n << "; dcol_str(" << c << ", " << ix(nd.col) << ", " << p << ", " << n
              << ");\n";
          if (nd.op == P_CMP_STR)
            out << "    bool " << v << " = bytes_cmp(" << p << ", " << n << ", K.ps" << K << ", K.pn" << K << ") "
                << cmp_op(nd.cmp) << " 0;\n";
          else
            out << "    bool " << v << " = like_match(" << p << ", " << n << ", K.ps" << K << ", K.pn" << K << ", "
                << (nd.cmp != 0 ? "true" : "false") << ");\n";
          break;
        }
        case P_IS_NULL: case P_IS_NOT_NULL: {
          std::string c = col(nd.col);
          out << "    bool " << v << " = " << (nd.op == P_IS_NULL ? "!" : "") << "(" << V(nd.col) << "), " << a
              << " = true;\n";
          break;
        }
        case P_AND: case P_OR: {
          if (st.size() < 2) { gen_fail("AND/OR without two operands"); return bad; }
          auto r = st.back(); st.pop_back();
          auto l = st.back(); st.pop_back();
          out << "    bool " << v << " = " << l.first << (nd.op == P_AND ? " && " : " || ") << r.first << ", " << a
              << " = " << l.second << " && " << r.second << ";\n";
          break;
        }
        case P_NOT: {
          if (st.empty()) { gen_fail("NOT without an operand"); return bad; }
          auto x = st.back(); st.pop_back();
          out << "    bool " << v << " = !" << x.first << ", " << a << " = " << x.second << ";\n";
          break;
        }
        default:
          gen_fail("unknown predicate node");
          return bad;
      }
      st.push_back({v, a});
    }
    if (st.size() != 1) { gen_fail("predicate leaves more than one value"); return bad; }
    return st.back();
  }

  struct EV {
    std::string n;
    Mag mag;  // bound of |n.i|
  };

  // expression nodes [begin, end): emits statements, returns the Val
  // variable; `ovf` names the overflow flag of the enclosing scope
  std::string expr(int begin, int end, const std::string& ovf) {
    std::vector<EV> st;
    for (int k = begin; k < end; ++k) {
      const ENode& nd = pg.enodes[k];
      std::string n = fresh("e"), K = std::to_string(k);
      auto pop = [&]() -> EV {
        if (st.empty()) { gen_fail("expression stack underflow"); return EV{"e_bad", Mag{}}; }
        EV x = st.back();
        st.pop_back();
        return x;
      };
      switch (nd.op) {
        case E_COL_F64: {
          std::string c = col(nd.col);
          out << "    Val " << n << "; " << n << ".i = 0; " << n << ".f = "
              << (nd.a ? rd("dcol_fval", nd.col) : rd_cast("dcol_fval", "0.0", nd.col)) << "; " << n << ".valid = " << V(nd.col)
              << ";\n";
          st.push_back({n, Mag{}});
          break;
        }
        case E_COL_I128: {
          std::string c = col(nd.col);
          const Column& cc = *b.cols[pg.cols[std::max(0, std::min(nd.col, (int)pg.cols.size() - 1))]];
          int t = cc.type == TY_DICT ? cc.index_type : cc.type;
          out << "    Val " << n << "; " << n << ".f = 0; " << n << ".i = "
              << (nd.a ? rd("dcol_i128", nd.col) : rd_cast("dcol_i128", "(__int128)0", nd.col)) << "; " << n
              << ".valid = " << V(nd.col) << ";\n";
          st.push_back({n, type_mag(t)});
          break;
        }
        case E_LIT_F64:
          konst("double", "ef" + K, "a.en[" + K + "].f");
          out << "    Val " << n << "; " << n << ".i = 0; " << n << ".f = K.ef" << K << "; " << n << ".valid = true;\n";
          st.push_back({n, Mag{}});
          break;
        case E_LIT_I128: {
          // the bound used is the literal's power-of-two ceiling, which the
          // source records: literals of one size class share a kernel
          __int128 v = (__int128)(((unsigned __int128)(uint64_t)nd.hi << 64) | (uint64_t)nd.lo);
          unsigned __int128 m = v < 0 ? (unsigned __int128)0 - (unsigned __int128)v : (unsigned __int128)v;
          int bits = 0;
          while (bits < 127 && ((unsigned __int128)1 << bits) < m) ++bits;
          konst("__int128", "ei" + K,
                "(__int128)(((unsigned __int128)(uint64_t)a.en[" + K + "].hi << 64) | (uint64_t)a.en[" + K + "].lo)");
          out << "    Val " << n << "; " << n << ".f = 0; " << n << ".i = K.ei" << K << "; " << n
              << ".valid = true;  // |literal| <= 2^" << bits << "\n";
          st.push_back({n, mag_of((unsigned __int128)1 << bits)});
          break;
        }
        case E_ADD_F: case E_SUB_F: case E_MUL_F: case E_DIV_F: {
          EV r = pop(), l = pop();
          const char* op = nd.op == E_ADD_F ? "+" : nd.op == E_SUB_F ? "-" : nd.op == E_MUL_F ? "*" : "/";
          out << "    Val " << n << " = " << l.n << "; " << n << ".f = " << l.n << ".f " << op << " " << r.n << ".f; "
              << n << ".valid = " << l.n << ".valid && " << r.n << ".valid;\n";
          st.push_back({n, Mag{}});
          break;
        }
        case E_NEG_F: {
          EV x = pop();
          out << "    Val " << n << " = " << x.n << "; " << n << ".f = -" << x.n << ".f;\n";
          st.push_back({n, Mag{}});
          break;
        }
        case E_ADD_I: case E_SUB_I: case E_MUL_I: {
          EV r = pop(), l = pop();
          Mag bound = nd.op == E_MUL_I ? mag_mul(l.mag, r.mag) : mag_add(l.mag, r.mag);
          out << "    Val " << n << "; " << n << ".f = 0; " << n << ".valid = " << l.n << ".valid && " << r.n
              << ".valid;\n";
          if (mag_fits(bound)) {
            // operand ranges rule out a 128-bit overflow: wrapping
            // arithmetic gives the exact result
            const char* op = nd.op == E_ADD_I ? "+" : nd.op == E_SUB_I ? "-" : "*";
            out << "    " << n << ".i = (__int128)((unsigned __int128)" << l.n << ".i " << op << " (unsigned __int128)"
                << r.n << ".i);\n";
            st.push_back({n, bound});
          } else {
            const char* fn = nd.op == E_ADD_I ? "add_ovf_i128" : nd.op == E_SUB_I ? "sub_ovf_i128" : "mul_ovf_i128";
            out << "    { __int128 o; if (" << fn << "(" << l.n << ".i, " << r.n << ".i, o) && " << n << ".valid) "
                << ovf << " = true; " << n << ".i = o; }\n";
            st.push_back({n, Mag{}});
          }
          break;
        }
        case E_NEG_I: {
          EV x = pop();
          out << "    Val " << n << " = " << x.n << "; " << n
              << ".i = (__int128)((unsigned __int128)0 - (unsigned __int128)" << x.n << ".i);\n";
          st.push_back({n, x.mag});
          break;
        }
        case E_I2F: {
          EV x = pop();
          double sc = 1.0;
          for (int q = 0; q < nd.col; ++q) sc *= 10.0;
          uint64_t u;
          std::memcpy(&u, &sc, 8);
          out << "    Val " << n << " = " << x.n << "; " << n << ".f = (double)" << x.n << ".i / __longlong_as_double("
              << hex64(u) << ");  // 10^" << nd.col << "\n";
          st.push_back({n, Mag{}});
          break;
        }
        case E_SCALE_I: {
          EV x = pop();
          out << "    Val " << n << " = " << x.n << "; { __int128 o; if (mul_ovf_i128(" << x.n << ".i, pow10_i128("
              << nd.col << "), o) && " << x.n << ".valid) " << ovf << " = true; " << n << ".i = o; }\n";
          st.push_back({n, Mag{}});
          break;
        }
        case E_F2I: {
          EV x = pop();
          out << "    Val " << n << " = " << x.n << "; { double t = trunc(" << x.n << ".f); if (!" << x.n << ".valid) { "
              << n << ".i = 0; } else if (!(t >= -9.223372036854775808e18 && t < 9.223372036854775808e18)) { " << n
              << ".valid = false; " << n << ".i = 0; } else { " << n << ".i = (__int128)(long long)t; } }\n";
          st.push_back({n, mag_of((unsigned __int128)1 << 63)});
          break;
        }
        case E_SELECT: {
          int nc = nd.col, has_else = nd.a, need = nc + has_else;
          if ((int)st.size() < need || nc < 0) { gen_fail("IfThen without its branches"); return "e_bad"; }
          int base = (int)st.size() - need;
          Mag bound = mag_of(0);
          for (int q = base; q < (int)st.size(); ++q) bound = mag_max(bound, st[q].mag);
          out << "    Val " << n << ";";
          if (has_else) out << " " << n << " = " << st.back().n << ";\n";
          else out << " " << n << ".valid = false; " << n << ".i = 0; " << n << ".f = 0;\n";
          // the first clause that holds wins: evaluate from the last one
          // backwards, each match overriding
          for (int ci = nc - 1; ci >= 0; --ci) {
            if (nd.b + ci < 0 || nd.b + ci >= (int)pg.clauses.size()) { gen_fail("IfThen clause out of range"); return "e_bad"; }
            const PRange& cl = pg.clauses[nd.b + ci];
            out << "    {\n";
            auto pv = pred(cl.begin, cl.len);
            out << "    if (" << pv.first << " && " << pv.second << ") " << n << " = " << st[base + ci].n
                << ";\n    }\n";
          }
          st.resize(base);
          st.push_back({n, bound});
          break;
        }
        default:
          gen_fail("unknown expression node");
          return "e_bad";
      }
    }
    if (st.size() != 1) { gen_fail("expression leaves more than one value"); return "e_bad"; }
    return st.back().n;
  }

  // 64-bit fast path of an exact (int128) program: the same values computed
  // in int64, each step with an "ok" flag (no overflow, and for products
  // both factors inside int32); exact whenever the root's flag holds.
  // Emits into `out`; returns the names of the value, validity and ok
  // variables, or false when the program has a node the fast path does not
  // take (IfThen, Float64 steps, Decimal128 or UInt64 columns). With `cse`,
  // subtrees met before in this function (same columns, literal values and
  // operations) are reused instead of recomputed.
  struct FV {
    std::string n, v, ok;
    Mag mag;
  };
  std::unordered_map<std::string, FV> cse_map;
  bool cse = false;

  bool expr_fast64(int begin, int end, std::string& val, std::string& valid, std::string& okv) {
    for (int k = begin; k < end; ++k) {
      int op = pg.enodes[k].op;
      if (op == E_COL_I128) {
        const Column& cc = *b.cols[pg.cols[std::max(0, std::min(pg.enodes[k].col, (int)pg.cols.size() - 1))]];
        int t = cc.type == TY_DICT ? cc.index_type : cc.type;
        if (t == TY_U64 || type_mag(t).unknown) return false;
      } else if (op != E_LIT_I128 && op != E_ADD_I && op != E_SUB_I && op != E_MUL_I && op != E_NEG_I &&
                 !(op == E_SCALE_I && pg.enodes[k].col <= 18)) {
        return false;
      }
    }
    const unsigned __int128 I64_MAX = ((unsigned __int128)1 << 63) - 1;
    auto fits64 = [&](Mag m) { return !m.unknown && m.m <= I64_MAX; };
    auto in32 = [&](const std::string& x) { return "(long long)(int)" + x + " == " + x; };
    std::vector<std::pair<std::string, FV>> st;  // (signature, value)
    for (int k = begin; k < end; ++k) {
      const ENode& nd = pg.enodes[k];
      std::string K = std::to_string(k);
      std::string sig;
      std::vector<std::pair<std::string, FV>> kids;
      int arity = (nd.op == E_ADD_I || nd.op == E_SUB_I || nd.op == E_MUL_I) ? 2
                  : (nd.op == E_NEG_I || nd.op == E_SCALE_I) ? 1 : 0;
      if ((int)st.size() < arity) gen_fail("expression stack underflow");
      for (int q = 0; q < arity; ++q) kids.insert(kids.begin(), st.back()), st.pop_back();
      switch (nd.op) {
        case E_COL_I128: sig = "c" + std::to_string(nd.col) + (nd.a ? "r" : ""); break;
        case E_LIT_I128: sig = "l" + std::to_string(nd.lo) + ":" + std::to_string(nd.hi); break;
        case E_SCALE_I: sig = "s" + std::to_string(nd.col) + "(" + kids[0].first + ")"; break;
        case E_NEG_I: sig = "n(" + kids[0].first + ")"; break;
        default: sig = std::to_string(nd.op) + "(" + kids[0].first + "," + kids[1].first + ")";
      }
      if (cse) {
        auto it = cse_map.find(sig);
        if (it != cse_map.end()) {
          st.push_back({sig, it->second});
          continue;
        }
      }
      FV f;
      f.n = fresh("f");
      f.v = fresh("fv");
      f.ok = fresh("fo");
      switch (nd.op) {
        case E_COL_I128: {
          std::string c = col(nd.col);
          const Column& cc = *b.cols[pg.cols[nd.col]];
          int t = cc.type == TY_DICT ? cc.index_type : cc.type;
          out << "    long long " << f.n << " = " << (nd.a ? rd("dcol_ival", nd.col) : rd_cast("dcol_ival", "0LL", nd.col))
              << "; bool " << f.v << " = " << V(nd.col) << "; const bool " << f.ok << " = true;\n";
          f.mag = type_mag(t);
          break;
        }
        case E_LIT_I128: {
          // bound: the literal's power-of-two ceiling, recorded in the source
          __int128 lv = (__int128)(((unsigned __int128)(uint64_t)nd.hi << 64) | (uint64_t)nd.lo);
          unsigned __int128 m = lv < 0 ? (unsigned __int128)0 - (unsigned __int128)lv : (unsigned __int128)lv;
          int bits = 0;
          while (bits < 127 && ((unsigned __int128)1 << bits) < m) ++bits;
          konst("__int128", "ei" + K,
                "(__int128)(((unsigned __int128)(uint64_t)a.en[" + K + "].hi << 64) | (uint64_t)a.en[" + K + "].lo)");
          out << "    long long " << f.n << " = (long long)K.ei" << K << "; const bool " << f.v << " = true; bool " << f.ok
              << " = (__int128)" << f.n << " == K.ei" << K << ";  // |literal| <= 2^" << bits << "\n";
          f.mag = mag_of((unsigned __int128)1 << bits);
          break;
        }
        case E_ADD_I: case E_SUB_I: case E_MUL_I: {
          const FV& l = kids[0].second;
          const FV& r = kids[1].second;
          Mag bound = nd.op == E_MUL_I ? mag_mul(l.mag, r.mag) : mag_add(l.mag, r.mag);
          const char* o = nd.op == E_ADD_I ? "+" : nd.op == E_SUB_I ? "-" : "*";
          out << "    long long " << f.n << " = (long long)((unsigned long long)" << l.n << " " << o << " (unsigned long long)"
              << r.n << "); bool " << f.v << " = " << l.v << " && " << r.v << "; bool " << f.ok << " = " << l.ok << " && "
              << r.ok;
          if (!fits64(bound)) {
            if (nd.op == E_ADD_I)
              out << " && !(((" << l.n << " ^ " << f.n << ") & (" << r.n << " ^ " << f.n << ")) < 0)";
            else if (nd.op == E_SUB_I)
              out << " && !(((" << l.n << " ^ " << r.n << ") & (" << l.n << " ^ " << f.n << ")) < 0)";
            else  // safe when both factors lie inside int32; other rows take the 128-bit path
              out << " && " << (fits64(l.mag) && l.mag.m <= 0x7fffffff ? "true" : in32(l.n)) << " && "
                  << (fits64(r.mag) && r.mag.m <= 0x7fffffff ? "true" : in32(r.n));
            bound = Mag{};
          }
          out << ";\n";
          f.mag = bound;
          break;
        }
        case E_NEG_I: {
          const FV& x = kids[0].second;
          out << "    long long " << f.n << " = (long long)(0ULL - (unsigned long long)" << x.n << "); bool " << f.v << " = "
              << x.v << "; bool " << f.ok << " = " << x.ok << " && " << x.n << " != (long long)0x8000000000000000ULL;\n";
          f.mag = x.mag;
          break;
        }
        case E_SCALE_I: {
          const FV& x = kids[0].second;
          long long p10 = 1;
          for (int q = 0; q < nd.col; ++q) p10 *= 10;
          out << "    long long " << f.n << " = (long long)((unsigned long long)" << x.n << " * " << p10 << "ULL); bool "
              << f.v << " = " << x.v << "; bool " << f.ok << " = " << x.ok << " && (" << x.n
              << " < 0 ? 0ULL - (unsigned long long)" << x.n << " : (unsigned long long)" << x.n
              << ") <= " << (9223372036854775807LL / p10) << "ULL;\n";
          f.mag = Mag{};
          break;
        }
        default:
          gen_fail("unknown expression node");
      }
      if (cse) cse_map[sig] = f;
      st.push_back({sig, f});
    }
    if (st.size() != 1) gen_fail("expression leaves more than one value");
    val = st.back().second.n;
    valid = st.back().second.v;
    okv = st.back().second.ok;
    return true;
  }

  std::string take() {
    std::string s = out.str();
    out.str("");
    out.clear();
    return s;
  }
};

}  // namespace

bool jit_enabled() { return nvrtc().ok; }

void jit_stats(int64_t* compiles, double* ms) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (compiles) *compiles = g_compiles;
  if (ms) *ms = g_compile_ms;
}

// Compiles `source` with NVRTC and loads it (no lock held: a compile takes
// hundreds of milliseconds and must not stall lookups of other kernels).
static cudaLibrary_t compile_source(const std::string& source) {
  Nvrtc& N = nvrtc();
  if (!N.ok) fail(PRISM_ERR_INTERNAL, "run-time kernel compilation is not available (NVRTC not loaded)");
  nvrtcProgram prog;
  if (N.create(&prog, source.c_str(), "prism_query.cu", kJitHeaderCount, kJitHeaderTexts, kJitHeaderNames) !=
      NVRTC_SUCCESS)
    fail(PRISM_ERR_INTERNAL, "nvrtcCreateProgram failed");
  // no FMA contraction: generated Float64 arithmetic rounds after every
  // operation, like the interpreter and the reference
  // PRISM_JIT_VERBOSE=1: ptxas's resource report (registers, spills, shared
  // memory) of every compiled kernel on stderr
  const char* vb = std::getenv("PRISM_JIT_VERBOSE");
  const bool verbose = vb && vb[0] == '1';
  const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "--device-int128", "--fmad=false",
                        "--diag-suppress=550", "--ptxas-options=-v"};
  nvrtcResult r = N.compile(prog, verbose ? 6 : 5, opts);
  if (verbose && r == NVRTC_SUCCESS) {
    size_t ls = 0;
    N.log_size(prog, &ls);
    std::string log(ls, '\0');
    if (ls) N.log(prog, &log[0]);
    std::fprintf(stderr, "[prism jit] %s\n", log.c_str());
  }
  if (r != NVRTC_SUCCESS) {
    size_t ls = 0;
    N.log_size(prog, &ls);
    std::string log(ls, '\0');
    if (ls) N.log(prog, &log[0]);
    N.destroy(&prog);
    fail(PRISM_ERR_INTERNAL, "run-time kernel compilation failed:\n" + log);
  }
  size_t n = 0;
  N.cubin_size(prog, &n);
  std::vector<char> cubin(n);
  N.cubin(prog, cubin.data());
  N.destroy(&prog);
  cudaLibrary_t lib = nullptr;
  PRISM_CUDA(cudaLibraryLoadData(&lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
  return lib;
}

const void* jit_get(const std::string& source, const char* name) {
  std::unique_lock<std::mutex> lk(g_mu);
  auto it = g_cache.find(source);
  if (it == g_cache.end()) {
    g_cache.emplace(source, Entry{});  // this thread compiles it
    lk.unlock();
    auto t0 = std::chrono::steady_clock::now();
    cudaLibrary_t lib = nullptr;
    try {
      lib = compile_source(source);
    } catch (...) {
      lk.lock();
      g_cache.erase(source);
      g_cv.notify_all();
      throw;
    }
    lk.lock();
    it = g_cache.find(source);
    it->second.lib = lib;
    it->second.ready = true;
    g_compiles += 1;
    g_compile_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    g_cv.notify_all();
  } else if (!it->second.ready) {
    g_cv.wait(lk, [&] {
      auto f = g_cache.find(source);
      return f == g_cache.end() || f->second.ready;
    });
    it = g_cache.find(source);
    if (it == g_cache.end()) fail(PRISM_ERR_INTERNAL, "run-time kernel compilation failed in another thread");
  }
  auto kt = it->second.kernels.find(name);
  if (kt == it->second.kernels.end()) {
    cudaKernel_t k;
    PRISM_CUDA(cudaLibraryGetKernel(&k, it->second.lib, name));
    kt = it->second.kernels.emplace(name, k).first;
  }
  return reinterpret_cast<const void*>(kt->second);
}

namespace {

// The per-row logic every generated aggregation kernel shares: filter
// (keep), operands (values, value, slow) and the op kind / fast-path tables.
struct RowParts {
  std::string keep, value, values_body, slow, slow_cols, kinds, i64;
  bool ok = true;
};

RowParts row_parts(Gen& gen, const AggArgs& a) {
  RowParts rp;
  gen.declare_cols();
  if (a.has_filter) {
    auto p = gen.pred(a.filter.begin, a.filter.len);
    gen.out << "    return " << p.first << " && " << p.second << ";\n";
  } else {
    gen.out << "    return true;\n";
  }
  rp.keep = gen.take();
  // operands
  gen.declare_cols();
  gen.out << "    Val r; r.i = 0; r.f = 0; r.valid = true;\n";
  std::ostringstream kinds, slow, i64;
  for (int j = 0; j < a.n_ops; ++j) {
    const Op& o = a.op[j];
    if (o.kind == O_DISTINCT || o.src < 0 || o.src >= a.n_src) {
      rp.ok = false;
      return rp;
    }
    kinds << (j ? ", " : "") << o.kind;
    bool narrow = false;  // value fits int64 whenever the row's slow flag is clear
    const Src& sr = a.src[o.src];
    gen.out << "    " << (j ? "else " : "") << "if (j == " << j << ") {\n";
    switch (sr.kind) {
      case S_COL_F64: {
        std::string c = gen.col(sr.col);
        gen.out << "    r.f = " << gen.rd_cast("dcol_fval", "0.0", sr.col) << "; r.valid = " << gen.V(sr.col) << ";\n";
        break;
      }
      case S_COL_INT: {
        narrow = true;
        std::string c = gen.col(sr.col);
        gen.out << "    r.i = " << gen.rd_cast("dcol_ival", "0LL", sr.col) << "; r.valid = " << gen.V(sr.col) << ";\n";
        break;
      }
      case S_COL_I128: {
        std::string c = gen.col(sr.col);
        gen.out << "    r.i = " << gen.rd_cast("dcol_i128", "(__int128)0", sr.col) << "; r.valid = " << gen.V(sr.col) << ";\n";
        break;
      }
      case S_VALID: {
        std::string c = gen.col(sr.col);
        gen.out << "    r.valid = " << gen.V(sr.col) << ";\n";
        break;
      }
      default: {
        std::string fval, fvalid, fok;
        bool fast = sr.kind == S_EXPR_I128 && gen.expr_fast64(sr.begin, sr.end, fval, fvalid, fok);
        narrow = fast;
        if (fast) {
          // 64-bit steps here; when one of them overflowed, flag bit 2j asks
          // the caller for the 128-bit program (out of line in slow(), so it
          // costs the hot loop no registers and no ordering of its loads)
          gen.out << "    r.i = (__int128)" << fval << "; r.valid = " << fvalid << "; if (!" << fok << ") flags |= "
                  << (1u << (2 * j)) << "u;\n";
          std::string body = gen.take();
          gen.out << "    if (j == " << j << ") {\n    bool ovf = false;\n";
          std::string v = gen.expr(sr.begin, sr.end, "ovf");
          gen.out << "    SlowVal s; s.v = " << v << "; s.ovf = ovf;\n    return s;\n    }\n";
          slow << gen.take();
          gen.out << body;
        } else {
          // overflow is reported through flag bit 2j+1, never raised here
          gen.out << "    bool ovf = false;\n";
          std::string v = gen.expr(sr.begin, sr.end, "ovf");
          gen.out << "    r = " << v << ";\n    if (ovf) flags |= " << (2u << (2 * j)) << "u;\n";
        }
      }
    }
    gen.out << "    }\n";
    i64 << (j ? ", " : "") << (narrow ? "true" : "false");
  }
  gen.out << "    return r;\n";
  rp.value = gen.take();
  // values(): every op of a row in one straight-line body (the hot path);
  // subtrees shared between ops' 64-bit programs are computed once
  gen.declare_cols();
  gen.cse = true;
  gen.cse_map.clear();
  for (int j = 0; j < a.n_ops; ++j) {
    const Src& sr = a.src[a.op[j].src];
    std::string o = "out[" + std::to_string(j) + "]";
    switch (sr.kind) {
      case S_COL_F64:
        gen.col(sr.col);
        gen.out << "    " << o << ".i = 0; " << o << ".f = " << gen.rd_cast("dcol_fval", "0.0", sr.col) << "; " << o
                << ".valid = " << gen.V(sr.col) << ";\n";
        break;
      case S_COL_INT:
        gen.col(sr.col);
        gen.out << "    " << o << ".f = 0; " << o << ".i = " << gen.rd_cast("dcol_ival", "0LL", sr.col) << "; " << o
                << ".valid = " << gen.V(sr.col) << ";\n";
        break;
      case S_COL_I128:
        gen.col(sr.col);
        gen.out << "    " << o << ".f = 0; " << o << ".i = " << gen.rd_cast("dcol_i128", "(__int128)0", sr.col) << "; " << o
                << ".valid = " << gen.V(sr.col) << ";\n";
        break;
      case S_VALID:
        gen.col(sr.col);
        gen.out << "    " << o << ".i = 0; " << o << ".f = 0; " << o << ".valid = " << gen.V(sr.col) << ";\n";
        break;
      default: {
        std::string fval, fvalid, fok;
        if (sr.kind == S_EXPR_I128 && gen.expr_fast64(sr.begin, sr.end, fval, fvalid, fok)) {
          gen.out << "    " << o << ".f = 0; " << o << ".i = (__int128)" << fval << "; " << o << ".valid = " << fvalid
                  << "; if (!" << fok << ") flags |= " << (1u << (2 * j)) << "u;\n";
        } else {
          gen.out << "    {\n    bool ovf = false;\n";
          std::string v = gen.expr(sr.begin, sr.end, "ovf");
          gen.out << "    " << o << " = " << v << ";\n    if (ovf) flags |= " << (2u << (2 * j)) << "u;\n    }\n";
        }
      }
    }
  }
  gen.cse = false;
  rp.values_body = gen.take();
  gen.declare_cols();
  rp.slow_cols = gen.take();
  rp.slow = slow.str();
  rp.kinds = kinds.str();
  rp.i64 = i64.str();
  rp.ok = gen.ok;
  return rp;
}

// struct QueryRow: E of the kernel bodies in agg_device.cuh. `members`
// adds the body-specific functions and layout constants.
std::string query_row(Gen& gen, const Batch& b, const AggArgs& a, const RowParts& rp, const std::string& members) {
  // row indices address the longest column (a joined batch's build side
  // may be longer than its probe rows)
  int64_t max_rows = b.rows;
  for (auto& c : b.cols) max_rows = std::max<int64_t>(max_rows, c->length);
  std::string consts = gen.consts.str();
  if (consts.empty()) consts = "    int unused;\n";
  std::ostringstream s;
  s << "#include \"agg_device.cuh\"\n"
       "namespace prism {\n"
       "struct QueryRow {\n"
       "  typedef "
    << (max_rows < ((int64_t)1 << 31) - ((int64_t)1 << 26) ? "int" : "long long")
    << " idx_t;  // row index type: 32-bit below 2^31 rows\n"
       "  struct Consts {\n"
    << consts
    << "  };\n"
    << gen.row_struct()
    << "  static __device__ __forceinline__ Consts load(const AggArgs& a) {\n    Consts K;\n"
    << gen.load.str()
    << "    return K;\n  }\n"
       "  static __device__ __forceinline__ bool keep(const AggArgs& a, const Consts& K, const DCol* cols, idx_t idx, "
       "idx_t bidx, const Row& row) {\n"
    << rp.keep << "  }\n"
    << members
    << "  static constexpr bool kSkipNulls = " << (a.skip_nulls ? "true" : "false") << ";\n"
    << "  static constexpr int kKind[" << a.n_ops << "] = {" << rp.kinds << "};\n"
    << "  static constexpr bool kI64[" << a.n_ops << "] = {" << rp.i64 << "};\n"
    << "  // every op's exact value, out of line: 128-bit programs for ops with a\n"
       "  // 64-bit fast path, value() itself for the others\n"
       "  static __device__ __noinline__ SlowVal slow(const AggArgs& a, int j, const DCol* cols, idx_t idx, idx_t bidx) {\n"
       "    const Consts K = load(a);\n    const Row row = fetch(cols, idx, bidx);\n"
    << rp.slow_cols << rp.slow
    << "    unsigned fl = 0;\n    SlowVal s;\n    s.v = value(a, K, j, cols, idx, bidx, row, fl);\n"
       "    s.ovf = ((fl >> (2 * j + 1)) & 1u) != 0;\n    return s;\n  }\n"
    << "  static __device__ __forceinline__ void values(const AggArgs& a, const Consts& K, const DCol* cols, idx_t idx, "
       "idx_t bidx, const Row& row, Val* out, unsigned& flags) {\n"
    << rp.values_body << "  }\n"
    << "  static __device__ __forceinline__ Val value(const AggArgs& a, const Consts& K, int j, const DCol* cols, "
       "idx_t idx, idx_t bidx, const Row& row, unsigned& flags) {\n"
    << rp.value
    << "  }\n"
       "};\n"
       "}  // namespace prism\n";
  return s.str();
}

std::string query_row_kernel(const AggArgs& a, int n_probe_cols, const JoinKernelShape& join) {
  std::ostringstream k;
  if (n_probe_cols >= 0)
    k << "extern \"C\" __global__ void __launch_bounds__(" << join.block << ", " << join.min_blocks
      << ") prism_join_agg(prism::AggArgs a) {\n  prism::join_body<prism::QueryRow, " << a.n_ops << ", " << join.block
      << ", " << join.rows << ", " << (a.jent ? "true" : "false") << ", " << (a.jmatch ? "true" : "false") << ", "
      << (a.jkw ? "true" : "false") << ">(a);\n}\n";
  else
    k << "extern \"C\" __global__ void __launch_bounds__(" << join.hash_block << ", 1) prism_hash_agg(prism::AggArgs a) {\n"
         "  prism::hash_body<prism::QueryRow, " << a.n_ops << ", " << join.hash_block << ">(a);\n}\n";
  return k.str();
}

}  // namespace

namespace {

template <class T>
void key_put(std::string& k, const T& v) {
  k.append(reinterpret_cast<const char*>(&v), sizeof v);
}
void key_str(std::string& k, const std::string& v) {
  key_put(k, (uint64_t)v.size());
  k.append(v);
}
template <class P>
void key_nonnull(P*& p) {
  p = p ? reinterpret_cast<P*>(uintptr_t(1)) : nullptr;
}

bool plan_cache_on() {
  const char* e = std::getenv("PRISM_JIT_PLAN_CACHE");
  return !(e && std::strcmp(e, "0") == 0);
}

std::mutex g_plan_mu;
std::unordered_map<std::string, const void*> g_plan;

}  // namespace

const void* jit_plan_kernel(const Program& pg, const Batch& b, const AggArgs& a0, const std::vector<int64_t>& extra,
                            const char* name, const std::function<std::string()>& make) {
  if (!plan_cache_on()) {
    const std::string src = make();
    return src.empty() ? nullptr : jit_get(src, name);
  }
  std::string k;
  k.reserve(8192);
  key_str(k, name);
  for (int64_t x : extra) key_put(k, x);
  // the kernel arguments, pointers as null / non-null
  AggArgs a;
  std::memcpy(&a, &a0, sizeof a);
  key_nonnull(a.pn);
  key_nonnull(a.en);
  key_nonnull(a.cl);
  key_nonnull(a.cols);
  key_nonnull(a.gkeys);
  key_nonnull(a.gfirst);
  key_nonnull(a.gacc);
  key_nonnull(a.jslots);
  key_nonnull(a.jdup);
  key_nonnull(a.jdense);
  key_nonnull(a.jpk);
  key_nonnull(a.jbk);
  key_nonnull(a.jkrec);
  key_nonnull(a.jent);
  key_nonnull(a.jmatch);
  key_nonnull(a.jinl);
  key_nonnull(a.gnew);
  key_nonnull(a.gnew_count);
  for (auto& d : a.dt) key_nonnull(d.slots);
  key_nonnull(a.err);
  key_nonnull(a.maxexp);
  key_nonnull(a.gwide);
  key_put(k, a);
  // the program's host arrays
  key_put(k, (uint64_t)pg.cols.size());
  for (int c : pg.cols) key_put(k, c);
  key_put(k, (uint64_t)pg.pnodes.size());
  for (PNode n : pg.pnodes) {
    key_nonnull(n.s);
    key_put(k, n);
  }
  key_put(k, (uint64_t)pg.clauses.size());
  for (const PRange& r : pg.clauses) key_put(k, r);
  key_put(k, (uint64_t)pg.enodes.size());
  for (const ENode& e : pg.enodes) key_put(k, e);
  key_put(k, (uint64_t)pg.strings.size());
  for (const std::string& x : pg.strings) key_str(k, x);
  for (int i : pg.string_node) key_put(k, i);
  key_put(k, (int32_t)pg.has_filter);
  key_put(k, pg.filter);
  key_put(k, (uint64_t)pg.exprs.size());
  for (const CompiledExpr& e : pg.exprs) {
    key_put(k, e.kind);
    key_put(k, e.begin);
    key_put(k, e.end);
    key_put(k, e.scale);
    key_put(k, e.out_type);
    key_put(k, e.column);
    prism_scalar lit = e.literal;
    key_nonnull(lit.str);
    key_put(k, lit);
    key_str(k, e.literal_str);
    for (int32_t c : e.branch_cols) key_put(k, c);
    for (const std::string& x : e.branch_lits) key_str(k, x);
    key_put(k, e.sel_clause_begin);
    key_put(k, e.sel_n_clauses);
    key_put(k, (int32_t)e.sel_has_else);
  }
  // the row count and every column's type and attributes (not its data)
  key_put(k, b.rows);
  key_put(k, (uint64_t)b.cols.size());
  for (const ColP& c : b.cols) {
    key_put(k, c->type);
    key_put(k, c->index_type);
    key_put(k, (int32_t)c->nullable);
    key_put(k, c->precision);
    key_put(k, c->scale);
    key_put(k, c->length);
    key_put(k, c->data_base);
    key_put(k, (int32_t)((c->validity ? 1 : 0) | (c->values ? 2 : 0) | (c->offsets ? 4 : 0) | (c->data ? 8 : 0)));
    if (c->dict) {
      key_put(k, c->dict->type);
      key_put(k, c->dict->length);
      key_put(k, c->dict_fingerprint);
    } else {
      key_put(k, (int32_t)-1);
    }
  }
  {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    auto it = g_plan.find(k);
    if (it != g_plan.end()) return it->second;
  }
  const std::string src = make();
  const void* kern = src.empty() ? nullptr : jit_get(src, name);
  std::lock_guard<std::mutex> lk(g_plan_mu);
  g_plan.emplace(std::move(k), kern);
  return kern;
}

std::string jit_tiny_agg_source(const Program& pg, const Batch& b, const AggArgs& a, int g, bool f64) {
  Gen gen(pg, b);
  RowParts rp = row_parts(gen, a);
  if (!rp.ok) return "";
  // dense group id
  gen.declare_cols();
  gen.out << "    int g = 0;\n";
  for (int k = 0; k < a.n_gcols; ++k) {
    std::string c = gen.col(a.gcol[k]);
    // the dense id layout (dictionary sizes) is fixed per plan: constants
    gen.out << "    { int code = " << gen.V(a.gcol[k]) << " ? (int)" << gen.rd("dcol_ival", a.gcol[k]) << " : "
            << a.dnull[k] << "; g += code * " << a.dstride[k] << "; }\n";
  }
  gen.out << "    return g;\n";
  std::string gid = gen.take();
  // tiny layout: words 0, 1 of a group are the row count and first row
  std::ostringstream words;
  int nw = TINY_FIRST_OP_WORD;
  for (int j = 0; j < a.n_ops; ++j) {
    words << (j ? ", " : "") << nw;
    nw += tiny_words(a.op[j].kind);
  }
  const int block = tiny_block((g + 1) * nw);
  if (!gen.ok) return "";
  std::ostringstream m;
  m << "  static __device__ __forceinline__ int gid(const AggArgs& a, const Consts& K, const DCol* cols, idx_t idx, "
       "idx_t bidx, const Row& row) {\n"
    << gid << "  }\n"
    << "  static constexpr int kNW = " << nw << ";\n"
    << "  static constexpr int kWord[" << a.n_ops << "] = {" << words.str() << "};\n";
  std::ostringstream s;
  s << query_row(gen, b, a, rp, m.str())
    << "extern \"C\" __global__ void __launch_bounds__(" << block << ", " << 512 / block << ") prism_tiny_agg(prism::AggArgs a) {\n"
       "  prism::tiny_body<prism::QueryRow, "
    << g << ", " << a.n_ops << ", " << (f64 ? "true" : "false") << ", " << block << ">(a);\n"
       "}\n";
  return s.str();
}

std::string jit_hash_agg_source(const Program& pg, const Batch& b, const AggArgs& a, int n_probe_cols,
                                const JoinKernelShape& join) {
  Gen gen(pg, b);
  if (n_probe_cols >= 0)
    for (size_t s = 0; s < pg.cols.size(); ++s) {
      gen.bside.push_back(pg.cols[s] >= n_probe_cols ? 1 : 0);
      if ((a.jent || a.jmatch) && a.jent_col >= 0 && pg.cols[s] == a.jent_col) gen.inl_slot = (int)s;
    }
  RowParts rp = row_parts(gen, a);
  if (!rp.ok) return "";
  // FxHash of the key columns, as fx_value computes it (common.cuh): fixed
  // width integer and Float64 keys from the fetched row words, any other
  // type by fx_value itself on the column
  gen.declare_cols();
  gen.out << "    uint64_t h = 0;\n";
  for (int k = 0; k < a.n_gcols; ++k) {
    const int slot = a.gcol[k];
    std::string c = gen.col(slot);
    const int t = gen.col_type(slot);
    if (gen.fetched(slot) && (t == TY_I32 || t == TY_I64))
      gen.out << "    h = " << gen.V(slot) << " ? fx_word(h, (uint64_t)dcol_ival(" << c << ", 0)) : fx_word(h, 0);\n";
    else if (gen.fetched(slot) && t == TY_F64)
      gen.out << "    h = " << gen.V(slot) << " ? fx_word(h, (uint64_t)__double_as_longlong(static_cast<const double*>(" << c
              << ".values)[0])) : fx_word(h, 0);\n";
    else
      gen.out << "    h = fx_value(h, cols[" << slot << "], " << gen.rix(slot) << ");\n";
  }
  gen.out << "    return h;\n";
  std::string hash = gen.take();
  std::ostringstream words;
  for (int j = 0; j < a.n_ops; ++j) words << (j ? ", " : "") << a.op[j].word;
  if (!gen.ok) return "";
  std::ostringstream m;
  m << "  static __device__ __forceinline__ uint64_t hash(const AggArgs& a, const Consts& K, const DCol* cols, idx_t idx, "
       "idx_t bidx, const Row& row) {\n"
    << hash << "  }\n"
    << "  static constexpr int kW = " << a.W << ";\n"
    << "  static constexpr bool kCountRows = " << (a.count_rows ? "true" : "false") << ";\n"
    << "  static constexpr int kWord[" << a.n_ops << "] = {" << words.str() << "};\n";
  std::ostringstream s;
  s << query_row(gen, b, a, rp, m.str())
    << query_row_kernel(a, n_probe_cols, join);
  return s.str();
}

}  // namespace prism
