// oracle_arrow.hpp — TEST INFRASTRUCTURE ONLY.
//
// Host-side columnar model of the CPU oracle: zero-copy views over imported
// Arrow C Data Interface arrays, owned column builders, and export back to
// the C Data Interface. Independent of the GPU product's importer so that the
// checker shares no code with the thing it checks.
#pragma once

#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

#include "../include/prism_gpu.h"

namespace oracle {

struct Error {
  int code;
  std::string msg;
};
[[noreturn]] inline void fail(int code, std::string msg) { throw Error{code, std::move(msg)}; }

enum Ty {
  T_NULL, T_BOOL, T_I8, T_I16, T_I32, T_I64, T_U8, T_U16, T_U32, T_U64,
  T_F32, T_F64, T_DATE32, T_UTF8, T_DEC128, T_DICT
};

inline int64_t width_of(Ty t) {
  switch (t) {
    case T_I8: case T_U8: return 1;
    case T_I16: case T_U16: return 2;
    case T_I32: case T_U32: case T_F32: case T_DATE32: return 4;
    case T_I64: case T_U64: case T_F64: return 8;
    case T_DEC128: return 16;
    default: return 0;
  }
}
inline bool is_int_like(Ty t) {
  return t == T_I8 || t == T_I16 || t == T_I32 || t == T_I64 || t == T_U8 || t == T_U16 ||
         t == T_U32 || t == T_U64 || t == T_DATE32;
}

struct Col;
using ColP = std::shared_ptr<Col>;

struct Col {
  Ty ty = T_NULL;
  std::string name;
  bool nullable = true;
  int64_t len = 0;
  const uint8_t* vbits = nullptr;  // validity bitmap (nullptr: all valid)
  int64_t voff = 0;                // bit offset into vbits
  const uint8_t* vals = nullptr;   // values base (BOOL: bitmap)
  int64_t off = 0;                 // element offset (BOOL: bit offset)
  const int32_t* offs = nullptr;   // UTF8 offsets base (index off + i)
  const uint8_t* data = nullptr;   // UTF8 bytes
  ColP dict;                       // T_DICT values
  Ty idx_ty = T_I32;               // T_DICT index type
  int prec = 38, scale = 0;        // T_DEC128
  std::shared_ptr<void> hold;      // owned storage

  bool null_at(int64_t i) const {
    if (ty == T_NULL) return true;
    if (!vbits) return false;
    int64_t b = voff + i;
    return !((vbits[b >> 3] >> (b & 7)) & 1);
  }
  // raw integer value of integer-like / bool / dictionary index columns
  int64_t ival(int64_t i) const {
    int64_t j = off + i;
    Ty t = (ty == T_DICT) ? idx_ty : ty;
    switch (t) {
      case T_BOOL: return (vals[j >> 3] >> (j & 7)) & 1;
      case T_I8: return reinterpret_cast<const int8_t*>(vals)[j];
      case T_I16: return reinterpret_cast<const int16_t*>(vals)[j];
      case T_I32: case T_DATE32: return reinterpret_cast<const int32_t*>(vals)[j];
      case T_I64: return reinterpret_cast<const int64_t*>(vals)[j];
      case T_U8: return vals[j];
      case T_U16: return reinterpret_cast<const uint16_t*>(vals)[j];
      case T_U32: return reinterpret_cast<const uint32_t*>(vals)[j];
      case T_U64: return (int64_t)reinterpret_cast<const uint64_t*>(vals)[j];
      default: fail(PRISM_ERR_INTERNAL, "ival on non-integer column");
    }
  }
  double fval(int64_t i) const {  // arrow cast-to-Float64 of the raw value
    int64_t j = off + i;
    switch (ty) {
      case T_F64: return reinterpret_cast<const double*>(vals)[j];
      case T_F32: return reinterpret_cast<const float*>(vals)[j];
      case T_U64: return (double)reinterpret_cast<const uint64_t*>(vals)[j];
      case T_DEC128: {
        __int128 v = dval(i);
        double p = 1.0;
        for (int k = 0; k < scale; ++k) p *= 10.0;
        return (double)v / p;
      }
      default: return (double)ival(i);
    }
  }
  __int128 dval(int64_t i) const {
    __int128 v;
    std::memcpy(&v, vals + 16 * (off + i), 16);
    return v;
  }
  std::string_view sval(int64_t i) const {
    if (ty == T_DICT) return dict->sval(ival(i));
    int64_t j = off + i;
    int32_t a = offs[j], b = offs[j + 1];
    return std::string_view(reinterpret_cast<const char*>(data) + a, (size_t)(b - a));
  }
  uint64_t fbits(int64_t i) const {
    double d = reinterpret_cast<const double*>(vals)[off + i];
    uint64_t u;
    std::memcpy(&u, &d, 8);
    return u;
  }
};

struct Batch {
  std::vector<ColP> cols;
  int64_t rows = 0;
};

// ---------------------------------------------------------------- builder --
struct Owned {
  std::vector<uint8_t> vbits, vals, data;
  std::vector<int32_t> offs;
};

struct Builder {
  Ty ty;
  std::string name;
  bool nullable = true;
  int prec = 38, scale = 0;
  ColP dict;
  Ty idx_ty = T_I32;
  std::vector<uint8_t> valid;
  bool any_null = false;
  std::vector<uint8_t> raw;
  std::vector<int32_t> offs{0};
  std::vector<uint8_t> data;
  int64_t n = 0;

  Builder(Ty t, std::string nm, bool nul = true) : ty(t), name(std::move(nm)), nullable(nul) {}

  void reserve(int64_t k) {
    valid.reserve(k);
    if (width_of(ty == T_DICT ? idx_ty : ty) > 0)
      raw.reserve(k * width_of(ty == T_DICT ? idx_ty : ty));
  }
  void mark(bool ok) {
    valid.push_back(ok ? 1 : 0);
    if (!ok) any_null = true;
    ++n;
  }
  void push_raw(const void* p, int64_t w) {
    const uint8_t* b = static_cast<const uint8_t*>(p);
    raw.insert(raw.end(), b, b + w);
  }
  // a null row whose slot holds `w` raw bytes (arrow compute kernels fill
  // null slots with the operation applied to the raw operand slots)
  void push_raw_null(const void* p, int64_t w) {
    mark(false);
    push_raw(p, w);
  }
  void push_null() {
    mark(false);
    Ty t = ty == T_DICT ? idx_ty : ty;
    if (t == T_UTF8) offs.push_back((int32_t)data.size());
    else if (t == T_BOOL) raw.push_back(0);
    else if (t != T_NULL) raw.insert(raw.end(), width_of(t), 0);
  }
  void push_i64(int64_t v) {
    mark(true);
    Ty t = ty == T_DICT ? idx_ty : ty;
    switch (t) {
      case T_BOOL: raw.push_back(v ? 1 : 0); break;
      case T_I8: case T_U8: { int8_t x = (int8_t)v; push_raw(&x, 1); break; }
      case T_I16: case T_U16: { int16_t x = (int16_t)v; push_raw(&x, 2); break; }
      case T_I32: case T_U32: case T_DATE32: { int32_t x = (int32_t)v; push_raw(&x, 4); break; }
      case T_I64: case T_U64: push_raw(&v, 8); break;
      case T_F64: { double d = (double)v; push_raw(&d, 8); break; }
      default: fail(PRISM_ERR_INTERNAL, "push_i64 on wrong type");
    }
  }
  void push_f64(double v) {
    mark(true);
    if (ty == T_F64) push_raw(&v, 8);
    else if (ty == T_F32) { float f = (float)v; push_raw(&f, 4); }
    else fail(PRISM_ERR_INTERNAL, "push_f64 on wrong type");
  }
  void push_i128(__int128 v) {
    mark(true);
    push_raw(&v, 16);
  }
  void push_str(std::string_view s) {
    mark(true);
    data.insert(data.end(), s.begin(), s.end());
    if ((int64_t)data.size() > INT32_MAX) fail(PRISM_ERR_ARROW, "utf8 column exceeds 2 GiB");
    offs.push_back((int32_t)data.size());
  }
  // copy row i of c keeping the raw slot of a null row, as arrow-select's
  // filter kernels copy the selected values and bytes regardless of
  // validity (filter_primitive / filter_bytes, arrow 57)
  void push_slot(const Col& c, int64_t i) {
    if (!c.null_at(i)) { push_from(c, i); return; }
    Ty t = c.ty == T_DICT ? c.idx_ty : c.ty;
    int64_t w = width_of(t);
    if (t == T_UTF8) {
      mark(false);
      std::string_view v = c.sval(i);
      data.insert(data.end(), v.begin(), v.end());
      offs.push_back((int32_t)data.size());
    } else if (t == T_BOOL) {
      mark(false);
      raw.push_back((uint8_t)(c.ival(i) ? 1 : 0));
    } else if (w > 0) {
      mark(false);
      push_raw(c.vals + w * (c.off + i), w);
    } else {
      push_null();
    }
  }
  // copy row i of c (same type family) into this builder
  void push_from(const Col& c, int64_t i) {
    if (c.null_at(i)) { push_null(); return; }
    switch (c.ty) {
      case T_UTF8: push_str(c.sval(i)); break;
      case T_F64: case T_F32: {
        mark(true);
        int64_t w = width_of(c.ty);
        push_raw(c.vals + w * (c.off + i), w);
        break;
      }
      case T_DEC128: push_i128(c.dval(i)); break;
      case T_NULL: push_null(); break;
      default: push_i64(c.ival(i)); break;  // ints, bool, date, dict index
    }
  }
  ColP finish() {
    auto own = std::make_shared<Owned>();
    auto col = std::make_shared<Col>();
    col->ty = ty;
    col->name = name;
    col->nullable = nullable;
    col->len = n;
    col->prec = prec;
    col->scale = scale;
    col->dict = dict;
    col->idx_ty = idx_ty;
    if (any_null) {
      own->vbits.assign((n + 7) / 8 + 1, 0);
      for (int64_t i = 0; i < n; ++i)
        if (valid[i]) own->vbits[i >> 3] |= (uint8_t)(1u << (i & 7));
    }
    Ty t = ty == T_DICT ? idx_ty : ty;
    if (t == T_BOOL) {
      own->vals.assign((n + 7) / 8 + 1, 0);
      for (int64_t i = 0; i < n; ++i)
        if (raw[i]) own->vals[i >> 3] |= (uint8_t)(1u << (i & 7));
    } else {
      own->vals = std::move(raw);
      own->vals.resize(own->vals.size() + 16);  // never a null pointer
    }
    if (t == T_UTF8) {
      own->offs = std::move(offs);
      own->data = std::move(data);
      own->data.resize(own->data.size() + 1);
    }
    col->vbits = any_null ? own->vbits.data() : nullptr;
    col->vals = own->vals.data();
    col->offs = t == T_UTF8 ? own->offs.data() : nullptr;
    col->data = t == T_UTF8 ? own->data.data() : nullptr;
    col->hold = own;
    return col;
  }
};

inline Builder builder_like(const Col& c, const std::string& name, bool nullable) {
  Builder b(c.ty, name, nullable);
  b.prec = c.prec;
  b.scale = c.scale;
  b.dict = c.dict;
  b.idx_ty = c.idx_ty;
  return b;
}

// ----------------------------------------------------------------- import --
inline bool parse_format(const char* f, Ty& t, int& prec, int& scale) {
  std::string s(f);
  if (s == "n") t = T_NULL;
  else if (s == "b") t = T_BOOL;
  else if (s == "c") t = T_I8;
  else if (s == "C") t = T_U8;
  else if (s == "s") t = T_I16;
  else if (s == "S") t = T_U16;
  else if (s == "i") t = T_I32;
  else if (s == "I") t = T_U32;
  else if (s == "l") t = T_I64;
  else if (s == "L") t = T_U64;
  else if (s == "f") t = T_F32;
  else if (s == "g") t = T_F64;
  else if (s == "tdD") t = T_DATE32;
  else if (s == "u") t = T_UTF8;
  else if (s.rfind("d:", 0) == 0) {
    t = T_DEC128;
    int p = 0, sc = 0, bw = 128;
    int k = sscanf(s.c_str() + 2, "%d,%d,%d", &p, &sc, &bw);
    if (k < 2 || bw != 128) return false;
    prec = p;
    scale = sc;
  } else return false;
  return true;
}

inline ColP import_col(const ArrowArray* a, const ArrowSchema* s, int64_t extra_off) {
  auto c = std::make_shared<Col>();
  c->name = s->name ? s->name : "";
  c->nullable = (s->flags & ARROW_FLAG_NULLABLE) != 0;
  c->len = a->length;
  Ty t;
  int prec = 38, scale = 0;
  if (!parse_format(s->format, t, prec, scale))
    fail(PRISM_ERR_ARROW, std::string("unsupported arrow format '") + s->format + "'");
  c->prec = prec;
  c->scale = scale;
  int64_t off = a->offset + extra_off;
  if (s->dictionary) {
    if (!is_int_like(t) || t == T_DATE32) fail(PRISM_ERR_ARROW, "bad dictionary index type");
    c->ty = T_DICT;
    c->idx_ty = t;
    c->dict = import_col(a->dictionary, s->dictionary, 0);
  } else {
    c->ty = t;
  }
  if (t == T_NULL) return c;
  c->vbits = (a->null_count != 0 && a->buffers[0]) ? static_cast<const uint8_t*>(a->buffers[0]) : nullptr;
  c->voff = off;
  c->off = off;
  if (c->ty == T_UTF8) {
    c->offs = static_cast<const int32_t*>(a->buffers[1]);
    c->data = static_cast<const uint8_t*>(a->buffers[2]);
  } else {
    c->vals = static_cast<const uint8_t*>(a->buffers[1]);
  }
  return c;
}

inline Batch import_batch(const ArrowArray* a, const ArrowSchema* s) {
  if (!a || !s) fail(PRISM_ERR_INVALID_ARGUMENT, "null batch");
  if (std::string(s->format) != "+s") fail(PRISM_ERR_ARROW, "batch must be a struct array");
  Batch b;
  b.rows = a->length;
  for (int64_t i = 0; i < s->n_children; ++i) {
    auto c = import_col(a->children[i], s->children[i], a->offset);
    c->len = a->length;
    b.cols.push_back(c);
  }
  return b;
}

// ----------------------------------------------------------------- export --
struct SchemaPriv {
  std::string format, name;
  std::vector<ArrowSchema*> children;
  ArrowSchema* dict = nullptr;
};
inline void release_schema(ArrowSchema* s) {
  if (!s || !s->release) return;
  auto* p = static_cast<SchemaPriv*>(s->private_data);
  for (auto* ch : p->children) {
    if (ch->release) ch->release(ch);
    delete ch;
  }
  if (p->dict) {
    if (p->dict->release) p->dict->release(p->dict);
    delete p->dict;
  }
  delete p;
  s->release = nullptr;
}
struct ArrayPriv {
  ColP col;
  std::vector<const void*> bufs;
  std::vector<ArrowArray*> children;
  ArrowArray* dict = nullptr;
};
inline void release_array(ArrowArray* a) {
  if (!a || !a->release) return;
  auto* p = static_cast<ArrayPriv*>(a->private_data);
  for (auto* ch : p->children) {
    if (ch->release) ch->release(ch);
    delete ch;
  }
  if (p->dict) {
    if (p->dict->release) p->dict->release(p->dict);
    delete p->dict;
  }
  delete p;
  a->release = nullptr;
}

inline std::string format_of(const Col& c) {
  switch (c.ty == T_DICT ? c.idx_ty : c.ty) {
    case T_NULL: return "n";
    case T_BOOL: return "b";
    case T_I8: return "c";
    case T_U8: return "C";
    case T_I16: return "s";
    case T_U16: return "S";
    case T_I32: return "i";
    case T_U32: return "I";
    case T_I64: return "l";
    case T_U64: return "L";
    case T_F32: return "f";
    case T_F64: return "g";
    case T_DATE32: return "tdD";
    case T_UTF8: return "u";
    case T_DEC128: return "d:" + std::to_string(c.prec) + "," + std::to_string(c.scale);
    default: return "n";
  }
}

// Materialise any column (view or owned) into a fresh owned, offset-0 copy.
inline ColP materialize(const Col& c) {
  Builder b = builder_like(c, c.name, c.nullable);
  b.reserve(c.len);
  for (int64_t i = 0; i < c.len; ++i) b.push_from(c, i);
  return b.finish();
}

inline void export_schema_col(const Col& c, ArrowSchema* s) {
  auto* p = new SchemaPriv();
  p->format = format_of(c);
  p->name = c.name;
  s->format = p->format.c_str();
  s->name = p->name.c_str();
  s->metadata = nullptr;
  s->flags = c.nullable ? ARROW_FLAG_NULLABLE : 0;
  s->n_children = 0;
  s->children = nullptr;
  s->dictionary = nullptr;
  if (c.ty == T_DICT) {
    p->dict = new ArrowSchema();
    export_schema_col(*c.dict, p->dict);
    s->dictionary = p->dict;
  }
  s->release = release_schema;
  s->private_data = p;
}

inline void export_array_col(const ColP& in, ArrowArray* a) {
  ColP c = (in->off == 0 && in->voff == 0 && in->hold) ? in : materialize(*in);
  auto* p = new ArrayPriv();
  p->col = c;
  int64_t nulls = 0;
  for (int64_t i = 0; i < c->len; ++i) nulls += c->null_at(i) ? 1 : 0;
  a->length = c->len;
  a->null_count = c->ty == T_NULL ? c->len : nulls;
  a->offset = 0;
  a->n_children = 0;
  a->children = nullptr;
  a->dictionary = nullptr;
  if (c->ty == T_NULL) {
    a->n_buffers = 0;
  } else if (c->ty == T_UTF8) {
    p->bufs = {nulls ? c->vbits : nullptr, c->offs, c->data};
  } else {
    p->bufs = {nulls ? c->vbits : nullptr, c->vals};
  }
  a->n_buffers = (int64_t)p->bufs.size();
  a->buffers = p->bufs.data();
  if (c->ty == T_DICT) {
    p->dict = new ArrowArray();
    export_array_col(c->dict, p->dict);
    a->dictionary = p->dict;
  }
  a->release = release_array;
  a->private_data = p;
}

inline void export_batch(const Batch& b, ArrowArray* a, ArrowSchema* s) {
  // nullability check done by RecordBatch::try_new in arrow-rs
  for (auto& c : b.cols) {
    if (!c->nullable)
      for (int64_t i = 0; i < c->len; ++i)
        if (c->null_at(i))
          fail(PRISM_ERR_ARROW, "Invalid argument error: Column '" + c->name +
                                    "' is declared as non-nullable but contains null values");
    if (c->len != b.rows) fail(PRISM_ERR_INTERNAL, "column length mismatch on export");
  }
  auto* sp = new SchemaPriv();
  sp->format = "+s";
  sp->name = "";
  for (auto& c : b.cols) {
    auto* cs = new ArrowSchema();
    export_schema_col(*c, cs);
    sp->children.push_back(cs);
  }
  s->format = sp->format.c_str();
  s->name = sp->name.c_str();
  s->metadata = nullptr;
  s->flags = 0;
  s->n_children = (int64_t)sp->children.size();
  s->children = sp->children.data();
  s->dictionary = nullptr;
  s->release = release_schema;
  s->private_data = sp;

  auto* ap = new ArrayPriv();
  ap->bufs = {nullptr};
  for (auto& c : b.cols) {
    auto* ca = new ArrowArray();
    export_array_col(c, ca);
    ap->children.push_back(ca);
  }
  a->length = b.rows;
  a->null_count = 0;
  a->offset = 0;
  a->n_buffers = 1;
  a->buffers = ap->bufs.data();
  a->n_children = (int64_t)ap->children.size();
  a->children = ap->children.data();
  a->dictionary = nullptr;
  a->release = release_array;
  a->private_data = ap;
}

}  // namespace oracle
