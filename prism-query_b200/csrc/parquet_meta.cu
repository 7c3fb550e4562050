// parquet_meta.cu — host side of the Parquet scan: the Thrift compact
// protocol reader for the footer (FileMetaData) and page headers, and the
// file listing. Field ids and enum values are those of parquet.thrift.
#include <dirent.h>
#include <sys/stat.h>

#include <algorithm>
#include <cstring>
#include <functional>

#include "parquet.hpp"

namespace prism {
namespace pq {

namespace {

// Thrift compact protocol types
enum TType : int { T_STOP = 0, T_TRUE = 1, T_FALSE = 2, T_BYTE = 3, T_I16 = 4, T_I32 = 5, T_I64 = 6, T_DOUBLE = 7,
                   T_BINARY = 8, T_LIST = 9, T_SET = 10, T_MAP = 11, T_STRUCT = 12 };

[[noreturn]] void bad(const char* what) { fail(PRISM_ERR_INTERNAL, std::string("parquet metadata: ") + what); }

struct TReader {
  const uint8_t* p;
  const uint8_t* end;
  int depth = 0;

  uint8_t byte() {
    if (p >= end) bad("truncated");
    return *p++;
  }
  uint64_t varint() {
    uint64_t v = 0;
    for (int s = 0;; s += 7) {
      if (s > 63) bad("varint too long");
      const uint8_t b = byte();
      v |= (uint64_t)(b & 0x7f) << s;
      if (!(b & 0x80)) return v;
    }
  }
  int64_t zz() {
    const uint64_t v = varint();
    return (int64_t)(v >> 1) ^ -(int64_t)(v & 1);
  }
  int32_t i32() { return (int32_t)zz(); }
  std::string binary() {
    const uint64_t n = varint();
    if (n > (uint64_t)(end - p)) bad("binary field runs past the end");
    std::string s(reinterpret_cast<const char*>(p), (size_t)n);
    p += n;
    return s;
  }
  // next field header of a struct; false at STOP
  bool field(int& last, int& id, int& type) {
    const uint8_t b = byte();
    if (b == 0) return false;
    type = b & 0x0f;
    const int delta = b >> 4;
    id = delta ? last + delta : (int)(int16_t)zz();
    last = id;
    return true;
  }
  void list_header(int64_t& n, int& etype) {
    const uint8_t b = byte();
    n = b >> 4;
    etype = b & 0x0f;
    if (n == 15) n = (int64_t)varint();
    if (n < 0 || n > (int64_t)(end - p) * 8 + 15) bad("list size out of range");
  }
  void skip(int type) {
    if (++depth > 64) bad("nesting too deep");
    switch (type) {
      case T_TRUE: case T_FALSE: break;
      case T_BYTE: byte(); break;
      case T_I16: case T_I32: case T_I64: varint(); break;
      case T_DOUBLE:
        if (end - p < 8) bad("truncated");
        p += 8;
        break;
      case T_BINARY: binary(); break;
      case T_LIST: case T_SET: {
        int64_t n;
        int et;
        list_header(n, et);
        for (int64_t i = 0; i < n; ++i) {
          if (et == T_TRUE || et == T_FALSE) byte();
          else skip(et);
        }
        break;
      }
      case T_MAP: {
        const uint64_t n = varint();
        if (n) {
          const uint8_t kv = byte();
          for (uint64_t i = 0; i < n; ++i) {
            skip(kv >> 4);
            skip(kv & 0x0f);
          }
        }
        break;
      }
      case T_STRUCT: {
        int last = 0, id, t;
        while (field(last, id, t)) skip(t);
        break;
      }
      default: bad("unknown field type");
    }
    --depth;
  }
  // iterate a struct's fields: fn(id, type) must consume the value (or skip)
  void each(const std::function<void(int, int)>& fn) {
    if (++depth > 64) bad("nesting too deep");
    int last = 0, id, t;
    while (field(last, id, t)) fn(id, t);
    --depth;
  }
  template <class F>
  void each_in_list(F fn) {
    int64_t n;
    int et;
    list_header(n, et);
    for (int64_t i = 0; i < n; ++i) fn(et);
  }
  bool boolean(int t) { return t == T_TRUE; }
};

Stats read_stats(TReader& r) {
  Stats s;
  std::string old_min, old_max;
  bool has_old_min = false, has_old_max = false;
  r.each([&](int id, int t) {
    if (id == 1 && t == T_BINARY) { old_max = r.binary(); has_old_max = true; }
    else if (id == 2 && t == T_BINARY) { old_min = r.binary(); has_old_min = true; }
    else if (id == 5 && t == T_BINARY) { s.max = r.binary(); s.has_max = true; }
    else if (id == 6 && t == T_BINARY) { s.min = r.binary(); s.has_min = true; }
    else r.skip(t);
  });
  // min_value / max_value when written, else the deprecated min / max
  if (!s.has_min && !s.has_max) {
    s.min = old_min;
    s.max = old_max;
    s.has_min = has_old_min;
    s.has_max = has_old_max;
  }
  return s;
}

ColumnChunk read_column_meta(TReader& r) {
  ColumnChunk c;
  r.each([&](int id, int t) {
    switch (id) {
      case 1: c.type = r.i32(); break;
      case 3: r.each_in_list([&](int et) { if (et == T_BINARY) c.path.push_back(r.binary()); else r.skip(et); }); break;
      case 4: c.codec = r.i32(); break;
      case 5: c.num_values = r.zz(); break;
      case 7: c.total_compressed = r.zz(); break;
      case 9: c.data_page_offset = r.zz(); break;
      case 11: c.dict_page_offset = r.zz(); break;
      case 12: c.stats = read_stats(r); c.has_stats = true; break;
      default: r.skip(t);
    }
  });
  return c;
}

RowGroup read_row_group(TReader& r) {
  RowGroup g;
  r.each([&](int id, int t) {
    if (id == 1 && t == T_LIST) {
      r.each_in_list([&](int et) {
        if (et != T_STRUCT) bad("column chunk is not a struct");
        ColumnChunk cc;
        bool have_meta = false;
        r.each([&](int cid, int ct) {
          if (cid == 1 && ct == T_BINARY) {
            r.binary();
            fail(PRISM_ERR_INVALID_ARGUMENT, "parquet: column chunks in other files are not supported");
          } else if (cid == 3 && ct == T_STRUCT) {
            cc = read_column_meta(r);
            have_meta = true;
          } else if (cid == 8 || cid == 9) {
            fail(PRISM_ERR_INVALID_ARGUMENT, "parquet: encrypted columns are not supported");
          } else {
            r.skip(ct);
          }
        });
        if (!have_meta) bad("column chunk without metadata");
        g.columns.push_back(std::move(cc));
      });
    } else if (id == 3) {
      g.num_rows = r.zz();
    } else {
      r.skip(t);
    }
  });
  return g;
}

struct SchemaEl {
  Leaf leaf;
  int32_t num_children = 0;
  bool has_type = false;
};

SchemaEl read_schema_element(TReader& r) {
  SchemaEl e;
  r.each([&](int id, int t) {
    switch (id) {
      case 1: e.leaf.type = r.i32(); e.has_type = true; break;
      case 2: e.leaf.type_length = r.i32(); break;
      case 3: e.leaf.repetition = r.i32(); break;
      case 4: e.leaf.name = r.binary(); break;
      case 5: e.num_children = r.i32(); break;
      case 6: e.leaf.converted = r.i32(); break;
      case 7: e.leaf.scale = r.i32(); break;
      case 8: e.leaf.precision = r.i32(); break;
      case 10:  // LogicalType union: the id of its one member
        r.each([&](int lid, int lt) {
          e.leaf.logical = lid;
          if (lid == 10 && lt == T_STRUCT) {  // IntType {1: bitWidth, 2: isSigned}
            r.each([&](int iid, int it) {
              if (iid == 1 && it == T_BYTE) e.leaf.int_bits = (int8_t)r.byte();
              else if (iid == 2) e.leaf.int_signed = r.boolean(it);
              else r.skip(it);
            });
          } else {
            r.skip(lt);
          }
        });
        break;
      default: r.skip(t);
    }
  });
  return e;
}

}  // namespace

FileMeta parse_footer(const uint8_t* footer, size_t len, int64_t file_size) {
  TReader r{footer, footer + len};
  FileMeta m;
  m.file_size = file_size;
  std::vector<SchemaEl> schema;
  r.each([&](int id, int t) {
    if (id == 2 && t == T_LIST) {
      r.each_in_list([&](int et) {
        if (et != T_STRUCT) bad("schema element is not a struct");
        schema.push_back(read_schema_element(r));
      });
    } else if (id == 3) {
      m.num_rows = r.zz();
    } else if (id == 4 && t == T_LIST) {
      r.each_in_list([&](int et) {
        if (et != T_STRUCT) bad("row group is not a struct");
        m.row_groups.push_back(read_row_group(r));
      });
    } else if (id == 8) {
      fail(PRISM_ERR_INVALID_ARGUMENT, "parquet: encrypted footers are not supported");
    } else {
      r.skip(t);
    }
  });
  if (schema.empty()) bad("empty schema");
  // depth-first: element 0 is the root; its children are the top-level fields
  size_t i = 1;
  std::function<void()> skip_subtree = [&]() {
    if (i >= schema.size()) bad("schema shorter than its child counts");
    const int32_t nc = schema[i].num_children;
    ++i;
    for (int32_t k = 0; k < nc; ++k) skip_subtree();
  };
  for (int32_t f = 0; f < schema[0].num_children; ++f) {
    if (i >= schema.size()) bad("schema shorter than its child counts");
    SchemaEl& e = schema[i];
    Leaf l = e.leaf;
    if (e.num_children > 0 || !e.has_type) {
      l.nested = true;
      skip_subtree();
    } else {
      ++i;
    }
    m.leaves.push_back(l);
  }
  return m;
}

PageHeader parse_page_header(const uint8_t* p, size_t avail) {
  TReader r{p, p + avail};
  PageHeader h;
  r.each([&](int id, int t) {
    switch (id) {
      case 1: h.type = r.i32(); break;
      case 2: h.uncompressed = r.i32(); break;
      case 3: h.compressed = r.i32(); break;
      case 5:  // DataPageHeader
        r.each([&](int did, int dt) {
          if (did == 1) h.num_values = r.i32();
          else if (did == 2) h.encoding = r.i32();
          else if (did == 3) h.def_encoding = r.i32();
          else r.skip(dt);
        });
        break;
      case 7:  // DictionaryPageHeader
        r.each([&](int did, int dt) {
          if (did == 1) h.dict_values = r.i32();
          else if (did == 2) h.encoding = r.i32();
          else r.skip(dt);
        });
        break;
      case 8:  // DataPageHeaderV2
        r.each([&](int did, int dt) {
          switch (did) {
            case 1: h.num_values = r.i32(); break;
            case 2: h.num_nulls = r.i32(); break;
            case 3: h.num_rows = r.i32(); break;
            case 4: h.encoding = r.i32(); break;
            case 5: h.def_len = r.i32(); break;
            case 6: h.rep_len = r.i32(); break;
            case 7: h.v2_compressed = r.boolean(dt); break;
            default: r.skip(dt);
          }
        });
        break;
      default: r.skip(t);
    }
  });
  h.header_bytes = (int32_t)(r.p - p);
  if (h.compressed < 0 || h.uncompressed < 0 || h.num_values < 0 || h.def_len < 0 || h.rep_len < 0)
    bad("negative page size");
  return h;
}

// parquet.thrift ConvertedType / LogicalType ids used here
constexpr int CT_UTF8 = 0, CT_DATE = 6, CT_INT_32 = 17, CT_INT_64 = 18;
constexpr int LT_STRING = 1, LT_DATE = 6, LT_INTEGER = 10;

int32_t arrow_type_of(const Leaf& l) {
  if (l.nested || l.repetition == 2) return TY_NULL;
  switch (l.type) {
    case P_BOOLEAN: return TY_BOOL;
    case P_INT32:
      if (l.converted == CT_DATE || l.logical == LT_DATE) return TY_DATE32;
      if (l.converted >= 0 && l.converted != CT_INT_32) return TY_NULL;
      if (l.logical >= 0 && !(l.logical == LT_INTEGER && l.int_bits == 32 && l.int_signed)) return TY_NULL;
      return TY_I32;
    case P_INT64:
      if (l.converted >= 0 && l.converted != CT_INT_64) return TY_NULL;
      if (l.logical >= 0 && !(l.logical == LT_INTEGER && l.int_bits == 64 && l.int_signed)) return TY_NULL;
      return TY_I64;
    case P_FLOAT: return TY_F32;
    case P_DOUBLE: return TY_F64;
    case P_BYTE_ARRAY:
      if (l.converted == CT_UTF8 || l.logical == LT_STRING) return TY_UTF8;
      return TY_NULL;
    default: return TY_NULL;
  }
}

}  // namespace pq

std::vector<std::string> list_parquet_files(const std::string& uri) {
  std::string path = uri;
  if (path.rfind("file://", 0) == 0) path = path.substr(7);
  else if (path.find("://") != std::string::npos)
    fail(PRISM_ERR_INVALID_ARGUMENT, "only local paths and file:// URIs are readable here: " + uri);
  std::vector<std::string> out;
  struct stat st{};
  if (stat(path.c_str(), &st) != 0) return out;
  if (S_ISREG(st.st_mode)) {
    if (path.size() >= 8 && path.compare(path.size() - 8, 8, ".parquet") == 0) out.push_back(path);
    return out;
  }
  std::function<void(const std::string&, int)> walk = [&](const std::string& dir, int depth) {
    if (depth > 32) return;
    DIR* d = opendir(dir.c_str());
    if (!d) return;
    while (dirent* e = readdir(d)) {
      const std::string nm = e->d_name;
      if (nm == "." || nm == "..") continue;
      const std::string full = dir + (dir.empty() || dir.back() == '/' ? "" : "/") + nm;
      struct stat s{};
      if (stat(full.c_str(), &s) != 0) continue;
      if (S_ISDIR(s.st_mode)) walk(full, depth + 1);
      else if (S_ISREG(s.st_mode) && nm.size() >= 8 && nm.compare(nm.size() - 8, 8, ".parquet") == 0)
        out.push_back(full);
    }
    closedir(d);
  };
  walk(path, 0);
  std::sort(out.begin(), out.end());
  return out;
}

}  // namespace prism
