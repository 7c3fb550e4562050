// parquet.hpp — Parquet scan (native/prism-executor/src/parquet_scan.rs) on
// the GPU: footer and page headers parsed on the host (Thrift compact
// protocol), row groups skipped by their statistics, the selected column
// chunks copied to HBM in one transfer, then Snappy decompression and page
// decoding (RLE / bit-packed levels and dictionary indices, PLAIN values)
// in CUDA kernels, producing device batches.
//
// The reference reads with the `parquet` crate 57.3.0 (arrow-rs) and its
// `snap` 1.1.1 Snappy codec; neither is part of the reference's sources.
// The format follows the published Parquet specification (parquet.thrift,
// Encodings.md) and the Snappy format description.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "runtime.hpp"

namespace prism {
namespace pq {

// parquet.thrift enums
enum PhysType : int32_t { P_BOOLEAN = 0, P_INT32 = 1, P_INT64 = 2, P_INT96 = 3, P_FLOAT = 4, P_DOUBLE = 5,
                          P_BYTE_ARRAY = 6, P_FIXED = 7 };
enum Codec : int32_t { C_UNCOMPRESSED = 0, C_SNAPPY = 1 };
enum PageType : int32_t { PT_DATA = 0, PT_INDEX = 1, PT_DICT = 2, PT_DATA_V2 = 3 };
enum Enc : int32_t { E_PLAIN = 0, E_PLAIN_DICT = 2, E_RLE = 3, E_BIT_PACKED = 4, E_RLE_DICT = 8 };

struct Stats {
  bool has_min = false, has_max = false;
  std::string min, max;  // plain-encoded values (little-endian numbers, raw bytes)
};

struct ColumnChunk {
  int32_t type = -1;
  int32_t codec = 0;
  int64_t num_values = 0;
  int64_t total_compressed = 0;
  int64_t data_page_offset = -1;
  int64_t dict_page_offset = -1;
  std::vector<std::string> path;
  bool has_stats = false;
  Stats stats;
};

struct RowGroup {
  int64_t num_rows = 0;
  std::vector<ColumnChunk> columns;
};

struct Leaf {  // a top-level primitive column (flat schemas)
  std::string name;
  int32_t type = -1;
  int32_t type_length = 0;
  int32_t repetition = 0;  // 0 required, 1 optional, 2 repeated
  int32_t converted = -1;
  int32_t logical = -1;    // LogicalType union member id, -1 when absent
  int32_t int_bits = 0;    // LogicalType INTEGER
  bool int_signed = true;
  int32_t scale = 0, precision = 0;
  bool nested = false;     // part of a group: not supported
};

struct FileMeta {
  int64_t num_rows = 0;
  std::vector<Leaf> leaves;  // one per top-level field
  std::vector<RowGroup> row_groups;
  int64_t file_size = 0;
};

struct PageHeader {
  int32_t type = -1;
  int32_t uncompressed = 0;
  int32_t compressed = 0;
  // data page (v1 / v2)
  int32_t num_values = 0;
  int32_t encoding = 0;
  int32_t def_encoding = E_RLE;
  int32_t num_nulls = 0, num_rows = 0;
  int32_t def_len = 0, rep_len = 0;  // v2
  bool v2_compressed = true;
  // dictionary page
  int32_t dict_values = 0;
  int32_t header_bytes = 0;  // bytes of the Thrift header itself
};

// Parses the footer of a whole file held in memory (the last 8 bytes are
// the footer length and "PAR1"). Fails with PRISM_ERR_ARROW on malformed
// input, PRISM_ERR_INVALID_ARGUMENT on unsupported shapes is left to the
// scan (nested leaves are flagged).
FileMeta parse_footer(const uint8_t* footer, size_t len, int64_t file_size);
// Parses one page header at p (at most `avail` bytes).
PageHeader parse_page_header(const uint8_t* p, size_t avail);

// Arrow type of a leaf (TY_*), or TY_NULL when unsupported.
int32_t arrow_type_of(const Leaf& l);

}  // namespace pq

// A field of ParquetScanConfig.target_schema (parquet_scan.rs:45-50).
struct TargetField {
  std::string name;
  int32_t type = TY_NULL;
  bool nullable = true;
  int32_t precision = 38, scale = 0;
};

struct ParquetScanArgs {
  std::vector<std::string> uris;
  const prism_predicate* predicate = nullptr;
  bool has_projection = false;
  std::vector<int32_t> projection;
  int64_t batch_size = 8192;
  bool skip_expand = false;
  bool has_target = false;
  std::vector<TargetField> target;
};

struct ParquetScanStats {
  int64_t files = 0, row_groups = 0, row_groups_skipped = 0, pages = 0;
  int64_t compressed_bytes = 0, inflated_bytes = 0, decoded_bytes = 0;
};

// parquet_scan (parquet_scan.rs:55-168) into device batches: prepare, then decode.
std::vector<Batch> parquet_scan(Ctx& ctx, const ParquetScanArgs& args, ParquetScanStats* stats);

// The scan in two steps: the selected column chunks of every file read and
// kept in HBM still compressed (with their page tables), then decoded on the
// GPU as often as asked.
struct ParquetPrepared;
std::shared_ptr<ParquetPrepared> parquet_prepare(Ctx& ctx, const ParquetScanArgs& args, ParquetScanStats* stats);
std::vector<Batch> parquet_decode(Ctx& ctx, const ParquetPrepared& p, ParquetScanStats* stats);
int64_t parquet_prepared_rows(const ParquetPrepared& p);
int64_t parquet_prepared_bytes(const ParquetPrepared& p);
// parquet_row_count (parquet_scan.rs:240-266): rows of the row groups the
// predicate might match, from the footers alone.
int64_t parquet_row_count(const std::vector<std::string>& uris, const prism_predicate* predicate);
// The files a URI names (parquet_scan.rs:60-77, object_source.rs:74-103):
// a directory lists every *.parquet below it, a file names itself; sorted.
std::vector<std::string> list_parquet_files(const std::string& uri);

}  // namespace prism
