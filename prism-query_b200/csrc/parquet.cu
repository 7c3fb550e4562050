// parquet.cu — the Parquet scan on the GPU.
//
// Host: list the files, read each footer, skip row groups whose statistics
// rule the predicate out (parquet_scan.rs:338-469, restated), read the
// selected column chunks with pread into page-locked staging, walk their page
// headers, and copy the chunks to HBM in one transfer per file.
// Device, per file:
//   pq_snappy_kernel      one warp per compressed page (or V2 values section)
//   pq_dict_kernel        byte-array dictionaries: value starts and lengths
//   pq_positions_kernel   PLAIN byte-array pages: value starts and lengths
//   pq_page_kernel        one CTA per data page: definition levels (RLE /
//                         bit-packed hybrid) -> validity, then values (PLAIN,
//                         or dictionary indices in the hybrid encoding)
//   Utf8 columns: one scan of all row lengths -> offsets, pq_copy_kernel.
// Output: per row group, device columns; batches of at most batch_size rows
// are views of them (a validity bitmap is re-aligned when a batch starts off
// a byte boundary).
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <thread>

#include "arrow_io.hpp"
#include "parquet.hpp"
#include "prims.hpp"

namespace prism {

namespace {

using namespace pq;

constexpr int PQ_THREADS = 256;
constexpr int PQ_CHUNK = 1024;          // rows per round of a page CTA
constexpr int PQ_RUNS = PQ_CHUNK + 16;  // hybrid runs held per round (a run covers >= 1 value)

enum PqEnc : int32_t { PE_PLAIN = 0, PE_DICT = 1, PE_RLE_BOOL = 2 };

struct PqPage {
  const uint8_t* body;    // V1: the whole page; V2: the values section
  const uint8_t* levels;  // V2: definition levels (no length prefix)
  int64_t out_row;        // first row of the page in its row-group column
  int32_t body_len;
  int32_t levels_len;
  int32_t rows;
  int32_t enc;
  int32_t type;
  int32_t out;            // PqOut slot
  int32_t dict;           // PqDict slot or -1
  int32_t v1;
  int32_t optional;
  int32_t pos_base;       // PLAIN byte arrays: first slot in the positions scratch
};

struct PqOut {
  uint32_t* valid;             // bitmap words, zeroed; null for a required column
  void* values;                // fixed width, or bitmap words for booleans (zeroed)
  uint32_t* lens;              // Utf8: byte length per row
  unsigned long long* srcs;    // Utf8: device address of the row's bytes
};

struct PqDict {
  const uint8_t* body;
  uint32_t* starts;  // byte arrays: offset of value k's bytes in body
  uint32_t* lens;
  int32_t body_len;
  int32_t count;
  int32_t type;
};

struct SnappyJob {
  const uint8_t* src;
  uint8_t* dst;
  int32_t src_len;
  int32_t dst_len;
  int32_t preamble;    // the job starts its stream (reads the length varint)
  int32_t stream_len;  // the stream's uncompressed length
};

// ---------------------------------------------------------------- snappy --
// The Snappy format: a varint of the uncompressed length, then elements whose
// tag's low two bits select a literal (length in the tag, or in 1-4 following
// bytes when the tag says 60-63), or a copy of (length <= 64, offset) with a
// 1-, 2- or 4-byte offset.
//
// A stream longer than 64 KB is cut on the host (snappy_segments) at the 64 KB
// output boundaries that no later copy reaches back across (the reference
// compressor works in independent 64 KB blocks, so every boundary qualifies
// for its streams), and each segment is a job. One warp inflates one job, a
// batch of elements at a time:
//   1. the warp loads 64 input bytes; every lane decodes the element that
//      would start at its byte (its header is within the window);
//   2. a shuffle walk from lane 0 follows the real element starts (up to 32,
//      until the batch writes SNAP_SPAN bytes or meets a literal longer than
//      64 bytes, which gets a batch of its own);
//   3. literals and copies whose source lies before the batch run in
//      parallel, one lane per element; copies that read the batch's own
//      output then run in order, the warp's lanes over their bytes;
//   4. the batch's output goes from shared memory to HBM, consecutive lanes
//      on consecutive bytes.
// The last SNAP_RING output bytes are kept in shared memory (the batch is
// assembled there) for copies with offsets up to SNAP_RING_REACH; longer
// ones read the output in HBM.
constexpr int SNAP_WARPS = 8;
constexpr int SNAP_RING = 8192;  // power of two
constexpr int SNAP_SPAN = 1024;
constexpr int SNAP_RING_REACH = SNAP_RING - 2 * SNAP_SPAN;
constexpr int64_t SNAP_BLOCK = 65536;

__global__ void __launch_bounds__(32 * SNAP_WARPS) pq_snappy_kernel(const SnappyJob* jobs, int n, uint32_t* err) {
  extern __shared__ __align__(16) uint8_t snap_smem[];
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int w = threadIdx.x >> 5;
  const int job = blockIdx.x * SNAP_WARPS + w;
  if (job >= n) return;
  const SnappyJob J = jobs[job];
  uint8_t* const ring = snap_smem + (size_t)w * SNAP_RING;
  const uint8_t* const in = J.src;
  const int64_t in_len = J.src_len;
  uint8_t* const dst = J.dst;
  const int64_t out_len = J.dst_len;
  bool bad = false;
  int64_t ip = 0;
  if (J.preamble) {
    uint32_t ulen = 0;
    int s = 0;
    for (;; s += 7) {
      if (ip >= in_len || s > 28) { bad = true; break; }
      const uint8_t b = in[ip++];  // every lane reads the same bytes
      ulen |= (uint32_t)(b & 0x7f) << s;
      if (!(b & 0x80)) break;
    }
    if (ulen != (uint32_t)J.stream_len) bad = true;
  }
  int64_t op = 0;
  while (!bad && ip < in_len) {
    const int64_t base = ip;
    const uint32_t b0 = base + lane < in_len ? in[base + lane] : 0u;
    const uint32_t b1 = base + 32 + lane < in_len ? in[base + 32 + lane] : 0u;
    uint32_t nb[5];
    nb[0] = b0;
#pragma unroll
    for (int k = 1; k < 5; ++k) {
      const uint32_t x = __shfl_down_sync(FULL, b0, k);
      const uint32_t y = __shfl_sync(FULL, b1, (lane + k) & 31);
      nb[k] = lane + k < 32 ? x : y;
    }
    // the element that would start at this lane's byte
    const uint32_t tag = nb[0];
    const int t = tag & 3;
    int64_t len, elen_in;
    uint32_t off = 0;
    if (t == 0) {
      const int l = (int)(tag >> 2);
      if (l < 60) {
        len = l + 1;
        elen_in = 1 + len;
      } else {
        const int nbytes = l - 59;
        uint32_t v = 0;
        for (int q = 0; q < nbytes; ++q) v |= nb[1 + q] << (8 * q);
        len = (int64_t)v + 1;
        elen_in = 1 + nbytes + len;
      }
    } else if (t == 1) {
      len = ((tag >> 2) & 7) + 4;
      off = ((tag >> 5) << 8) | nb[1];
      elen_in = 2;
    } else if (t == 2) {
      len = (tag >> 2) + 1;
      off = nb[1] | (nb[2] << 8);
      elen_in = 3;
    } else {
      len = (tag >> 2) + 1;
      off = nb[1] | (nb[2] << 8) | (nb[3] << 16) | (nb[4] << 24);
      elen_in = 5;
    }
    // walk the real element starts (uniform across the warp)
    int64_t pos = 0, o = op;
    int cnt = 0;
    int64_t my_o = -1;
    while (cnt < 32 && pos < 32 && base + pos < in_len) {
      const int src_lane = (int)pos;
      const int64_t e_in = __shfl_sync(FULL, elen_in, src_lane);
      const int64_t e_len = __shfl_sync(FULL, len, src_lane);
      const int e_t = __shfl_sync(FULL, t, src_lane);
      const bool long_lit = e_t == 0 && e_len > 64;
      if (cnt > 0 && long_lit) break;
      if (lane == src_lane) my_o = o;
      o += e_len;
      pos += e_in;
      ++cnt;
      if (long_lit || o - op >= SNAP_SPAN) break;
    }
    const bool mine = my_o >= 0;
    // element checks: inside the input, inside the output, copies after the job's start
    bool ok = true;
    if (mine) {
      if (base + lane + elen_in > in_len || my_o + len > out_len) ok = false;
      if (t != 0 && (off == 0 || (int64_t)off > my_o)) ok = false;
    }
    if (__any_sync(FULL, !ok)) {
      bad = true;
      break;
    }
    const int64_t batch_end = o;
    const bool first_long = cnt == 1 && __shfl_sync(FULL, (int)(t == 0 && len > 64), 0);
    // 3a. independent elements, one lane each
    const bool indep_copy = mine && t != 0 && my_o - (int64_t)off + (len < (int64_t)off ? len : (int64_t)off) <= op;
    // (the batch's output goes to the ring only; it is written to HBM by
    // the whole warp at the end of the batch)
    if (mine && t == 0 && len <= 64) {
      const uint8_t* src = in + base + lane + (elen_in - len);
      for (int i = 0; i < (int)len; ++i) ring[(my_o + i) & (SNAP_RING - 1)] = src[i];
    } else if (indep_copy) {
      // byte i of a copy repeats the source's first min(len, off) bytes:
      // source index i % off, kept incrementally
      const bool near = off <= (uint32_t)SNAP_RING_REACH;
      const int64_t s0 = my_o - off;
      uint32_t j = 0;
      for (int i = 0; i < (int)len; ++i) {
        const int64_t p = s0 + j;
        ring[(my_o + i) & (SNAP_RING - 1)] = near ? ring[p & (SNAP_RING - 1)] : dst[p];
        if (++j == off) j = 0;
      }
    }
    __syncwarp();
    if (first_long) {  // one long literal: the warp copies it
      const int64_t L = __shfl_sync(FULL, len, 0);
      const int64_t so = base + __shfl_sync(FULL, elen_in, 0) - L;
      for (int64_t i = lane; i < L; i += 32) {
        const uint8_t v = in[so + i];
        dst[op + i] = v;
        ring[(op + i) & (SNAP_RING - 1)] = v;
      }
      __syncwarp();
    }
    // 3b. copies that read this batch's output, in order
    unsigned dep = __ballot_sync(FULL, mine && t != 0 && !indep_copy);
    while (dep) {
      const int sl = __ffs(dep) - 1;
      dep &= dep - 1;
      const int64_t eo = __shfl_sync(FULL, my_o, sl);
      const uint32_t eoff = __shfl_sync(FULL, off, sl);
      const int el = (int)__shfl_sync(FULL, len, sl);
      // el <= 64: lane i takes bytes i and i + 32 (source index (i mod eoff))
      uint32_t j = (uint32_t)lane % eoff;
      const uint32_t step = 32u % eoff;
      for (int i = lane; i < el; i += 32) {
        const int64_t p = eo - eoff + j;
        ring[(eo + i) & (SNAP_RING - 1)] = ring[p & (SNAP_RING - 1)];
        j += step;
        if (j >= eoff) j -= eoff;
      }
      __syncwarp();
    }
    // the batch's output, ring -> HBM, consecutive lanes on consecutive bytes
    // (a long literal batch wrote HBM directly)
    if (!first_long)
      for (int64_t q = op + lane; q < batch_end; q += 32) dst[q] = ring[q & (SNAP_RING - 1)];
    __syncwarp();
    op = batch_end;
    ip = base + pos;
  }
  if (lane == 0 && (bad || op != out_len || ip != in_len)) atomicOr(err, DERR_CORRUPT);
}

// ------------------------------------------------------- hybrid streams --
// RLE / bit-packed hybrid (Encodings.md): a varint header; an odd header
// starts (header >> 1) groups of 8 bit-packed values (LSB first, bw bits
// each), an even one a run of (header >> 1) copies of a value stored in
// ceil(bw / 8) little-endian bytes.
struct Runs {
  int32_t start[PQ_RUNS];   // value index (within the page) of the run's first value
  int32_t count[PQ_RUNS];
  unsigned long long data[PQ_RUNS];  // RLE: value; bit-packed: address of its bits
  uint8_t rle[PQ_RUNS];
  int32_t n;
};

struct RunCursor {
  const uint8_t* p;
  const uint8_t* end;
  int32_t next;   // value index where the next unparsed run starts
  int32_t bw;
  int32_t bad;
};

__device__ __forceinline__ uint32_t read_bits(const uint8_t* base, const uint8_t* end, int64_t bit, int bw,
                                              bool& bad) {
  const uint8_t* b = base + (bit >> 3);
  const int sh = (int)(bit & 7);
  const int need = (sh + bw + 7) >> 3;
  unsigned long long v = 0;
  for (int k = 0; k < need; ++k) {
    if (b + k >= end) { bad = true; break; }
    v |= (unsigned long long)b[k] << (8 * k);
  }
  return (uint32_t)((v >> sh) & (bw == 32 ? 0xffffffffull : ((1ull << bw) - 1)));
}

// Thread-0 work: the runs that cover value indices [lo, hi); the last run of
// the previous round is kept when it reaches into this one.
__device__ void fill_runs(Runs& R, RunCursor& C, int32_t lo, int32_t hi) {
  int keep = 0;
  if (R.n > 0) {
    const int last = R.n - 1;
    if (R.start[last] + R.count[last] > lo) {
      R.start[0] = R.start[last];
      R.count[0] = R.count[last];
      R.data[0] = R.data[last];
      R.rle[0] = R.rle[last];
      keep = 1;
    }
  }
  R.n = keep;
  while (C.next < hi && R.n < PQ_RUNS && C.p < C.end) {
    uint32_t h = 0;
    int s = 0;
    for (;; s += 7) {
      if (C.p >= C.end || s > 28) { C.bad = 1; return; }
      const uint8_t b = *C.p++;
      h |= (uint32_t)(b & 0x7f) << s;
      if (!(b & 0x80)) break;
    }
    const int i = R.n;
    if (h & 1) {
      const int64_t groups = h >> 1;
      const int64_t bytes = groups * C.bw;
      R.rle[i] = 0;
      R.data[i] = (unsigned long long)C.p;
      R.count[i] = (int32_t)(groups * 8 < ((int64_t)1 << 30) ? groups * 8 : ((int64_t)1 << 30));
      C.p = (C.end - C.p) < bytes ? C.end : C.p + bytes;
    } else {
      const int nb = (C.bw + 7) >> 3;
      uint32_t v = 0;
      for (int k = 0; k < nb; ++k) {
        if (C.p >= C.end) { C.bad = 1; return; }
        v |= (uint32_t)(*C.p++) << (8 * k);
      }
      R.rle[i] = 1;
      R.data[i] = v;
      R.count[i] = (int32_t)((h >> 1) < (1u << 30) ? (h >> 1) : (1u << 30));
    }
    if (R.count[i] == 0) continue;
    R.start[i] = C.next;
    C.next += R.count[i];
    R.n = i + 1;
  }
}

// value j of the stream (its run is among R's); false when no run holds it
__device__ __forceinline__ bool run_value(const Runs& R, const RunCursor& C, int32_t j, uint32_t& v) {
  int lo = 0, hi = R.n - 1, at = -1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    if (R.start[mid] <= j) { at = mid; lo = mid + 1; }
    else hi = mid - 1;
  }
  if (at < 0 || j >= R.start[at] + R.count[at]) return false;
  if (R.rle[at]) { v = (uint32_t)R.data[at]; return true; }
  bool bad = false;
  v = read_bits(reinterpret_cast<const uint8_t*>(R.data[at]), C.end, (int64_t)(j - R.start[at]) * C.bw, C.bw, bad);
  return !bad;
}

__device__ __forceinline__ uint32_t le32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

// The page's level and value sections (a V1 page of an optional column
// carries a 4-byte length before its levels).
__device__ __forceinline__ bool sections(const PqPage& pg, const uint8_t*& lv, int32_t& lvlen, const uint8_t*& vals,
                                         int32_t& vlen) {
  lv = nullptr;
  lvlen = 0;
  vals = pg.body;
  vlen = pg.body_len;
  if (!pg.optional) return true;
  if (!pg.v1) {
    lv = pg.levels;
    lvlen = pg.levels_len;
    return true;
  }
  if (pg.body_len < 4) return false;
  const uint32_t L = le32(pg.body);
  if ((int64_t)L + 4 > pg.body_len) return false;
  lv = pg.body + 4;
  lvlen = (int32_t)L;
  vals = pg.body + 4 + L;
  vlen = pg.body_len - 4 - (int32_t)L;
  return true;
}

// -------------------------------------------- byte-array value positions --
// PLAIN byte arrays are a 4-byte length then the bytes, back to back: the
// starts follow from a walk, one thread per page (or dictionary).
__device__ int32_t walk_byte_arrays(const uint8_t* vals, int32_t vlen, int32_t count, uint32_t* starts, uint32_t* lens) {
  int64_t pos = 0;
  int32_t k = 0;
  for (; k < count; ++k) {
    if (pos + 4 > vlen) break;
    const uint32_t L = le32(vals + pos);
    if ((int64_t)L > vlen - pos - 4) break;
    starts[k] = (uint32_t)(pos + 4);
    lens[k] = L;
    pos += 4 + (int64_t)L;
  }
  return k;
}

__global__ void pq_dict_kernel(PqDict* dicts, int n, uint32_t* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  PqDict& d = dicts[i];
  if (d.type != TY_UTF8) return;
  const int32_t got = walk_byte_arrays(d.body, d.body_len, d.count, d.starts, d.lens);
  if (got != d.count) atomicOr(err, DERR_CORRUPT);
}

__global__ void pq_positions_kernel(const PqPage* pages, const int32_t* list, int n, uint32_t* starts, uint32_t* lens,
                                    int32_t* found, uint32_t* err) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const PqPage& pg = pages[list[i]];
  const uint8_t* lv;
  const uint8_t* vals;
  int32_t lvlen, vlen;
  if (!sections(pg, lv, lvlen, vals, vlen)) {
    atomicOr(err, DERR_CORRUPT);
    found[list[i]] = 0;
    return;
  }
  found[list[i]] = walk_byte_arrays(vals, vlen, pg.rows, starts + pg.pos_base, lens + pg.pos_base);
}

// --------------------------------------------------------- data pages --
__global__ void __launch_bounds__(PQ_THREADS) pq_page_kernel(const PqPage* pages, const PqOut* outs,
                                                              const PqDict* dicts, const uint32_t* pos_starts,
                                                              const uint32_t* pos_lens, const int32_t* pos_found,
                                                              uint32_t* err) {
  __shared__ Runs def_runs, idx_runs;
  __shared__ RunCursor dc, ic;
  __shared__ uint32_t s_word[PQ_CHUNK / 32], s_pre[PQ_CHUNK / 32];
  __shared__ int32_t s_total;
  __shared__ const uint8_t* s_vals;
  __shared__ int32_t s_vlen;
  __shared__ int32_t s_ok;
  const int tid = threadIdx.x;
  const int pi = blockIdx.x;
  const PqPage pg = pages[pi];
  const PqOut O = outs[pg.out];
  if (tid == 0) {
    const uint8_t* lv;
    const uint8_t* vals;
    int32_t lvlen, vlen;
    s_ok = sections(pg, lv, lvlen, vals, vlen) ? 1 : 0;
    s_vals = vals;
    s_vlen = vlen;
    dc = RunCursor{lv, lv + lvlen, 0, 1, 0};
    def_runs.n = 0;
    idx_runs.n = 0;
    ic = RunCursor{nullptr, nullptr, 0, 0, 0};
    if (s_ok && pg.enc == PE_DICT) {
      if (vlen < 1 || vals[0] > 32) s_ok = 0;
      else ic = RunCursor{vals + 1, vals + vlen, 0, vals[0], 0};
    } else if (s_ok && pg.enc == PE_RLE_BOOL) {
      if (vlen < 4 || (int64_t)le32(vals) + 4 > vlen) s_ok = 0;
      else ic = RunCursor{vals + 4, vals + 4 + le32(vals), 0, 1, 0};
    }
  }
  __syncthreads();
  if (!s_ok) {
    if (tid == 0) atomicOr(err, DERR_CORRUPT);
    return;
  }
  const uint8_t* vals = s_vals;
  const int32_t vlen = s_vlen;
  const int32_t npos = pg.enc == PE_PLAIN && pg.type == TY_UTF8 ? pos_found[pi] : 0;
  const PqDict* D = pg.dict >= 0 ? dicts + pg.dict : nullptr;
  int32_t jbase = 0;
  bool bad = false;
  // Each round: warp 0 alone parses the level runs, builds the round's 32
  // validity words, scans their populations and parses the index runs (warp
  // barriers only); then every thread writes values. Two block barriers.
  for (int32_t lo = 0; lo < pg.rows; lo += PQ_CHUNK) {
    const int32_t hi = min(lo + PQ_CHUNK, pg.rows);
    const int nw = (hi - lo + 31) >> 5;
    if (tid < 32) {
    if (pg.optional && tid == 0) fill_runs(def_runs, dc, lo, hi);
    __syncwarp();
    // validity words of this round (definition level 1 = present)
    if (tid < nw) {
      const int32_t r0 = lo + 32 * tid;
      const int32_t nr = min(32, hi - r0);
      uint32_t w = 0;
      if (!pg.optional) {
        w = nr == 32 ? 0xffffffffu : ((1u << nr) - 1);
      } else {
        for (int b = 0; b < nr; ++b) {
          uint32_t lvl = 0;
          if (!run_value(def_runs, dc, r0 + b, lvl)) { bad = true; break; }
          w |= (lvl & 1u) << b;
        }
      }
      s_word[tid] = w;
      if (O.valid) {
        const int64_t bit = pg.out_row + r0;
        const int sh = (int)(bit & 31);
        atomicOr(O.valid + (bit >> 5), w << sh);
        if (sh && (w >> (32 - sh))) atomicOr(O.valid + (bit >> 5) + 1, w >> (32 - sh));
      }
    }
    __syncwarp();
    {  // exclusive scan of the words' populations
      const uint32_t c = tid < nw ? __popc(s_word[tid]) : 0;
      uint32_t x = c;
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (tid >= d) x += y;
      }
      s_pre[tid] = x - c;
      const int32_t tot = (int32_t)__shfl_sync(0xffffffffu, x, 31);
      if (tid == 0) {
        s_total = tot;
        if (pg.enc == PE_DICT || pg.enc == PE_RLE_BOOL) fill_runs(idx_runs, ic, jbase, jbase + tot);
      }
    }
    __syncwarp();
    if (pg.type == TY_BOOL) {
      // bits: one thread per word of 32 rows
      if (tid < nw) {
        const int32_t r0 = lo + 32 * tid;
        const uint32_t w = s_word[tid];
        uint32_t out = 0;
        int32_t j = jbase + (int32_t)s_pre[tid];
        for (int b = 0; b < 32; ++b) {
          if (!((w >> b) & 1)) continue;
          uint32_t v = 0;
          if (pg.enc == PE_PLAIN) {
            if ((int64_t)j >= (int64_t)vlen * 8) bad = true;
            else v = (vals[j >> 3] >> (j & 7)) & 1;
          } else if (!run_value(idx_runs, ic, j, v)) {
            bad = true;
          }
          out |= (v & 1u) << b;
          ++j;
        }
        const int64_t bit = pg.out_row + r0;
        const int sh = (int)(bit & 31);
        uint32_t* ov = static_cast<uint32_t*>(O.values);
        if (out) {
          atomicOr(ov + (bit >> 5), out << sh);
          if (sh && (out >> (32 - sh))) atomicOr(ov + (bit >> 5) + 1, out >> (32 - sh));
        }
      }
    }
    }  // warp 0
    __syncthreads();
    if (pg.type != TY_BOOL) {
      for (int32_t r = lo + tid; r < hi; r += PQ_THREADS) {
        const int w = (r - lo) >> 5, b = (r - lo) & 31;
        const int64_t row = pg.out_row + r;
        const uint32_t word = s_word[w];
        if (!((word >> b) & 1)) {  // a null row: zero length / zero value
          if (pg.type == TY_UTF8) O.lens[row] = 0;
          else if (pg.type == TY_I64 || pg.type == TY_F64) static_cast<unsigned long long*>(O.values)[row] = 0;
          else static_cast<uint32_t*>(O.values)[row] = 0;
          continue;
        }
        const int32_t j = jbase + (int32_t)s_pre[w] + __popc(word & ((1u << b) - 1));
        uint32_t k = 0;
        if (pg.enc == PE_DICT) {
          if (!run_value(idx_runs, ic, j, k) || !D || (int32_t)k >= D->count) { bad = true; continue; }
        }
        switch (pg.type) {
          case TY_I32: case TY_DATE32: case TY_F32: {
            uint32_t v;
            if (pg.enc == PE_DICT) v = le32(D->body + 4 * (size_t)k);
            else if ((int64_t)(j + 1) * 4 > vlen) { bad = true; continue; }
            else v = le32(vals + 4 * (size_t)j);
            static_cast<uint32_t*>(O.values)[row] = v;
            break;
          }
          case TY_I64: case TY_F64: {
            const uint8_t* src;
            if (pg.enc == PE_DICT) src = D->body + 8 * (size_t)k;
            else if ((int64_t)(j + 1) * 8 > vlen) { bad = true; continue; }
            else src = vals + 8 * (size_t)j;
            const unsigned long long v = (unsigned long long)le32(src) | ((unsigned long long)le32(src + 4) << 32);
            static_cast<unsigned long long*>(O.values)[row] = v;
            break;
          }
          case TY_UTF8: {
            if (pg.enc == PE_DICT) {
              O.lens[row] = D->lens[k];
              O.srcs[row] = (unsigned long long)(D->body + D->starts[k]);
            } else {
              if (j >= npos) { bad = true; O.lens[row] = 0; continue; }
              O.lens[row] = pos_lens[pg.pos_base + j];
              O.srcs[row] = (unsigned long long)(vals + pos_starts[pg.pos_base + j]);
            }
            break;
          }
          default: bad = true;
        }
      }
    }
    jbase += s_total;
    __syncthreads();  // warp 0 rewrites the round's words and runs next
  }
  if (tid == 0 && (dc.bad || ic.bad)) bad = true;
  if (bad) atomicOr(err, DERR_CORRUPT);
}

// Row i of a segment: offsets at [seg_row + seg_index + i] (each segment has
// rows + 1 offsets); lengths / addresses at [seg_row + i].
struct SegView {
  int64_t row0;     // first row in the lens array
  int64_t off0;     // first slot in the int32 offsets array
  int64_t rows;
};

__global__ void pq_seg_offsets_kernel(const unsigned long long* g, const SegView* segs, int n_seg, int32_t* off) {
  const int s = blockIdx.y;
  if (s >= n_seg) return;
  const SegView S = segs[s];
  const unsigned long long base = g[S.row0];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= S.rows; i += (int64_t)gridDim.x * blockDim.x)
    off[S.off0 + i] = (int32_t)(g[S.row0 + i] - base);
}

// Copies every row's bytes: one warp per 32 rows, the warp moving one row's
// bytes at a time (lanes over bytes).
__global__ void pq_copy_kernel(const unsigned long long* srcs, const uint32_t* lens, const unsigned long long* g,
                               int64_t n, uint8_t* data) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = warp * 32; base < n; base += nwarps * 32) {
    const int64_t r = base + lane;
    const uint32_t L = r < n ? lens[r] : 0;
    const unsigned long long s = r < n ? srcs[r] : 0;
    const unsigned long long d = r < n ? g[r] : 0;
    if (L <= 16) {  // short strings: each lane its own row
      const uint8_t* sp = reinterpret_cast<const uint8_t*>(s);
      uint8_t* dp = data + d;
      for (uint32_t i = 0; i < L; ++i) dp[i] = sp[i];
    }
    for (int k = 0; k < 32; ++k) {
      const uint32_t Lk = __shfl_sync(0xffffffffu, L, k);
      if (Lk <= 16) continue;
      const uint8_t* sp = reinterpret_cast<const uint8_t*>(__shfl_sync(0xffffffffu, s, k));
      uint8_t* dp = data + __shfl_sync(0xffffffffu, d, k);
      for (uint32_t i = lane; i < Lk; i += 32) dp[i] = sp[i];
    }
  }
}

__global__ void pq_gather_u64_kernel(const unsigned long long* g, const int64_t* at, int n, unsigned long long* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = g[at[i]];
}

// bits [start, start + n) of src into a new bitmap starting at bit 0
__global__ void pq_slice_bits_kernel(const uint32_t* src, int64_t start, int64_t n, uint32_t* dst) {
  const int64_t nw = (n + 31) >> 5;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += (int64_t)gridDim.x * blockDim.x) {
    const int64_t bit = start + 32 * w;
    const int sh = (int)(bit & 31);
    uint64_t v = src[bit >> 5];
    if (sh) v = (v >> sh) | ((uint64_t)src[(bit >> 5) + 1] << (32 - sh));
    uint32_t x = (uint32_t)v;
    const int64_t left = n - 32 * w;
    if (left < 32) x &= (1u << left) - 1;
    dst[w] = x;
  }
}

// ------------------------------------------------------------ host side --
struct SnapSeg {
  int64_t in_off;
  int64_t out_off;
};

// The points a Snappy stream can be cut at: element starts on 64 KB output
// boundaries that no later copy reaches back across. Empty when the stream
// is malformed (it is then inflated whole, and the kernel reports it).
std::vector<SnapSeg> snappy_segments(const uint8_t* p, int64_t n, int64_t out_len) {
  std::vector<SnapSeg> segs;
  int64_t ip = 0;
  uint64_t ulen = 0;
  for (int s = 0;; s += 7) {
    if (ip >= n || s > 28) return {};
    const uint8_t b = p[ip++];
    ulen |= (uint64_t)(b & 0x7f) << s;
    if (!(b & 0x80)) break;
  }
  if ((int64_t)ulen != out_len) return {};
  segs.push_back({0, 0});
  int64_t op = 0;
  while (ip < n) {
    if (op > 0 && op % SNAP_BLOCK == 0 && segs.back().out_off != op) segs.push_back({ip, op});
    const uint8_t tag = p[ip++];
    const int t = tag & 3;
    int64_t len;
    if (t == 0) {
      len = (tag >> 2) + 1;
      if (len > 60) {
        const int nb = (int)len - 60;
        if (n - ip < nb) return {};
        uint32_t v = 0;
        for (int q = 0; q < nb; ++q) v |= (uint32_t)p[ip + q] << (8 * q);
        ip += nb;
        len = (int64_t)v + 1;
      }
      if (n - ip < len) return {};
      ip += len;
    } else {
      const int nb = t == 1 ? 1 : (t == 2 ? 2 : 4);
      if (n - ip < nb) return {};
      int64_t off;
      if (t == 1) {
        len = ((tag >> 2) & 7) + 4;
        off = ((int64_t)(tag >> 5) << 8) | p[ip];
      } else {
        len = (tag >> 2) + 1;
        off = 0;
        for (int q = 0; q < nb; ++q) off |= (int64_t)p[ip + q] << (8 * q);
      }
      ip += nb;
      if (off <= 0 || off > op) return {};
      while (segs.size() > 1 && op - off < segs.back().out_off) segs.pop_back();
    }
    op += len;
    if (op > out_len) return {};
  }
  if (op != out_len) return {};
  return segs;
}

struct FileHandle {
  int fd = -1;
  ~FileHandle() {
    if (fd >= 0) close(fd);
  }
};

void read_at(int fd, void* dst, size_t bytes, int64_t off, const std::string& path) {
  size_t done = 0;
  while (done < bytes) {
    const ssize_t got = pread(fd, static_cast<uint8_t*>(dst) + done, bytes - done, (off_t)(off + done));
    if (got <= 0) fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": short read");
    done += (size_t)got;
  }
}

FileMeta read_meta(const std::string& path, FileHandle& fh) {
  fh.fd = open(path.c_str(), O_RDONLY);
  if (fh.fd < 0) fail(PRISM_ERR_INTERNAL, "parquet builder for " + path + ": cannot open");
  struct stat st{};
  if (fstat(fh.fd, &st) != 0) fail(PRISM_ERR_INTERNAL, "parquet builder for " + path + ": cannot stat");
  const int64_t size = st.st_size;
  if (size < 12) fail(PRISM_ERR_INTERNAL, "parquet builder for " + path + ": file too small");
  uint8_t tail[8];
  read_at(fh.fd, tail, 8, size - 8, path);
  if (std::memcmp(tail + 4, "PAR1", 4) != 0)
    fail(PRISM_ERR_INTERNAL, "parquet builder for " + path + ": not a Parquet file");
  const uint32_t flen = (uint32_t)tail[0] | ((uint32_t)tail[1] << 8) | ((uint32_t)tail[2] << 16) | ((uint32_t)tail[3] << 24);
  if ((int64_t)flen + 8 > size) fail(PRISM_ERR_INTERNAL, "parquet builder for " + path + ": bad footer length");
  std::vector<uint8_t> footer(flen);
  read_at(fh.fd, footer.data(), flen, size - 8 - flen, path);
  return parse_footer(footer.data(), flen, size);
}

// ---------------------------------------------- row-group statistics --
// row_group_might_match / col_stats_might_match / stats_might_match /
// check_range (parquet_scan.rs:355-469): a comparison can skip a row group
// only when the scalar's type matches the column's physical statistics
// (Int64 / Int32 / Float64 / Utf8); NOT, LIKE, NE and null tests never skip.
bool check_range_f(double v, double mn, double mx, int op) {
  switch (op) {
    case PRISM_PRED_EQ: return v >= mn && v <= mx;
    case PRISM_PRED_LT: return mn < v;
    case PRISM_PRED_LE: return mn <= v;
    case PRISM_PRED_GT: return mx > v;
    case PRISM_PRED_GE: return mx >= v;
    default: return true;
  }
}
bool check_range_s(const std::string& v, const std::string& mn, const std::string& mx, int op) {
  switch (op) {
    case PRISM_PRED_EQ: return v >= mn && v <= mx;
    case PRISM_PRED_LT: return mn < v;
    case PRISM_PRED_LE: return mn <= v;
    case PRISM_PRED_GT: return mx > v;
    case PRISM_PRED_GE: return mx >= v;
    default: return true;
  }
}

int64_t le_int(const std::string& s, int bytes, bool& ok) {
  if ((int)s.size() != bytes) {
    ok = false;
    return 0;
  }
  uint64_t v = 0;
  for (int k = 0; k < bytes; ++k) v |= (uint64_t)(uint8_t)s[k] << (8 * k);
  return bytes == 4 ? (int64_t)(int32_t)(uint32_t)v : (int64_t)v;
}

// Rust's String::from_utf8_lossy: each maximal invalid sequence becomes U+FFFD
std::string utf8_lossy(const std::string& s) {
  std::string out;
  size_t i = 0;
  const size_t n = s.size();
  auto cont = [&](size_t k) { return k < n && ((uint8_t)s[k] & 0xC0) == 0x80; };
  while (i < n) {
    const uint8_t c = (uint8_t)s[i];
    size_t len = 0;
    if (c < 0x80) len = 1;
    else if (c >= 0xC2 && c <= 0xDF) len = cont(i + 1) ? 2 : 0;
    else if (c >= 0xE0 && c <= 0xEF) {
      const uint8_t c1 = i + 1 < n ? (uint8_t)s[i + 1] : 0;
      const bool ok1 = (c == 0xE0) ? (c1 >= 0xA0 && c1 <= 0xBF) : (c == 0xED) ? (c1 >= 0x80 && c1 <= 0x9F) : cont(i + 1);
      len = ok1 ? (cont(i + 2) ? 3 : 0) : 0;
      if (!len) {
        out += "\xEF\xBF\xBD";
        i += ok1 ? 2 : 1;
        continue;
      }
    } else if (c >= 0xF0 && c <= 0xF4) {
      const uint8_t c1 = i + 1 < n ? (uint8_t)s[i + 1] : 0;
      const bool ok1 = (c == 0xF0) ? (c1 >= 0x90 && c1 <= 0xBF) : (c == 0xF4) ? (c1 >= 0x80 && c1 <= 0x8F) : cont(i + 1);
      if (ok1 && cont(i + 2) && cont(i + 3)) len = 4;
      else {
        out += "\xEF\xBF\xBD";
        i += !ok1 ? 1 : (!cont(i + 2) ? 2 : 3);
        continue;
      }
    }
    if (!len) {
      out += "\xEF\xBF\xBD";
      i += 1;
      continue;
    }
    out.append(s, i, len);
    i += len;
  }
  return out;
}

bool col_stats_might_match(const prism_pred_node& nd, const RowGroup& rg, const std::vector<Leaf>& leaves) {
  if (nd.column < 0 || nd.column >= (int)leaves.size()) return true;
  const std::string& name = leaves[nd.column].name;
  const ColumnChunk* cc = nullptr;
  for (const auto& c : rg.columns)
    if (!c.path.empty() && c.path.back() == name) {
      cc = &c;
      break;
    }
  if (!cc || !cc->has_stats) return true;
  const Stats& st = cc->stats;
  const int op = nd.op;
  bool ok = true;
  if (nd.value.type == PRISM_SCALAR_INT64 && cc->type == P_INT64) {
    const int64_t mn = st.has_min ? le_int(st.min, 8, ok) : INT64_MIN;
    const int64_t mx = st.has_max ? le_int(st.max, 8, ok) : INT64_MAX;
    if (!ok) return true;
    return check_range_f((double)nd.value.i64, (double)mn, (double)mx, op);
  }
  if (nd.value.type == PRISM_SCALAR_INT32 && cc->type == P_INT32) {
    const int64_t mn = st.has_min ? le_int(st.min, 4, ok) : INT32_MIN;
    const int64_t mx = st.has_max ? le_int(st.max, 4, ok) : INT32_MAX;
    if (!ok) return true;
    return check_range_f((double)(int32_t)nd.value.i64, (double)mn, (double)mx, op);
  }
  if (nd.value.type == PRISM_SCALAR_FLOAT64 && cc->type == P_DOUBLE) {
    double mn = -1.7976931348623157e308, mx = 1.7976931348623157e308;
    if (st.has_min) {
      if (st.min.size() != 8) return true;
      std::memcpy(&mn, st.min.data(), 8);
    }
    if (st.has_max) {
      if (st.max.size() != 8) return true;
      std::memcpy(&mx, st.max.data(), 8);
    }
    return check_range_f(nd.value.f64, mn, mx, op);
  }
  if (nd.value.type == PRISM_SCALAR_UTF8 && cc->type == P_BYTE_ARRAY) {
    if (!st.has_min || !st.has_max) return true;
    const std::string v(nd.value.str ? nd.value.str : "", nd.value.str ? (size_t)nd.value.str_len : 0);
    return check_range_s(v, utf8_lossy(st.min), utf8_lossy(st.max), op);
  }
  return true;
}

bool row_group_might_match(const prism_predicate& p, const RowGroup& rg, const std::vector<Leaf>& leaves) {
  std::vector<bool> st;
  for (int i = 0; i < p.n_nodes; ++i) {
    const prism_pred_node& nd = p.nodes[i];
    switch (nd.op) {
      case PRISM_PRED_LITERAL: st.push_back(nd.value.i64 != 0); break;
      case PRISM_PRED_EQ: case PRISM_PRED_LT: case PRISM_PRED_LE: case PRISM_PRED_GT: case PRISM_PRED_GE:
        st.push_back(col_stats_might_match(nd, rg, leaves));
        break;
      case PRISM_PRED_NE: case PRISM_PRED_IS_NULL: case PRISM_PRED_IS_NOT_NULL: case PRISM_PRED_LIKE:
      case PRISM_PRED_ILIKE:
        st.push_back(true);
        break;
      case PRISM_PRED_NOT:
        if (st.empty()) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed predicate");
        st.back() = true;
        break;
      case PRISM_PRED_AND: case PRISM_PRED_OR: {
        if (st.size() < 2) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed predicate");
        const bool b = st.back();
        st.pop_back();
        const bool a = st.back();
        st.back() = nd.op == PRISM_PRED_AND ? (a && b) : (a || b);
        break;
      }
      default: fail(PRISM_ERR_INVALID_ARGUMENT, "unknown predicate node");
    }
  }
  if (st.size() != 1) fail(PRISM_ERR_INVALID_ARGUMENT, "malformed predicate");
  return st[0];
}

// ------------------------------------------------------- scan plumbing --
struct Carve {  // bump allocation inside one device block
  uint8_t* base = nullptr;
  size_t size = 0, used = 0;
  void* take(size_t bytes) {
    used = (used + 255) & ~(size_t)255;
    void* p = base + used;
    used += bytes;
    return p;
  }
};

struct ColPlan {
  int leaf;       // file column
  int32_t type;   // TY_*
  bool optional;
};

struct RgOut {  // one row group's decoded columns
  int64_t rows = 0;
  std::vector<ColP> cols;
};

int fixed_width(int32_t ty) { return ty == TY_BOOL ? 0 : width_of(ty); }

struct Chunk {  // one column chunk of one selected row group
  int rg, c;
  int64_t file_off, len;
  size_t host_off;  // offset in the staging buffer and in the device copy
  int codec, ptype;
};

struct PendingJob {  // a Snappy stream to inflate: kind 0 a data page, 1 a dictionary
  size_t chunk_src;
  int32_t src_len, dst_len;
  int kind, idx;
};

// One file's selected column chunks resident in HBM (still compressed), with
// the page tables that the decode kernels need.
struct PreparedFile {
  std::string path;
  FileMeta meta;
  std::vector<int> rgs;
  std::vector<ColPlan> plan;
  std::vector<Chunk> chunks;
  MemP raw_mem;
  std::vector<PqPage> pages;  // bodies of compressed pages are filled in per decode
  std::vector<PqDict> dicts;
  std::vector<PendingJob> pend;
  std::vector<std::vector<SnapSeg>> segs;  // per pending stream: its cut points (empty: whole)
  std::vector<int32_t> plain_utf8;
  int64_t pos_total = 0;
  size_t unc_total = 0;
  int64_t staged = 0;
  int64_t inflated = 0;
  // device side, built once: the inflate target and the kernels' tables
  MemP unc_mem, jobs_dev, pages_dev, dicts_dev, list_dev, dstarts_mem, dlens_mem;
  int64_t n_jobs = 0;
};

// Reads the selected chunks of one file into HBM and walks their pages.
PreparedFile prepare_file(Ctx& ctx, const std::string& path, FileHandle& fh, const FileMeta& m,
                          const std::vector<int>& rgs, const std::vector<ColPlan>& plan, ParquetScanStats* stats) {
  PreparedFile P;
  P.path = path;
  P.meta = m;
  P.rgs = rgs;
  P.plan = plan;
  // 1. column chunk ranges
  std::vector<Chunk>& chunks = P.chunks;
  size_t staged = 0;
  for (int g : rgs) {
    const RowGroup& R = m.row_groups[g];
    for (size_t c = 0; c < plan.size(); ++c) {
      if (plan[c].leaf >= (int)R.columns.size()) fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": missing column chunk");
      const ColumnChunk& cc = R.columns[plan[c].leaf];
      if (cc.codec != C_UNCOMPRESSED && cc.codec != C_SNAPPY)
        fail(PRISM_ERR_INVALID_ARGUMENT, "parquet " + path + ": compression codec " + std::to_string(cc.codec) +
                                             " is not supported by the GPU decoder (UNCOMPRESSED and SNAPPY are)");
      int64_t start = cc.data_page_offset;
      if (cc.dict_page_offset > 0 && cc.dict_page_offset < start) start = cc.dict_page_offset;
      if (start < 4 || cc.total_compressed < 0 || start + cc.total_compressed > m.file_size - 8)
        fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": column chunk out of the file");
      chunks.push_back({g, (int)c, start, cc.total_compressed, staged, cc.codec, cc.type});
      staged += (size_t)((cc.total_compressed + 15) & ~15LL);
    }
  }
  // 2. pread into page-locked staging, then one copy to HBM
  size_t hsize = 0;
  void* pinned = pinned_get(std::max<size_t>(staged, 16), &hsize);
  std::vector<uint8_t> pageable;
  uint8_t* host = static_cast<uint8_t*>(pinned);
  if (!host) {
    pageable.resize(std::max<size_t>(staged, 16));
    host = pageable.data();
  }
  struct PinnedHold {  // back to the pool once no copy from it can be in flight
    void* p;
    size_t n;
    cudaStream_t st;
    ~PinnedHold() {
      if (!p) return;
      cudaStreamSynchronize(st);
      pinned_put(p, n);
    }
  } pin_hold{pinned, hsize, ctx.stream};
  for (const Chunk& ch : chunks) read_at(fh.fd, host + ch.host_off, (size_t)ch.len, ch.file_off, path);
  P.raw_mem = ctx.alloc(std::max<size_t>(staged, 16));
  uint8_t* raw = static_cast<uint8_t*>(P.raw_mem->ptr);
  PRISM_CUDA(cudaMemcpyAsync(raw, host, staged, cudaMemcpyHostToDevice, ctx.stream));
  P.staged = (int64_t)staged;

  // 3. page headers (host) -> pages, dictionaries, decompression jobs
  std::vector<PqPage>& pages = P.pages;
  std::vector<PqDict>& dicts = P.dicts;
  std::vector<int32_t>& plain_utf8 = P.plain_utf8;
  int64_t& pos_total = P.pos_total;
  size_t& unc_total = P.unc_total;
  std::vector<PendingJob>& pend = P.pend;
  for (size_t ci = 0; ci < chunks.size(); ++ci) {
    const Chunk& ch = chunks[ci];
    const ColPlan& cp = plan[ch.c];
    int dict_slot = -1;
    int64_t pos = 0, row = 0;
    const int64_t want_rows = m.row_groups[ch.rg].num_rows;
    while (pos < ch.len && row < want_rows) {
      const PageHeader h = parse_page_header(host + ch.host_off + pos, (size_t)(ch.len - pos));
      const int64_t data_at = pos + h.header_bytes;
      if (h.compressed < 0 || data_at + h.compressed > ch.len)
        fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": page runs past its column chunk");
      const size_t src_off = ch.host_off + (size_t)data_at;
      if (h.type == PT_DICT) {
        if (dict_slot >= 0) fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": second dictionary page");
        if (h.encoding != E_PLAIN && h.encoding != E_PLAIN_DICT)
          fail(PRISM_ERR_INVALID_ARGUMENT, "parquet " + path + ": dictionary page encoding not supported");
        PqDict d{};
        d.count = h.dict_values;
        d.type = cp.type;
        d.body_len = h.uncompressed;
        dict_slot = (int)dicts.size();
        if (ch.codec == C_SNAPPY) {
          pend.push_back({src_off, h.compressed, h.uncompressed, 1, dict_slot});
          unc_total += (size_t)((h.uncompressed + 15) & ~15);
        } else {
          d.body = raw + src_off;
          d.body_len = h.compressed;
        }
        const int w = fixed_width(cp.type);
        if (cp.type == TY_BOOL) fail(PRISM_ERR_INVALID_ARGUMENT, "parquet " + path + ": dictionary-encoded booleans");
        if (w && (int64_t)d.count * w > (int64_t)d.body_len) fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": short dictionary page");
        dicts.push_back(d);
      } else if (h.type == PT_DATA || h.type == PT_DATA_V2) {
        PqPage p{};
        p.v1 = h.type == PT_DATA;
        p.optional = cp.optional;
        p.rows = h.type == PT_DATA_V2 ? h.num_rows : h.num_values;
        if (h.type == PT_DATA_V2 && h.num_rows != h.num_values)
          fail(PRISM_ERR_INVALID_ARGUMENT, "parquet " + path + ": repeated values are not supported");
        p.type = cp.type;
        p.out = (int)ci;
        p.out_row = row;
        p.dict = -1;
        if (h.encoding == E_PLAIN) p.enc = PE_PLAIN;
        else if (h.encoding == E_PLAIN_DICT || h.encoding == E_RLE_DICT) {
          p.enc = PE_DICT;
          if (dict_slot < 0) fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": dictionary page missing");
          p.dict = dict_slot;
        } else if (h.encoding == E_RLE && cp.type == TY_BOOL) p.enc = PE_RLE_BOOL;
        else fail(PRISM_ERR_INVALID_ARGUMENT, "parquet " + path + ": page encoding " + std::to_string(h.encoding) +
                                                  " is not supported by the GPU decoder");
        if (p.v1 && cp.optional && h.def_encoding != E_RLE)
          fail(PRISM_ERR_INVALID_ARGUMENT, "parquet " + path + ": BIT_PACKED definition levels are not supported");
        if (!p.v1 && h.rep_len != 0) fail(PRISM_ERR_INVALID_ARGUMENT, "parquet " + path + ": repetition levels");
        const int32_t lv = p.v1 ? 0 : h.def_len + h.rep_len;
        if (lv > h.compressed) fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": level bytes past the page");
        if (!p.v1) {
          p.levels = raw + src_off + h.rep_len;
          p.levels_len = h.def_len;
        }
        const bool compressed = ch.codec == C_SNAPPY && (p.v1 || h.v2_compressed);
        const int32_t body_c = h.compressed - lv, body_u = h.uncompressed - lv;
        if (compressed) {
          pend.push_back({src_off + (size_t)lv, body_c, body_u, 0, (int)pages.size()});
          unc_total += (size_t)((std::max(body_u, 0) + 15) & ~15);
          p.body_len = body_u;
        } else {
          p.body = raw + src_off + lv;
          p.body_len = body_c;
        }
        if (cp.type == TY_UTF8 && p.enc == PE_PLAIN) {
          p.pos_base = (int32_t)pos_total;
          pos_total += p.rows;
          plain_utf8.push_back((int)pages.size());
        }
        row += p.rows;
        pages.push_back(p);
      }  // index pages are skipped
      pos = data_at + h.compressed;
    }
    if (row != want_rows) fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": column chunk rows differ from its row group");
  }
  // cut points of the long Snappy streams, on every core
  P.segs.resize(pend.size());
  {
    std::vector<size_t> longs;
    for (size_t j = 0; j < pend.size(); ++j)
      if (pend[j].dst_len > SNAP_BLOCK) longs.push_back(j);
    std::atomic<size_t> next{0};
    auto work = [&] {
      for (size_t k; (k = next.fetch_add(1)) < longs.size();) {
        const PendingJob& pj = pend[longs[k]];
        P.segs[longs[k]] = snappy_segments(host + pj.chunk_src, pj.src_len, pj.dst_len);
      }
    };
    const unsigned nt = std::min<unsigned>(std::max(1u, std::thread::hardware_concurrency()), 32u);
    std::vector<std::thread> pool;
    for (unsigned q = 1; q < nt && q < longs.size(); ++q) pool.emplace_back(work);
    work();
    for (auto& th : pool) th.join();
  }
  // inflate targets and Snappy jobs (segments of long streams), longest first
  P.unc_mem = ctx.alloc(std::max<size_t>(unc_total, 16));
  uint8_t* unc = static_cast<uint8_t*>(P.unc_mem->ptr);
  std::vector<SnappyJob> jobs;
  size_t uo = 0;
  for (size_t pj = 0; pj < pend.size(); ++pj) {
    const PendingJob& j = pend[pj];
    if (j.dst_len < 0 || j.src_len < 0) fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": negative page size");
    uint8_t* dstp = unc + uo;
    uo += (size_t)((j.dst_len + 15) & ~15);
    P.inflated += j.dst_len;
    const std::vector<SnapSeg>& sg = P.segs[pj];
    if (sg.size() < 2) {
      jobs.push_back({raw + j.chunk_src, dstp, j.src_len, j.dst_len, 1, j.dst_len});
    } else {
      for (size_t q = 0; q < sg.size(); ++q) {
        const int64_t in_end = q + 1 < sg.size() ? sg[q + 1].in_off : j.src_len;
        const int64_t out_end = q + 1 < sg.size() ? sg[q + 1].out_off : j.dst_len;
        jobs.push_back({raw + j.chunk_src + sg[q].in_off, dstp + sg[q].out_off, (int32_t)(in_end - sg[q].in_off),
                        (int32_t)(out_end - sg[q].out_off), q == 0 ? 1 : 0, j.dst_len});
      }
    }
    if (j.kind == 0) pages[j.idx].body = dstp;
    else dicts[j.idx].body = dstp;
  }
  std::stable_sort(jobs.begin(), jobs.end(), [](const SnappyJob& a, const SnappyJob& b) { return a.dst_len > b.dst_len; });
  P.n_jobs = (int64_t)jobs.size();
  // byte-array dictionaries: room for their value starts / lengths
  int64_t dict_slots = 0;
  for (auto& d : dicts)
    if (d.type == TY_UTF8) dict_slots += d.count;
  uint32_t* ds = ctx.alloc_t<uint32_t>((size_t)std::max<int64_t>(dict_slots, 1), P.dstarts_mem);
  uint32_t* dl = ctx.alloc_t<uint32_t>((size_t)std::max<int64_t>(dict_slots, 1), P.dlens_mem);
  int64_t at = 0;
  for (auto& d : dicts)
    if (d.type == TY_UTF8) {
      d.starts = ds + at;
      d.lens = dl + at;
      at += d.count;
    }
  auto upload = [&](const void* src, size_t bytes, MemP& hold) {
    hold = ctx.alloc(std::max<size_t>(bytes, 16));
    if (bytes) PRISM_CUDA(cudaMemcpyAsync(hold->ptr, src, bytes, cudaMemcpyHostToDevice, ctx.stream));
  };
  upload(jobs.data(), jobs.size() * sizeof(SnappyJob), P.jobs_dev);
  upload(pages.data(), pages.size() * sizeof(PqPage), P.pages_dev);
  upload(dicts.data(), dicts.size() * sizeof(PqDict), P.dicts_dev);
  upload(plain_utf8.data(), plain_utf8.size() * 4, P.list_dev);
  (void)stats;
  ctx.sync();  // the staging buffer goes back to the pool on return
  return P;
}

// Decodes a prepared file into device columns, one RgOut per row group.
std::vector<RgOut> decode_prepared(Ctx& ctx, const PreparedFile& P, ParquetScanStats* stats) {
  const std::string& path = P.path;
  const FileMeta& m = P.meta;
  const std::vector<int>& rgs = P.rgs;
  const std::vector<ColPlan>& plan = P.plan;
  const std::vector<Chunk>& chunks = P.chunks;
  const std::vector<PqPage>& pages = P.pages;
  const std::vector<PqDict>& dicts = P.dicts;
  const std::vector<int32_t>& plain_utf8 = P.plain_utf8;
  const int64_t pos_total = P.pos_total;
  std::vector<RgOut> res(rgs.size());
  if (stats) {
    stats->pages += (int64_t)pages.size();
    stats->compressed_bytes += P.staged;
    stats->inflated_bytes += P.inflated;
  }

  // 4. outputs: one carve per file
  std::vector<PqOut> outs(chunks.size());
  int64_t utf8_rows = 0;
  size_t out_bytes = 0;
  auto words = [](int64_t n) { return (size_t)((n + 31) / 32 + 1) * 4; };
  for (const Chunk& ch : chunks) {
    const ColPlan& cp = plan[ch.c];
    const int64_t n = m.row_groups[ch.rg].num_rows;
    if (cp.optional) out_bytes += words(n) + 256;
    if (cp.type == TY_BOOL) out_bytes += words(n) + 256;
    else if (cp.type == TY_UTF8) utf8_rows += n + 1;  // + 1: the closing offset slot
    else out_bytes += (size_t)std::max<int64_t>(n, 1) * width_of(cp.type) + 256;
  }
  MemP out_mem = ctx.alloc(std::max<size_t>(out_bytes, 16));
  Carve cv{static_cast<uint8_t*>(out_mem->ptr), out_bytes, 0};
  // Utf8 scratch: lengths (u32) and source addresses (u64), one slot per row
  // plus a closing slot per segment (length 0), so one scan gives every
  // segment's offsets
  MemP ulens_mem, usrc_mem, ug_mem;
  uint32_t* ulens = nullptr;
  unsigned long long* usrcs = nullptr;
  unsigned long long* ug = nullptr;
  if (utf8_rows) {
    ulens = ctx.alloc_t<uint32_t>((size_t)utf8_rows, ulens_mem);
    usrcs = ctx.alloc_t<unsigned long long>((size_t)utf8_rows, usrc_mem);
    ug = ctx.alloc_t<unsigned long long>((size_t)utf8_rows + 1, ug_mem);
    PRISM_CUDA(cudaMemsetAsync(ulens, 0, (size_t)utf8_rows * 4, ctx.stream));
  }
  std::vector<SegView> segs;
  std::vector<int> seg_of_chunk(chunks.size(), -1);
  int64_t urow = 0;
  // bitmaps (validity, boolean values) first, zeroed by one memset: the page
  // kernel ORs bits into them; fixed-width values are written for every row
  for (size_t ci = 0; ci < chunks.size(); ++ci) {
    const ColPlan& cp = plan[chunks[ci].c];
    const int64_t n = m.row_groups[chunks[ci].rg].num_rows;
    if (cp.optional) outs[ci].valid = static_cast<uint32_t*>(cv.take(words(n)));
    if (cp.type == TY_BOOL) outs[ci].values = cv.take(words(n));
  }
  if (cv.used) PRISM_CUDA(cudaMemsetAsync(cv.base, 0, cv.used, ctx.stream));
  for (size_t ci = 0; ci < chunks.size(); ++ci) {
    const Chunk& ch = chunks[ci];
    const ColPlan& cp = plan[ch.c];
    const int64_t n = m.row_groups[ch.rg].num_rows;
    PqOut& o = outs[ci];
    if (cp.type == TY_BOOL) {
    } else if (cp.type == TY_UTF8) {
      o.lens = ulens + urow;
      o.srcs = usrcs + urow;
      seg_of_chunk[ci] = (int)segs.size();
      segs.push_back({urow, 0, n});
      urow += n + 1;
    } else {
      o.values = cv.take((size_t)std::max<int64_t>(n, 1) * width_of(cp.type));
    }
  }

  // 5. kernels
  uint32_t* err = ctx.d_err;
  auto upload = [&](const void* src, size_t bytes, MemP& hold) -> void* {
    hold = ctx.alloc(std::max<size_t>(bytes, 16));
    if (bytes) PRISM_CUDA(cudaMemcpyAsync(hold->ptr, src, bytes, cudaMemcpyHostToDevice, ctx.stream));
    return hold->ptr;
  };
  MemP outs_mem, list_mem;
  if (P.n_jobs) {
    KernelTimer kt(ctx, "pq_snappy_kernel");
    static const bool attr = [] {
      return cudaFuncSetAttribute(pq_snappy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  SNAP_WARPS * SNAP_RING) == cudaSuccess;
    }();
    if (!attr) fail(PRISM_ERR_CUDA, "cannot reserve shared memory for pq_snappy_kernel");
    pq_snappy_kernel<<<(unsigned)((P.n_jobs + SNAP_WARPS - 1) / SNAP_WARPS), 32 * SNAP_WARPS, SNAP_WARPS * SNAP_RING,
                       ctx.stream>>>(static_cast<const SnappyJob*>(P.jobs_dev->ptr), (int)P.n_jobs, err);
    ctx.check_launch("pq_snappy_kernel");
  }
  PqDict* ddicts = static_cast<PqDict*>(P.dicts_dev->ptr);
  if (!dicts.empty()) {
    KernelTimer kt(ctx, "pq_dict_kernel");
    pq_dict_kernel<<<(unsigned)((dicts.size() + 127) / 128), 128, 0, ctx.stream>>>(ddicts, (int)dicts.size(), err);
    ctx.check_launch("pq_dict_kernel");
  }
  PqPage* dpages = static_cast<PqPage*>(P.pages_dev->ptr);
  PqOut* douts = static_cast<PqOut*>(upload(outs.data(), outs.size() * sizeof(PqOut), outs_mem));
  MemP pstart_mem, plen_mem, pfound_mem;
  uint32_t* pstarts = pos_total ? ctx.alloc_t<uint32_t>((size_t)pos_total, pstart_mem) : nullptr;
  uint32_t* plens = pos_total ? ctx.alloc_t<uint32_t>((size_t)pos_total, plen_mem) : nullptr;
  int32_t* pfound = ctx.alloc_t<int32_t>(std::max<size_t>(pages.size(), 1), pfound_mem);
  if (!plain_utf8.empty()) {
    auto* dl = static_cast<int32_t*>(P.list_dev->ptr);
    KernelTimer kt(ctx, "pq_positions_kernel");
    pq_positions_kernel<<<(unsigned)((plain_utf8.size() + 127) / 128), 128, 0, ctx.stream>>>(
        dpages, dl, (int)plain_utf8.size(), pstarts, plens, pfound, err);
    ctx.check_launch("pq_positions_kernel");
  }
  if (!pages.empty()) {
    KernelTimer kt(ctx, "pq_page_kernel");
    pq_page_kernel<<<(unsigned)pages.size(), PQ_THREADS, 0, ctx.stream>>>(dpages, douts, ddicts, pstarts, plens, pfound,
                                                                          err);
    ctx.check_launch("pq_page_kernel");
  }
  // 6. Utf8: offsets and bytes
  MemP data_mem, offs_mem;
  std::vector<unsigned long long> seg_bounds;
  std::vector<int32_t*> utf8_offs(chunks.size(), nullptr);
  std::vector<uint8_t*> utf8_data(chunks.size(), nullptr);
  bool errors_read = false;  // read with the Utf8 segment bounds (one synchronisation)
  uint32_t derr_early = 0;
  if (utf8_rows) {
    MemP tot_mem;
    unsigned long long* tot = ctx.alloc_t<unsigned long long>(1, tot_mem);
    scan_u32_async(ctx, ulens, reinterpret_cast<uint64_t*>(ug), utf8_rows, reinterpret_cast<uint64_t*>(tot));
    // segment bounds: g at each segment start and at its closing slot
    std::vector<int64_t> at;
    for (const SegView& s : segs) {
      at.push_back(s.row0);
      at.push_back(s.row0 + s.rows);
    }
    MemP at_mem, gb_mem;
    auto* dat = static_cast<int64_t*>(upload(at.data(), at.size() * 8, at_mem));
    unsigned long long* gb = ctx.alloc_t<unsigned long long>(at.size(), gb_mem);
    pq_gather_u64_kernel<<<(unsigned)((at.size() + 127) / 128), 128, 0, ctx.stream>>>(ug, dat, (int)at.size(), gb);
    ctx.check_launch("pq_gather_u64_kernel");
    seg_bounds.resize(at.size() + 1);
    PRISM_CUDA(cudaMemcpyAsync(seg_bounds.data(), gb, at.size() * 8, cudaMemcpyDeviceToHost, ctx.stream));
    PRISM_CUDA(cudaMemcpyAsync(&seg_bounds[at.size()], tot, 8, cudaMemcpyDeviceToHost, ctx.stream));
    // the error word rides along: the kernels after this point report none
    PRISM_CUDA(cudaMemcpyAsync(ctx.h_err, ctx.d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx.stream));
    ctx.sync();
    errors_read = true;
    derr_early = *ctx.h_err;
    if (derr_early) {
      PRISM_CUDA(cudaMemsetAsync(ctx.d_err, 0, sizeof(uint32_t), ctx.stream));
      if (derr_early & DERR_CORRUPT) fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": malformed page data");
      fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": device error " + std::to_string(derr_early));
    }
    const unsigned long long total_bytes = seg_bounds[at.size()];
    for (size_t s = 0; s < segs.size(); ++s)
      if (seg_bounds[2 * s + 1] - seg_bounds[2 * s] > 0x7fffffffULL)
        fail(PRISM_ERR_INVALID_ARGUMENT, "parquet " + path + ": a row group's Utf8 column exceeds 2 GiB (Utf8 offsets are 32-bit)");
    uint8_t* data = static_cast<uint8_t*>((data_mem = ctx.alloc(std::max<unsigned long long>(total_bytes, 16)))->ptr);
    int32_t* offs = ctx.alloc_t<int32_t>((size_t)utf8_rows, offs_mem);
    int64_t o = 0;
    for (SegView& s : segs) {
      s.off0 = o;
      o += s.rows + 1;
    }
    MemP seg_mem;
    auto* dsegs = static_cast<SegView*>(upload(segs.data(), segs.size() * sizeof(SegView), seg_mem));
    pq_seg_offsets_kernel<<<dim3(64, (unsigned)segs.size()), 256, 0, ctx.stream>>>(ug, dsegs, (int)segs.size(), offs);
    ctx.check_launch("pq_seg_offsets_kernel");
    {
      KernelTimer kt(ctx, "pq_copy_kernel");
      pq_copy_kernel<<<grid_for(ctx, (utf8_rows + 7) / 8, 256), 256, 0, ctx.stream>>>(usrcs, ulens, ug, utf8_rows, data);
      ctx.check_launch("pq_copy_kernel");
    }
    for (size_t ci = 0; ci < chunks.size(); ++ci) {
      const int s = seg_of_chunk[ci];
      if (s < 0) continue;
      utf8_offs[ci] = offs + segs[s].off0;
      utf8_data[ci] = data + seg_bounds[2 * (size_t)s];
    }
    if (stats) stats->decoded_bytes += (int64_t)total_bytes + (int64_t)utf8_rows * 4;
  }
  const uint32_t derr = errors_read ? derr_early : ctx.take_device_errors();
  if (derr & DERR_CORRUPT) fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": malformed page data");
  if (derr) fail(PRISM_ERR_INTERNAL, "parquet read " + path + ": device error " + std::to_string(derr));

  // 7. columns per row group
  for (size_t gi = 0; gi < rgs.size(); ++gi) res[gi].rows = m.row_groups[rgs[gi]].num_rows;
  for (size_t gi = 0; gi < rgs.size(); ++gi) res[gi].cols.resize(plan.size());
  for (size_t ci = 0; ci < chunks.size(); ++ci) {
    const Chunk& ch = chunks[ci];
    const ColPlan& cp = plan[ch.c];
    const size_t gi = (size_t)(std::find(rgs.begin(), rgs.end(), ch.rg) - rgs.begin());
    const int64_t n = res[gi].rows;
    auto c = std::make_shared<Column>();
    c->type = cp.type;
    c->name = m.leaves[cp.leaf].name;
    c->nullable = cp.optional;
    c->length = n;
    c->validity = reinterpret_cast<uint8_t*>(outs[ci].valid);
    c->owners.push_back(out_mem);
    if (cp.type == TY_UTF8) {
      const int s = seg_of_chunk[ci];
      c->offsets = utf8_offs[ci];
      c->data = utf8_data[ci];
      c->data_base = 0;
      c->data_bytes = (int64_t)(seg_bounds[2 * (size_t)s + 1] - seg_bounds[2 * (size_t)s]);
      c->owners.push_back(data_mem);
      c->owners.push_back(offs_mem);
    } else {
      c->values = outs[ci].values;
    }
    if (stats) stats->decoded_bytes += cp.type == TY_UTF8 ? 0 : (cp.type == TY_BOOL ? (n + 7) / 8 : n * width_of(cp.type));
    res[gi].cols[ch.c] = c;
  }
  return res;
}

// A row-group column cut to rows [start, start + n) as a view (validity
// re-aligned when start is not a multiple of 8).
ColP slice_column(Ctx& ctx, const ColP& c, int64_t start, int64_t n, const std::vector<int64_t>& utf8_base) {
  if (start == 0 && n == c->length) return c;
  auto s = std::make_shared<Column>(*c);
  s->length = n;
  if (c->validity) {
    if (start % 8 == 0) {
      s->validity = c->validity + start / 8;
    } else {
      MemP m;
      uint32_t* dst = ctx.alloc_t<uint32_t>((size_t)((n + 31) / 32 + 1), m);
      pq_slice_bits_kernel<<<grid_for(ctx, (n + 31) / 32, 256), 256, 0, ctx.stream>>>(
          reinterpret_cast<const uint32_t*>(c->validity), start, n, dst);
      ctx.check_launch("pq_slice_bits_kernel");
      s->validity = reinterpret_cast<uint8_t*>(dst);
      s->owners.push_back(m);
    }
  }
  if (c->type == TY_BOOL) {
    MemP m;
    uint32_t* dst = ctx.alloc_t<uint32_t>((size_t)((n + 31) / 32 + 1), m);
    pq_slice_bits_kernel<<<grid_for(ctx, (n + 31) / 32, 256), 256, 0, ctx.stream>>>(
        static_cast<const uint32_t*>(c->values), start, n, dst);
    ctx.check_launch("pq_slice_bits_kernel");
    s->values = dst;
    s->owners.push_back(m);
  } else if (c->type == TY_UTF8) {
    s->offsets = c->offsets + start;
    // offsets stay relative to the row group's first byte: data_base is the
    // slice's first offset, so `data` points at the slice's first byte
    s->data_base = (int32_t)utf8_base[0];
    s->data = c->data + utf8_base[0];
    s->data_bytes = utf8_base[1] - utf8_base[0];
  } else if (c->values) {
    s->values = static_cast<uint8_t*>(c->values) + start * width_of(c->type);
  }
  return s;
}

ColP null_column(Ctx& ctx, const std::string& name, int32_t type, int64_t n) {
  // all-null column of `type` (parquet_scan.rs:541-546 uses new_null_array)
  auto c = std::make_shared<Column>();
  c->type = type;
  c->name = name;
  c->nullable = true;
  c->length = n;
  MemP m = ctx.alloc((size_t)((n + 31) / 32 + 1) * 4);
  PRISM_CUDA(cudaMemsetAsync(m->ptr, 0, (size_t)((n + 31) / 32 + 1) * 4, ctx.stream));
  c->validity = static_cast<uint8_t*>(m->ptr);
  c->owners.push_back(m);
  if (type == TY_UTF8) {
    MemP o = ctx.alloc((size_t)(n + 1) * 4);
    PRISM_CUDA(cudaMemsetAsync(o->ptr, 0, (size_t)(n + 1) * 4, ctx.stream));
    c->offsets = static_cast<int32_t*>(o->ptr);
    c->data = static_cast<uint8_t*>(m->ptr);
    c->data_bytes = 0;
    c->owners.push_back(o);
  } else if (type == TY_BOOL) {
    c->values = m->ptr;
  } else {
    const size_t b = (size_t)std::max<int64_t>(n, 1) * width_of(type);
    MemP v = ctx.alloc(b);
    PRISM_CUDA(cudaMemsetAsync(v->ptr, 0, b, ctx.stream));
    c->values = v->ptr;
    c->owners.push_back(v);
  }
  return c;
}

}  // namespace

int64_t parquet_row_count(const std::vector<std::string>& uris, const prism_predicate* predicate) {
  int64_t total = 0;
  for (const auto& uri : uris) {
    for (const auto& f : list_parquet_files(uri)) {
      FileHandle fh;
      const FileMeta m = read_meta(f, fh);
      for (const RowGroup& g : m.row_groups)
        if (!predicate || predicate->n_nodes == 0 || row_group_might_match(*predicate, g, m.leaves)) total += g.num_rows;
    }
  }
  return total;
}

// ------------------------------------------------- target schema (casts) --
// arrow_cast::cast with the default CastOptions { safe: true } between the
// numeric, boolean and Date32 types: a value the target cannot hold becomes
// null (integer range, float to integer out of range or NaN, truncating
// toward zero otherwise), Float64 -> Float32 rounds, booleans are 0 / 1 and
// a number casts to `value != 0`.
namespace {

__device__ __forceinline__ bool cast_is_float(int t) { return t == TY_F32 || t == TY_F64; }

__device__ __forceinline__ void int_range(int t, long long& lo, unsigned long long& hi) {
  switch (t) {
    case TY_I8: lo = -128; hi = 127; break;
    case TY_I16: lo = -32768; hi = 32767; break;
    case TY_I32: case TY_DATE32: lo = -2147483648LL; hi = 2147483647ULL; break;
    case TY_I64: lo = (long long)0x8000000000000000ULL; hi = 0x7FFFFFFFFFFFFFFFULL; break;
    case TY_U8: lo = 0; hi = 255; break;
    case TY_U16: lo = 0; hi = 65535; break;
    case TY_U32: lo = 0; hi = 4294967295ULL; break;
    default: lo = 0; hi = 0xFFFFFFFFFFFFFFFFULL; break;  // TY_U64
  }
}

__device__ __forceinline__ void store_int(void* out, int t, int64_t i, unsigned long long v) {
  switch (width_of(t)) {
    case 1: static_cast<uint8_t*>(out)[i] = (uint8_t)v; break;
    case 2: static_cast<uint16_t*>(out)[i] = (uint16_t)v; break;
    case 4: static_cast<uint32_t*>(out)[i] = (uint32_t)v; break;
    default: static_cast<unsigned long long*>(out)[i] = v; break;
  }
}

// one thread per 32 rows (one validity word)
__global__ void cast_column_kernel(DCol src, int32_t dst_type, void* out, uint32_t* out_valid, int64_t n) {
  for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w * 32 < n; w += (int64_t)gridDim.x * blockDim.x) {
    uint32_t word = 0;
    for (int k = 0; k < 32; ++k) {
      const int64_t i = w * 32 + k;
      if (i >= n) break;
      bool ok = dcol_valid(src, i);
      // the source value as a double, or as a 64-bit integer with its sign
      bool sf = cast_is_float(src.type);
      double d = 0;
      long long si = 0;
      unsigned long long ui = 0;
      bool neg = false;
      if (ok) {
        if (src.type == TY_F64) d = static_cast<const double*>(src.values)[i];
        else if (src.type == TY_F32) d = (double)static_cast<const float*>(src.values)[i];
        else if (src.type == TY_BOOL) ui = (static_cast<const uint8_t*>(src.values)[i >> 3] >> (i & 7)) & 1;
        else if (src.type == TY_U64) ui = static_cast<const unsigned long long*>(src.values)[i];
        else {
          si = dcol_ival(src, i);
          neg = si < 0;
          ui = (unsigned long long)si;
        }
      }
      if (ok) {
        if (dst_type == TY_BOOL) {
          const bool b = sf ? d != 0.0 : ui != 0;
          if (b) atomicOr(reinterpret_cast<unsigned int*>(out) + (i >> 5), 1u << (i & 31));
        } else if (cast_is_float(dst_type)) {
          const double v = sf ? d : (neg ? (double)si : (double)ui);
          if (dst_type == TY_F64) static_cast<double*>(out)[i] = v;
          else static_cast<float*>(out)[i] = sf && src.type == TY_F32 ? static_cast<const float*>(src.values)[i]
                                                                      : (float)(sf ? d : (neg ? (float)si : (float)ui));
        } else {
          long long lo;
          unsigned long long hi;
          int_range(dst_type, lo, hi);
          if (sf) {
            // truncate toward zero; out of range (or NaN) -> null
            const double t = trunc(d);
            const double flo = (double)lo, fhi_p1 = hi == 0xFFFFFFFFFFFFFFFFULL ? 18446744073709551616.0
                                                    : hi == 0x7FFFFFFFFFFFFFFFULL ? 9223372036854775808.0
                                                                                  : (double)hi + 1.0;
            ok = t == t && t >= flo && t < fhi_p1;
            if (ok) store_int(out, dst_type, i, t < 0 ? (unsigned long long)(long long)t : (unsigned long long)t);
          } else if (neg) {
            ok = si >= lo;
            if (ok) store_int(out, dst_type, i, (unsigned long long)si);
          } else {
            ok = ui <= hi;
            if (ok) store_int(out, dst_type, i, ui);
          }
        }
      }
      if (ok) word |= 1u << k;
    }
    out_valid[w] = word;
  }
}

bool castable(int32_t from, int32_t to) {
  auto num = [](int32_t t) {
    return t == TY_BOOL || t == TY_I8 || t == TY_I16 || t == TY_I32 || t == TY_I64 || t == TY_U8 || t == TY_U16 ||
           t == TY_U32 || t == TY_U64 || t == TY_F32 || t == TY_F64 || t == TY_DATE32;
  };
  if (!num(from) || !num(to)) return false;
  // Date32 casts to and from the integers only (as arrow does)
  if ((from == TY_DATE32 || to == TY_DATE32) && (from == TY_F32 || from == TY_F64 || to == TY_F32 ||
                                                 to == TY_F64 || from == TY_BOOL || to == TY_BOOL))
    return false;
  return true;
}

std::string type_text(int32_t t) {
  static const char* names[] = {"Null", "Boolean", "Int8", "Int16", "Int32", "Int64", "UInt8", "UInt16", "UInt32",
                                "UInt64", "Float32", "Float64", "Date32", "Utf8", "Decimal128", "Dictionary"};
  return t >= 0 && t < (int)(sizeof names / sizeof *names) ? names[t] : "type " + std::to_string(t);
}

// byte loads: a batch sliced off a row group points its bitmap at any byte
// (only a byte boundary is guaranteed), so no wider loads
__global__ void null_count_kernel(const uint8_t* valid, int64_t n, unsigned long long* out) {
  unsigned long long c = 0;
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b * 8 < n; b += (int64_t)gridDim.x * blockDim.x) {
    const int64_t rem = n - b * 8;
    const uint32_t m = rem >= 8 ? 0xFFu : ((1u << rem) - 1u);
    c += __popc(~(uint32_t)valid[b] & m);
  }
  if (c) atomicAdd(out, c);
}

// nulls in the first n rows of a column (0 without a validity bitmap)
int64_t count_nulls(Ctx& ctx, const Column& c, int64_t n) {
  if (!c.validity || n == 0) return 0;
  if (c.type == TY_NULL) return n;
  MemP m;
  unsigned long long* d = ctx.alloc_t<unsigned long long>(1, m);
  PRISM_CUDA(cudaMemsetAsync(d, 0, 8, ctx.stream));
  // bitmaps start at bit 0 of their first byte
  null_count_kernel<<<grid_for(ctx, (n + 7) / 8, 256), 256, 0, ctx.stream>>>(c.validity, n, d);
  ctx.check_launch("null_count_kernel");
  unsigned long long h = 0;
  PRISM_CUDA(cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, ctx.stream));
  ctx.sync();
  return (int64_t)h;
}

ColP cast_column(Ctx& ctx, const Column& src, const TargetField& f, int64_t n) {
  if (!castable(src.type, f.type))
    fail(PRISM_ERR_INTERNAL, "adapt_batch_to_schema: cannot cast column '" + f.name + "' from " + type_text(src.type) +
                                 " to " + type_text(f.type) + " (the GPU scan casts between numeric, Boolean and Date32 types)");
  auto c = std::make_shared<Column>();
  c->type = f.type;
  c->name = f.name;
  c->nullable = f.nullable;
  c->length = n;
  const size_t words = (size_t)((n + 31) / 32 + 1);
  MemP mv = ctx.alloc(words * 4);
  c->validity = static_cast<uint8_t*>(mv->ptr);
  c->owners.push_back(mv);
  MemP vals = ctx.alloc(f.type == TY_BOOL ? words * 4 : (size_t)std::max<int64_t>(n, 1) * width_of(f.type));
  PRISM_CUDA(cudaMemsetAsync(vals->ptr, 0, f.type == TY_BOOL ? words * 4 : (size_t)std::max<int64_t>(n, 1) * width_of(f.type),
                             ctx.stream));
  c->values = vals->ptr;
  c->owners.push_back(vals);
  if (n > 0) {
    cast_column_kernel<<<grid_for(ctx, (n + 31) / 32, 256), 256, 0, ctx.stream>>>(src.view(), f.type, vals->ptr,
                                                                                   reinterpret_cast<uint32_t*>(mv->ptr), n);
    ctx.check_launch("cast_column_kernel");
  }
  return c;
}

// adapt_batch_to_schema (parquet_scan.rs:306-339): the target's fields in
// its order, by name; a different type cast, a missing column all null; a
// non-nullable field holding a null fails as RecordBatch::try_new does.
Batch adapt_batch(Ctx& ctx, const Batch& b, const std::vector<TargetField>& target) {
  Batch out;
  out.rows = b.rows;
  for (const TargetField& f : target) {
    const Column* src = nullptr;
    for (auto& c : b.cols)
      if (c->name == f.name) {
        src = c.get();
        break;
      }
    ColP col;
    if (!src) {
      col = null_column(ctx, f.name, f.type, b.rows);
      col->precision = f.precision;
      col->scale = f.scale;
    } else if (src->type == f.type && (f.type != TY_DEC128 || (src->precision == f.precision && src->scale == f.scale))) {
      col = std::make_shared<Column>(*src);
      col->name = f.name;
      col->nullable = f.nullable;
    } else {
      col = cast_column(ctx, *src, f, b.rows);
    }
    if (!f.nullable && count_nulls(ctx, *col, b.rows) > 0)
      fail(PRISM_ERR_INTERNAL, "adapt_batch_to_schema: Invalid argument error: Column '" + f.name +
                                   "' is declared as non-nullable but contains null values");
    out.cols.push_back(col);
  }
  return out;
}

}  // namespace

struct ParquetPrepared {
  const Ctx* owner = nullptr;  // decodes run on the preparing context's stream (they share the inflate buffer)
  ParquetScanArgs args;
  std::vector<Leaf> full;  // the first file's schema
  std::vector<PreparedFile> files;
  int64_t rows = 0;
};

std::shared_ptr<ParquetPrepared> parquet_prepare(Ctx& ctx, const ParquetScanArgs& args, ParquetScanStats* stats) {
  auto P = std::make_shared<ParquetPrepared>();
  P->owner = &ctx;
  P->args = args;
  P->args.predicate = nullptr;  // used here only: the caller's predicate need not outlive this call
  if (args.uris.empty()) return P;
  if (args.batch_size <= 0) fail(PRISM_ERR_INVALID_ARGUMENT, "batch_size must be positive");
  std::vector<std::string> files;
  for (const auto& uri : args.uris) {
    const auto fs = list_parquet_files(uri);
    if (fs.empty()) fail(PRISM_ERR_INTERNAL, "no .parquet files found at " + uri);
    files.insert(files.end(), fs.begin(), fs.end());
  }
  const bool has_pred = args.predicate && args.predicate->n_nodes > 0;
  for (size_t fi = 0; fi < files.size(); ++fi) {
    const std::string& path = files[fi];
    FileHandle fh;
    const FileMeta m = read_meta(path, fh);
    if (fi == 0) P->full = m.leaves;
    if (stats) {
      stats->files += 1;
      stats->row_groups += (int64_t)m.row_groups.size();
    }
    std::vector<int> rgs;
    for (int g = 0; g < (int)m.row_groups.size(); ++g) {
      if (has_pred && !row_group_might_match(*args.predicate, m.row_groups[g], m.leaves)) {
        if (stats) stats->row_groups_skipped += 1;
        continue;
      }
      if (m.row_groups[g].num_rows > 0) rgs.push_back(g);  // an empty row group yields no batch
    }
    if (rgs.empty()) continue;
    // ProjectionMask::roots: the valid indices, in file order; none valid -> all
    std::vector<int> cols;
    if (args.has_projection)
      for (int32_t c : args.projection)
        if (c >= 0 && c < (int)m.leaves.size()) cols.push_back(c);
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    if (cols.empty())
      for (int c = 0; c < (int)m.leaves.size(); ++c) cols.push_back(c);
    std::vector<ColPlan> plan;
    for (int c : cols) {
      const Leaf& l = m.leaves[c];
      const int32_t ty = arrow_type_of(l);
      if (ty == TY_NULL)
        fail(PRISM_ERR_INVALID_ARGUMENT, "parquet " + path + ": column '" + l.name +
                                             "' has a type the GPU decoder does not read (flat BOOLEAN, INT32, DATE, "
                                             "INT64, FLOAT, DOUBLE and UTF8 BYTE_ARRAY columns are read)");
      plan.push_back({c, ty, l.repetition == 1});
    }
    P->files.push_back(prepare_file(ctx, path, fh, m, rgs, plan, stats));
    for (int g : rgs) P->rows += m.row_groups[g].num_rows;
  }
  return P;
}

int64_t parquet_prepared_rows(const ParquetPrepared& P) { return P.rows; }
int64_t parquet_prepared_bytes(const ParquetPrepared& P) {
  int64_t b = 0;
  for (const auto& f : P.files) b += f.staged;
  return b;
}

std::vector<Batch> parquet_decode(Ctx& ctx, const ParquetPrepared& P, ParquetScanStats* stats) {
  if (P.owner != &ctx) fail(PRISM_ERR_INVALID_ARGUMENT, "a prepared Parquet scan decodes on the context that prepared it");
  const ParquetScanArgs& args = P.args;
  std::vector<Batch> out;
  for (const PreparedFile& F : P.files) {
    const std::vector<ColPlan>& plan = F.plan;
    std::vector<RgOut> rg_out = decode_prepared(ctx, F, stats);
    // batches of at most batch_size rows, per row group
    for (RgOut& R : rg_out) {
      // Utf8 slice bounds need the row group's offsets at the cut points
      std::vector<int64_t> cuts;
      for (int64_t s = 0; s < R.rows; s += args.batch_size) cuts.push_back(s);
      std::vector<std::vector<int64_t>> bounds(plan.size());
      bool fetched = false;
      std::vector<std::vector<int32_t>> hb(plan.size());
      for (size_t c = 0; c < plan.size(); ++c) {
        if (plan[c].type != TY_UTF8 || cuts.size() <= 1) continue;
        hb[c].resize(cuts.size() + 1);
        for (size_t k = 0; k < cuts.size(); ++k)
          PRISM_CUDA(cudaMemcpyAsync(&hb[c][k], R.cols[c]->offsets + cuts[k], 4, cudaMemcpyDeviceToHost, ctx.stream));
        PRISM_CUDA(cudaMemcpyAsync(&hb[c][cuts.size()], R.cols[c]->offsets + R.rows, 4, cudaMemcpyDeviceToHost,
                                   ctx.stream));
        fetched = true;
      }
      if (fetched) ctx.sync();
      for (size_t c = 0; c < plan.size(); ++c) bounds[c].assign(hb[c].begin(), hb[c].end());
      for (size_t k = 0; k < cuts.size(); ++k) {
        const int64_t s = cuts[k], n = std::min(args.batch_size, R.rows - s);
        Batch b;
        b.rows = n;
        for (size_t c = 0; c < plan.size(); ++c) {
          std::vector<int64_t> ub;
          if (!bounds[c].empty()) ub = {bounds[c][k], bounds[c][k + 1]};
          b.cols.push_back(cuts.size() <= 1 ? R.cols[c] : slice_column(ctx, R.cols[c], s, n, ub));
        }
        if (n > 0) out.push_back(std::move(b));
      }
    }
  }
  // the target schema adapts full scans (with a projection the batches stay
  // file-native, parquet_scan.rs:226-236)
  if (args.has_target && !args.has_projection)
    for (Batch& b : out) b = adapt_batch(ctx, b, args.target);
  // expand_projected_batches (parquet_scan.rs:471-526) to the target schema
  // when one is given, else to the first file's
  std::vector<TargetField> full;
  if (args.has_target) {
    full = args.target;
  } else {
    for (const Leaf& l : P.full) {
      TargetField f;
      f.name = l.name;
      f.type = arrow_type_of(l);
      f.nullable = l.repetition != 0;
      full.push_back(f);
    }
  }
  if (!args.skip_expand && args.has_projection && args.projection.size() < full.size()) {
    std::vector<int> proj_map(full.size(), -1);
    for (size_t bi = 0; bi < args.projection.size(); ++bi) {
      const int32_t oi = args.projection[bi];
      if (oi >= 0 && oi < (int)full.size()) proj_map[oi] = (int)bi;
    }
    for (Batch& b : out) {
      Batch e;
      e.rows = b.rows;
      for (size_t i = 0; i < full.size(); ++i) {
        const int32_t ty = full[i].type;
        if (proj_map[i] >= 0) {
          if (proj_map[i] >= (int)b.cols.size())
            fail(PRISM_ERR_INTERNAL, "expand batch: projection index past the batch's columns");
          const ColP& src = b.cols[proj_map[i]];
          if (src->type != ty) fail(PRISM_ERR_INTERNAL, "expand batch: column types differ from the schema");
          if (!full[i].nullable && count_nulls(ctx, *src, b.rows) > 0)
            fail(PRISM_ERR_INTERNAL, "expand batch: Invalid argument error: Column '" + full[i].name +
                                         "' is declared as non-nullable but contains null values");
          auto c = std::make_shared<Column>(*src);  // the schema's field: its name and nullability
          c->name = full[i].name;
          c->nullable = full[i].nullable;
          e.cols.push_back(c);
        } else {
          if (ty == TY_NULL)
            fail(PRISM_ERR_INVALID_ARGUMENT, "parquet: column '" + full[i].name + "' has a type the GPU decoder does not read");
          e.cols.push_back(null_column(ctx, full[i].name, ty, b.rows));
        }
      }
      b = std::move(e);
    }
  }
  return out;
}

std::vector<Batch> parquet_scan(Ctx& ctx, const ParquetScanArgs& args, ParquetScanStats* stats) {
  const auto P = parquet_prepare(ctx, args, stats);
  return parquet_decode(ctx, *P, stats);
}

}  // namespace prism
