// sort.cu — sort / top-N of a batch on the device.
//
// Replaces sort_batch / sort_batch_limit (native/prism-executor/src/sort.rs:
// 35-78, arrow's lexsort_to_indices + take) and covers topn_single_col
// (sort.rs:97-146, a Float64 descending top-N) as a limit. Order per key as
// arrow's sort options define it: a key's nulls first or last whatever its
// direction; values ascending or descending; integers numerically, floats by
// IEEE totalOrder (arrow's total_cmp: -0.0 < +0.0, NaN by sign and payload at
// the ends), Utf8 / dictionary values bytewise then by length. Ties keep the
// input order (a stable sort).
//
// Method: a stable LSD radix sort of (order word, row) pairs. Every key is
// encoded, least significant part first, into 64-bit order words whose
// unsigned order is the key's order — fixed-width values in one word (their
// width in bits), Utf8 as its length and then big-endian 8-byte chunks of its
// bytes from last to first, and last the null rank — and each word is sorted
// 8 bits per pass, the row ids riding along; the next word is encoded by
// gathering through the rows' current order. A pass is a per-tile digit
// histogram, one exclusive scan over (digit, tile) and a stable scatter
// (warp match for ranks inside a warp, per-warp digit counts for ranks
// across warps, tiles in input order).
#include <algorithm>
#include <vector>

#include "prims.hpp"
#include "runtime.hpp"
#include "sort.hpp"

namespace prism {

namespace {

constexpr int RB = 256;          // threads per block
constexpr int RR = 16;           // elements per thread per tile
constexpr int RT = RB * RR;      // elements per tile
constexpr int RW = RB / 32;      // warps per block

__global__ void iota_u32_kernel(uint32_t* p, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = (uint32_t)i;
}

// digit of an element: bits [shift, shift + log2(mask + 1)) of key * mul
// (mul = 1 sorts by the key; an odd multiplier partitions by hash bits)
__device__ __forceinline__ uint32_t radix_digit(uint64_t key, uint64_t mul, int shift, uint32_t mask) {
  return (uint32_t)((key * mul) >> shift) & mask;
}

__global__ void __launch_bounds__(RB) radix_hist_kernel(const uint64_t* __restrict__ k, int64_t n, int shift,
                                                         uint32_t mask, uint32_t* counts, int64_t ntiles,
                                                         uint64_t mul) {
  __shared__ uint32_t h[256];
  const int tid = threadIdx.x;
  h[tid] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * RT;
  uint64_t w[RR];  // every load in flight before the first atomic
#pragma unroll
  for (int r = 0; r < RR; ++r) {
    const int64_t i = base + r * RB + tid;
    w[r] = i < n ? k[i] : 0;
  }
#pragma unroll
  for (int r = 0; r < RR; ++r)
    if (base + r * RB + tid < n) atomicAdd(&h[radix_digit(w[r], mul, shift, mask)], 1u);
  __syncthreads();
  counts[(int64_t)tid * ntiles + blockIdx.x] = h[tid];
}

// Stable scatter of one tile: every element's rank inside the tile's
// digit-ordered sequence is computed in tile order (rounds of RB elements:
// warp match for ranks inside a warp, per-warp digit counts across warps),
// the tile is staged in shared memory in that order, and then written out
// with consecutive threads on consecutive positions, so each digit's run of
// the tile lands as one contiguous (coalesced) stretch of the output.
// Dynamic shared memory: RT keys + RT row ids.
constexpr size_t SCATTER_SMEM = (size_t)RT * (8 + 4);
__global__ void __launch_bounds__(RB) radix_scatter_kernel(const uint64_t* __restrict__ kin,
                                                            const uint32_t* __restrict__ vin, int64_t n, int shift,
                                                            uint32_t mask, const uint32_t* __restrict__ counts,
                                                            const uint64_t* __restrict__ offsets, int64_t ntiles,
                                                            uint64_t* __restrict__ kout, uint32_t* __restrict__ vout,
                                                            uint64_t mul) {
  extern __shared__ unsigned long long stage[];  // [RT] keys | [RT] row ids
  uint64_t* sk = reinterpret_cast<uint64_t*>(stage);
  uint32_t* sv = reinterpret_cast<uint32_t*>(stage + RT);
  __shared__ uint32_t start[256];    // tile-local start of each digit's run
  __shared__ uint32_t run[256];      // elements of each digit this tile has placed
  __shared__ uint32_t wc[RW][256];   // this round: each warp's count per digit
  __shared__ uint32_t total[RW];
  __shared__ unsigned long long goff[256];  // the digit's global offset for this tile, minus its tile-local start
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t base = (int64_t)blockIdx.x * RT;
  const int count = (int)min((int64_t)RT, n - base);
  // all of this thread's elements in flight at once, before the first barrier
  uint64_t keys[RR];
  uint32_t vals[RR];
#pragma unroll
  for (int r = 0; r < RR; ++r) {
    const int e = r * RB + tid;
    keys[r] = e < count ? kin[base + e] : 0;
    vals[r] = e < count ? (vin ? vin[base + e] : (uint32_t)(base + e)) : 0;  // no vin: the element's index
  }
  // tile-local digit starts: exclusive scan of this tile's digit counts
#pragma unroll
  for (int w = 0; w < RW; ++w) wc[w][tid] = 0;
  {
    const uint32_t x = counts[(int64_t)tid * ntiles + blockIdx.x];
    uint32_t incl = x;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
      if (lane >= d) incl += y;
    }
    if (lane == 31) total[warp] = incl;
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < warp; ++w) before += total[w];
    start[tid] = before + incl - x;
    run[tid] = 0;
    goff[tid] = offsets[(int64_t)tid * ntiles + blockIdx.x] - (before + incl - x);
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RR; ++r) {
    const int e = r * RB + tid;
    const bool valid = e < count;
    const uint64_t key = keys[r];
    const uint32_t val = vals[r];
    const uint32_t d = valid ? radix_digit(key, mul, shift, mask) : 256u;  // 256: no element
    const uint32_t peers = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && rank == 0) wc[warp][d] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t before = run[d];
      for (int w = 0; w < warp; ++w) before += wc[w][d];
      const uint32_t at = start[d] + before + rank;
      sk[at] = key;
      sv[at] = val;
    }
    __syncthreads();
    uint32_t s = 0;
#pragma unroll
    for (int w = 0; w < RW; ++w) {
      s += wc[w][tid];
      wc[w][tid] = 0;
    }
    run[tid] += s;
    __syncthreads();
  }
  // staged element j belongs to digit d(j); its output position is the
  // digit's global offset for this tile plus its rank inside the digit's run
  for (int j = tid; j < count; j += RB) {
    const uint64_t key = sk[j];
    const uint32_t d = radix_digit(key, mul, shift, mask);
    const uint64_t pos = goff[d] + (uint64_t)j;
    kout[pos] = key;
    vout[pos] = sv[j];
  }
}

// order word of a fixed-width key value (its `bits` low bits); a null row's
// word is 0 so that nulls tie (their order is decided by the null rank pass)
__device__ __forceinline__ uint64_t fixed_word(const DCol& c, int64_t row, int bits, bool desc) {
  if (!dcol_valid(c, row)) return 0;
  uint64_t u;
  switch (c.type) {
    case TY_BOOL: case TY_U8: case TY_U16: case TY_U32: case TY_U64: u = (uint64_t)dcol_ival(c, row); break;
    case TY_I8: case TY_I16: case TY_I32: case TY_DATE32: case TY_I64:
      u = (uint64_t)dcol_ival(c, row) ^ (1ULL << (bits - 1));
      break;
    case TY_F64: u = (uint64_t)total_key(static_cast<const double*>(c.values)[row]) ^ (1ULL << 63); break;
    case TY_F32: {
      int32_t i = __float_as_int(static_cast<const float*>(c.values)[row]);
      i ^= (int32_t)(((uint32_t)(i >> 31)) >> 1);
      u = (uint64_t)(uint32_t)i ^ (1ULL << 31);
      break;
    }
    default: u = 0;
  }
  const uint64_t m = bits == 64 ? ~0ULL : ((1ULL << bits) - 1);
  u &= m;
  return desc ? (~u & m) : u;
}

// The inverse of fixed_word for a key without nulls: a sorted column's values
// straight from its sorted order words (a sequential pass instead of a
// gather through the row ids).
__global__ void decode_fixed_kernel(const uint64_t* __restrict__ k, int64_t n, int type, int bits, int desc,
                                    void* __restrict__ out) {
  const uint64_t m = bits == 64 ? ~0ULL : ((1ULL << bits) - 1);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t u = k[i] & m;
    if (desc) u = ~u & m;
    switch (type) {
      case TY_U8: static_cast<uint8_t*>(out)[i] = (uint8_t)u; break;
      case TY_U16: static_cast<uint16_t*>(out)[i] = (uint16_t)u; break;
      case TY_U32: static_cast<uint32_t*>(out)[i] = (uint32_t)u; break;
      case TY_U64: static_cast<uint64_t*>(out)[i] = u; break;
      case TY_I8: static_cast<uint8_t*>(out)[i] = (uint8_t)(u ^ (1ULL << 7)); break;
      case TY_I16: static_cast<uint16_t*>(out)[i] = (uint16_t)(u ^ (1ULL << 15)); break;
      case TY_I32: case TY_DATE32: static_cast<uint32_t*>(out)[i] = (uint32_t)(u ^ (1ULL << 31)); break;
      case TY_I64: static_cast<uint64_t*>(out)[i] = u ^ (1ULL << 63); break;
      case TY_F64: static_cast<double*>(out)[i] = from_total_key((int64_t)(u ^ (1ULL << 63))); break;
      case TY_F32: {
        int32_t x = (int32_t)(uint32_t)(u ^ (1ULL << 31));
        x ^= (int32_t)(((uint32_t)(x >> 31)) >> 1);
        static_cast<int32_t*>(out)[i] = x;
        break;
      }
      default: break;
    }
  }
}

__global__ void encode_fixed_kernel(DCol c, const uint32_t* __restrict__ rows, int64_t n, int bits, int desc,
                                    uint64_t* __restrict__ k) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    k[i] = fixed_word(c, rows[i], bits, desc != 0);
}

// Decimal128 as two words: low 64 bits, then the high word with the sign flipped
__global__ void encode_dec_kernel(DCol c, const uint32_t* __restrict__ rows, int64_t n, int high, int desc,
                                  uint64_t* __restrict__ k) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = rows[i];
    uint64_t u = 0;
    if (dcol_valid(c, row)) {
      const uint64_t* p = static_cast<const uint64_t*>(c.values) + 2 * row;
      u = high ? (p[1] ^ (1ULL << 63)) : p[0];
      if (desc) u = ~u;
    }
    k[i] = u;
  }
}

// Utf8 / dictionary value: word `w` = big-endian bytes [8w, 8w + 8) padded
// with zeros, or (w < 0) the length
__global__ void encode_str_kernel(DCol c, const uint32_t* __restrict__ rows, int64_t n, int w, int desc,
                                  uint64_t* __restrict__ k) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = rows[i];
    uint64_t u = 0;
    if (dcol_valid(c, row)) {
      const uint8_t* p;
      int32_t len;
      dcol_str(c, row, p, len);
      if (w < 0) {
        u = (uint32_t)len;
        if (desc) u = ~u & 0xFFFFFFFFULL;
      } else {
        const int32_t at = 8 * w;
#pragma unroll
        for (int b = 0; b < 8; ++b) u = (u << 8) | (at + b < len ? p[at + b] : 0u);
        if (desc) u = ~u;
      }
    }
    k[i] = u;
  }
}

__global__ void encode_null_kernel(DCol c, const uint32_t* __restrict__ rows, int64_t n, int nulls_first,
                                   uint64_t* __restrict__ k) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const bool valid = dcol_valid(c, rows[i]);
    k[i] = nulls_first ? (valid ? 1 : 0) : (valid ? 0 : 1);
  }
}

__global__ void max_len_kernel(DCol c, int64_t n, unsigned int* out) {
  unsigned int m = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t* p;
    int32_t len;
    dcol_str(c, i, p, len);
    m = max(m, (unsigned int)len);
  }
  for (int d = 16; d > 0; d >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, d));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// ---------------------------------------------------- top-N selection --
// One fixed-width key: its order word with the null rank above the value
// bits (`bits` value bits, `nb` = 1 when the column has nulls).
__device__ __forceinline__ uint64_t select_word(const DCol& c, int64_t row, int bits, bool desc, int nb,
                                                bool nulls_first) {
  uint64_t w = fixed_word(c, row, bits, desc);
  if (nb) {
    const bool valid = dcol_valid(c, row);
    w |= (uint64_t)(nulls_first ? valid : !valid) << bits;
  }
  return w;
}

// digit (w >> shift) & 255 of the rows whose word above the digit equals `prefix`
__global__ void select_hist_kernel(DCol c, const uint32_t* __restrict__ rows, int64_t m, int bits, int desc, int nb,
                                   int nulls_first, int shift, int top, uint64_t prefix, uint32_t* hist) {
  // one histogram per warp: a key's top digits take few values (a Float64's
  // sign and exponent), so a block-wide histogram serialises on them
  __shared__ uint32_t h[8][256];
  const int wv = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < 8; ++q) h[q][threadIdx.x] = 0;
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = rows ? rows[i] : i;
    const uint64_t w = select_word(c, row, bits, desc != 0, nb, nulls_first != 0);
    if (top || (w >> (shift + 8)) == prefix) atomicAdd(&h[wv][(w >> shift) & 255], 1u);
  }
  __syncthreads();
  uint32_t t = 0;
#pragma unroll
  for (int q = 0; q < 8; ++q) t += h[q][threadIdx.x];
  if (t) atomicAdd(&hist[threadIdx.x], t);
}

// bit i set when row i's word above `shift` is at most `bound` (kept)
__global__ void select_flags_kernel(DCol c, const uint32_t* __restrict__ rows, int64_t m, int bits, int desc, int nb,
                                    int nulls_first, int shift, uint64_t bound, uint32_t* words) {
  const int64_t nw = (m + 31) / 32;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nw * 32; i += (int64_t)gridDim.x * blockDim.x) {
    bool keep = false;
    if (i < m) {
      const int64_t row = rows ? rows[i] : i;
      keep = (select_word(c, row, bits, desc != 0, nb, nulls_first != 0) >> shift) <= bound;
    }
    const uint32_t b = __ballot_sync(0xffffffffu, keep);
    if ((threadIdx.x & 31) == 0) words[i >> 5] = b;
  }
}

__global__ void gather_rows_kernel(const uint32_t* __restrict__ rows, const uint32_t* __restrict__ idx, int64_t m,
                                   uint32_t* __restrict__ out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = rows ? rows[idx[i]] : idx[i];
}

struct Sorter {
  Ctx& ctx;
  int64_t n, ntiles;
  uint64_t *ka, *kb;
  uint32_t *va, *vb;
  uint32_t* counts;
  uint64_t* offsets;
  uint64_t* total;
  MemP mka, mkb, mva, mvb, mc, mo, mt;
  int64_t passes = 0;

  // rows to sort: `init` (ordered, n entries) or, when null, 0..n-1
  Sorter(Ctx& c, int64_t rows, const uint32_t* init = nullptr) : ctx(c), n(rows), ntiles(ceil_div(rows, (int64_t)RT)) {
    ka = ctx.alloc_t<uint64_t>((size_t)n, mka);
    kb = ctx.alloc_t<uint64_t>((size_t)n, mkb);
    va = ctx.alloc_t<uint32_t>((size_t)n, mva);
    vb = ctx.alloc_t<uint32_t>((size_t)n, mvb);
    counts = ctx.alloc_t<uint32_t>((size_t)ntiles * 256, mc);
    offsets = ctx.alloc_t<uint64_t>((size_t)ntiles * 256, mo);
    total = ctx.alloc_t<uint64_t>(1, mt);
    if (init) {
      PRISM_CUDA(cudaMemcpyAsync(va, init, (size_t)n * 4, cudaMemcpyDeviceToDevice, ctx.stream));
    } else {
      iota_u32_kernel<<<grid_for(ctx, n, 256), 256, 0, ctx.stream>>>(va, n);
      ctx.check_launch("iota_u32_kernel");
    }
    PRISM_CUDA(cudaFuncSetAttribute(radix_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SCATTER_SMEM));
  }
  int grid() const { return grid_for(ctx, n, 256); }
  // stable sort of (ka, va) by the low `bits` bits of ka, 8 per pass
  void sort_word(int bits) {
    for (int shift = 0; shift < bits; shift += 8) {
      const int w = std::min(8, bits - shift);
      const uint32_t mask = (1u << w) - 1u;
      radix_hist_kernel<<<(unsigned)ntiles, RB, 0, ctx.stream>>>(ka, n, shift, mask, counts, ntiles, 1ULL);
      ctx.check_launch("radix_hist_kernel");
      scan_u32_async(ctx, counts, offsets, ntiles * 256, total);
      {
        KernelTimer kt(ctx, "radix_scatter_kernel");
        radix_scatter_kernel<<<(unsigned)ntiles, RB, SCATTER_SMEM, ctx.stream>>>(ka, va, n, shift, mask, counts, offsets,
                                                                                  ntiles, kb, vb, 1ULL);
      }
      ctx.check_launch("radix_scatter_kernel");
      std::swap(ka, kb);
      std::swap(va, vb);
      ++passes;
    }
  }
};

int key_bits(int type) {
  switch (type) {
    case TY_BOOL: return 1;
    case TY_I8: case TY_U8: return 8;
    case TY_I16: case TY_U16: return 16;
    case TY_I32: case TY_U32: case TY_F32: case TY_DATE32: return 32;
    case TY_I64: case TY_U64: case TY_F64: return 64;
    default: return 0;
  }
}

}  // namespace

Batch sort_batch(Ctx& ctx, const Batch& b, const prism_sort_key* keys, int n_keys, int64_t limit) {
  for (int i = 0; i < n_keys; ++i) {
    if (keys[i].column < 0 || keys[i].column >= (int)b.cols.size())
      fail(PRISM_ERR_INVALID_ARGUMENT, "sort column out of range");
    const int t = b.cols[keys[i].column]->type;
    if (t == TY_NULL) fail(PRISM_ERR_INVALID_ARGUMENT, "sorting by a null-typed column");
  }
  if (b.rows == 0 || n_keys == 0) return b;  // sort.rs:36-38: the batch as it is
  if (b.rows >= (int64_t)UINT32_MAX) fail(PRISM_ERR_INVALID_ARGUMENT, "sort input exceeds 2^32-1 rows");
  const int64_t n = b.rows;
  // top-N of one fixed-width key: radix select narrows the rows to those
  // whose order word is at most the limit-th smallest (ordered compaction,
  // so ties keep their input order), and only those are sorted
  MemP msel;
  const uint32_t* sel = nullptr;
  int64_t m = n;
  if (n_keys == 1 && limit >= 0 && limit <= n / 4) {
    const Column& col = *b.cols[keys[0].column];
    const int bits = key_bits(col.type);
    const int nb = col.validity ? 1 : 0;
    if (bits && bits + nb <= 64) {
      const DCol c = col.view();
      const int desc = keys[0].descending ? 1 : 0, nf = keys[0].nulls_first ? 1 : 0;
      const int total_bits = bits + nb;
      MemP mh, mw;
      uint32_t* hist = ctx.alloc_t<uint32_t>(256, mh);
      uint64_t prefix = 0, below = 0;
      for (int shift = ((total_bits - 1) / 8) * 8; shift >= 0 && m > std::max<int64_t>(65536, 2 * limit); shift -= 8) {
        PRISM_CUDA(cudaMemsetAsync(hist, 0, 256 * 4, ctx.stream));
        const bool top = shift + 8 >= 64;
        {
          KernelTimer kt(ctx, sel ? "select_hist_kernel(narrowed)" : "select_hist_kernel");  // the first reads every row
          select_hist_kernel<<<grid_for(ctx, m, 256), 256, 0, ctx.stream>>>(c, sel, m, bits, desc, nb, nf, shift,
                                                                            top ? 1 : 0, prefix, hist);
        }
        ctx.check_launch("select_hist_kernel");
        std::vector<uint32_t> h(256);
        PRISM_CUDA(cudaMemcpyAsync(h.data(), hist, 256 * 4, cudaMemcpyDeviceToHost, ctx.stream));
        ctx.sync();
        int dig = 0;
        uint64_t cum = below;
        for (; dig < 256; ++dig) {
          if (cum + h[dig] >= (uint64_t)std::max<int64_t>(limit, 1)) break;
          cum += h[dig];
        }
        if (dig == 256) dig = 255;
        below = cum;
        prefix = (prefix << 8) | (uint64_t)dig;
        // keep the rows whose word down to this digit is at most the prefix
        uint32_t* words = ctx.alloc_t<uint32_t>((size_t)((m + 31) / 32 + 1), mw);
        select_flags_kernel<<<grid_for(ctx, m, 256), 256, 0, ctx.stream>>>(c, sel, m, bits, desc, nb, nf, shift, prefix,
                                                                           words);
        ctx.check_launch("select_flags_kernel");
        int64_t kept = 0;
        MemP idx = compact_bits(ctx, reinterpret_cast<const uint8_t*>(words), m, false, &kept);
        MemP mnext;
        uint32_t* next = ctx.alloc_t<uint32_t>((size_t)std::max<int64_t>(kept, 1), mnext);
        if (kept) {
          gather_rows_kernel<<<grid_for(ctx, kept, 256), 256, 0, ctx.stream>>>(sel, static_cast<const uint32_t*>(idx->ptr),
                                                                               kept, next);
          ctx.check_launch("gather_rows_kernel");
        }
        msel = mnext;
        sel = next;
        m = kept;
      }
    }
  }
  Sorter s(ctx, m, sel);
  // keys from the least significant (last) to the most significant (first)
  for (int ki = n_keys - 1; ki >= 0; --ki) {
    const Column& col = *b.cols[keys[ki].column];
    const DCol c = col.view();
    const int desc = keys[ki].descending ? 1 : 0;
    if (col.type == TY_UTF8 || col.type == TY_DICT) {
      MemP mm;
      unsigned int* dmax = ctx.alloc_t<unsigned int>(1, mm);
      PRISM_CUDA(cudaMemsetAsync(dmax, 0, 4, ctx.stream));
      max_len_kernel<<<grid_for(ctx, n, 256), 256, 0, ctx.stream>>>(c, n, dmax);
      ctx.check_launch("max_len_kernel");
      unsigned int maxlen = 0;
      PRISM_CUDA(cudaMemcpyAsync(&maxlen, dmax, 4, cudaMemcpyDeviceToHost, ctx.stream));
      ctx.sync();
      encode_str_kernel<<<s.grid(), 256, 0, ctx.stream>>>(c, s.va, m, -1, desc, s.ka);
      ctx.check_launch("encode_str_kernel");
      s.sort_word(32);
      for (int w = (int)((maxlen + 7) / 8) - 1; w >= 0; --w) {
        encode_str_kernel<<<s.grid(), 256, 0, ctx.stream>>>(c, s.va, m, w, desc, s.ka);
        ctx.check_launch("encode_str_kernel");
        s.sort_word(64);
      }
    } else if (col.type == TY_DEC128) {
      for (int high = 0; high < 2; ++high) {
        encode_dec_kernel<<<s.grid(), 256, 0, ctx.stream>>>(c, s.va, m, high, desc, s.ka);
        ctx.check_launch("encode_dec_kernel");
        s.sort_word(64);
      }
    } else {
      const int bits = key_bits(col.type);
      if (!bits) fail(PRISM_ERR_INVALID_ARGUMENT, "unsupported sort key type");
      encode_fixed_kernel<<<s.grid(), 256, 0, ctx.stream>>>(c, s.va, m, bits, desc, s.ka);
      ctx.check_launch("encode_fixed_kernel");
      s.sort_word(bits);
    }
    if (col.validity) {
      encode_null_kernel<<<s.grid(), 256, 0, ctx.stream>>>(c, s.va, m, keys[ki].nulls_first ? 1 : 0, s.ka);
      ctx.check_launch("encode_null_kernel");
      s.sort_word(1);
    }
  }
  const int64_t outn = limit >= 0 ? std::min(limit, m) : m;
  Batch out;
  out.rows = outn;
  // the most significant key, fixed width without nulls: its sorted order
  // words (the last word sorted) decode back into the output column
  const Column& k0 = *b.cols[keys[0].column];
  const bool decode_k0 = !k0.validity && k0.type != TY_BOOL && key_bits(k0.type) > 0;
  for (size_t ci = 0; ci < b.cols.size(); ++ci) {
    const auto& c = b.cols[ci];
    if (decode_k0 && (int)ci == keys[0].column) {
      ColP d = make_column(ctx, c->type, c->name, outn, false);
      d->nullable = c->nullable;
      if (outn) {
        decode_fixed_kernel<<<grid_for(ctx, outn, 256), 256, 0, ctx.stream>>>(s.ka, outn, c->type, key_bits(c->type),
                                                                              keys[0].descending ? 1 : 0, d->values);
        ctx.check_launch("decode_fixed_kernel");
      }
      out.cols.push_back(d);
      continue;
    }
    out.cols.push_back(take(ctx, *c, s.va, nullptr, outn, c->name, c->nullable));
  }
  return out;  // stream-ordered: the sort buffers are freed after the gathers

}

// Radix partition of 64-bit keys (with their positions 0..n-1) by the digit
// bits [shift, shift + bits) of key * mul, bits <= 8: one pass of the sort's
// machinery — per-tile digit histograms, one scan over (digit, tile), and a
// scatter that ranks each tile in order, stages it in shared memory and
// writes every digit's run of the tile contiguously. Output: the keys and
// their original positions in partition order, positions ascending inside a
// partition (stable).
void radix_partition(Ctx& ctx, const uint64_t* keys, int64_t n, uint64_t mul, int shift, int bits,
                     uint64_t* kout, uint32_t* pos_out, const char* hist_name, const char* scatter_name) {
  if (n <= 0) return;
  if (bits < 1 || bits > 8) fail(PRISM_ERR_INTERNAL, "radix partition digit of 1..8 bits");
  if (n >= (int64_t)UINT32_MAX) fail(PRISM_ERR_INVALID_ARGUMENT, "radix partition of 2^32 rows or more");
  const int64_t ntiles = ceil_div(n, (int64_t)RT);
  const uint32_t mask = (1u << bits) - 1u;
  MemP mc, mo, mt;
  uint32_t* counts = ctx.alloc_t<uint32_t>((size_t)ntiles * 256, mc);
  uint64_t* offsets = ctx.alloc_t<uint64_t>((size_t)ntiles * 256, mo);
  uint64_t* total = ctx.alloc_t<uint64_t>(1, mt);
  {
    KernelTimer kt(ctx, hist_name);
    radix_hist_kernel<<<(unsigned)ntiles, RB, 0, ctx.stream>>>(keys, n, shift, mask, counts, ntiles, mul);
  }
  ctx.check_launch("radix_hist_kernel(partition)");
  scan_u32_async(ctx, counts, offsets, ntiles * 256, total);
  PRISM_CUDA(cudaFuncSetAttribute(radix_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SCATTER_SMEM));
  {
    KernelTimer kt(ctx, scatter_name);
    radix_scatter_kernel<<<(unsigned)ntiles, RB, SCATTER_SMEM, ctx.stream>>>(keys, nullptr, n, shift, mask, counts,
                                                                              offsets, ntiles, kout, pos_out, mul);
  }
  ctx.check_launch("radix_scatter_kernel(partition)");
}

}  // namespace prism
