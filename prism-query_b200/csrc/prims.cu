// prims.cu — scan, ordered bit compaction, stable pair sort, gather kernels.
#include "prims.hpp"

namespace prism {

namespace {

constexpr int SB = 256;      // scan block
constexpr int SI = 8;        // items per thread
constexpr int ST = SB * SI;  // scan tile

__device__ __forceinline__ uint64_t warp_incl_scan(uint64_t x) {
  int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint64_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  return x;
}

// Exclusive block scan of one value per thread; returns the block total.
__device__ __forceinline__ uint64_t block_excl_scan(uint64_t v, uint64_t& excl) {
  __shared__ uint64_t warp_sums[32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint64_t incl = warp_incl_scan(v);
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint64_t s = lane < nw ? warp_sums[lane] : 0;
    uint64_t si = warp_incl_scan(s);
    if (lane < nw) warp_sums[lane] = si - s;
    if (lane == 31) warp_sums[31] = si;  // total (nw <= 31 blocks of 32 lanes)
  }
  __syncthreads();
  excl = warp_sums[warp] + incl - v;
  uint64_t total = warp_sums[31];
  __syncthreads();
  return total;
}

__global__ void tile_sum_kernel(const uint32_t* __restrict__ in, int64_t n, uint64_t* __restrict__ sums) {
  int64_t base = (int64_t)blockIdx.x * ST;
  uint64_t s = 0;
  for (int k = 0; k < SI; ++k) {
    int64_t i = base + k * SB + threadIdx.x;
    if (i < n) s += in[i];
  }
  uint64_t excl;
  uint64_t tot = block_excl_scan(s, excl);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// single block: exclusive scan of ntiles sums in place; total into sums[ntiles]
__global__ void scan_sums_kernel(uint64_t* sums, int64_t ntiles) {
  uint64_t carry = 0;
  for (int64_t b = 0; b < ntiles; b += SB) {
    int64_t i = b + threadIdx.x;
    uint64_t v = i < ntiles ? sums[i] : 0;
    uint64_t excl;
    uint64_t tot = block_excl_scan(v, excl);
    if (i < ntiles) sums[i] = carry + excl;
    carry += tot;
  }
  if (threadIdx.x == 0) sums[ntiles] = carry;
}

__global__ void tile_scan_kernel(const uint32_t* __restrict__ in, int64_t n, const uint64_t* __restrict__ offs,
                                 uint64_t* __restrict__ out) {
  __shared__ uint32_t tile[ST];
  int64_t base = (int64_t)blockIdx.x * ST;
  for (int k = 0; k < SI; ++k) {
    int64_t i = base + k * SB + threadIdx.x;
    tile[k * SB + threadIdx.x] = i < n ? in[i] : 0;
  }
  __syncthreads();
  uint64_t local[SI];
  uint64_t s = 0;
  for (int k = 0; k < SI; ++k) {
    local[k] = s;
    s += tile[threadIdx.x * SI + k];
  }
  uint64_t excl;
  block_excl_scan(s, excl);
  uint64_t o = offs[blockIdx.x] + excl;
  for (int k = 0; k < SI; ++k) {
    int64_t i = base + threadIdx.x * SI + k;
    if (i < n) out[i] = o + local[k];
  }
}

__device__ __forceinline__ uint32_t load_word(const uint8_t* bm, int64_t w, int64_t n_bits, bool invert) {
  int64_t nbytes = (n_bits + 7) >> 3;
  uint32_t x = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    int64_t b = w * 4 + k;
    if (b < nbytes) x |= (uint32_t)bm[b] << (8 * k);
  }
  if (invert) x = ~x;
  int64_t lo = w * 32;
  if (lo + 32 > n_bits) {
    int keep = (int)(n_bits - lo);
    x &= keep <= 0 ? 0u : (keep >= 32 ? 0xffffffffu : ((1u << keep) - 1));
  }
  return x;
}

__global__ void word_popc_kernel(const uint8_t* bm, int64_t n_bits, bool invert, uint32_t* cnt, int64_t nw) {
  for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < nw; w += (int64_t)gridDim.x * blockDim.x)
    cnt[w] = __popc(load_word(bm, w, n_bits, invert));
}

__global__ void word_emit_kernel(const uint8_t* bm, int64_t n_bits, bool invert, const uint64_t* off, int64_t nw,
                                 uint32_t* out) {
  for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < nw; w += (int64_t)gridDim.x * blockDim.x) {
    uint32_t x = load_word(bm, w, n_bits, invert);
    uint64_t o = off[w];
    while (x) {
      int b = __ffs(x) - 1;
      out[o++] = (uint32_t)(w * 32 + b);
      x &= x - 1;
    }
  }
}

__global__ void split_flags_kernel(const uint32_t* keys, int64_t n, int bit, uint32_t* zf) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    zf[i] = ((keys[i] >> bit) & 1) ? 0u : 1u;
}

__global__ void split_scatter_kernel(const uint32_t* ki, const uint32_t* vi, int64_t n, int bit, const uint64_t* zpos,
                                     uint64_t total_zeros, uint32_t* ko, uint32_t* vo) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t k = ki[i];
    uint64_t d = ((k >> bit) & 1) ? total_zeros + ((uint64_t)i - zpos[i]) : zpos[i];
    ko[d] = k;
    vo[d] = vi[i];
  }
}

template <int W>
struct Blob {
  uint8_t b[W];
};

template <int W>
__global__ void gather_fixed_kernel(const Blob<W>* __restrict__ src, const uint32_t* __restrict__ idx,
                                    const uint8_t* __restrict__ idx_valid, int64_t n, Blob<W>* __restrict__ dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    bool ok = idx_valid == nullptr || ((idx_valid[i >> 3] >> (i & 7)) & 1);
    if (ok) dst[i] = src[idx[i]];
    else dst[i] = Blob<W>{};
  }
}

// gathers one bit per output (validity or Boolean values); warp-ballot writes
// whole 32-bit words. src_bits == nullptr means "all ones".
__global__ void gather_bits_kernel(const uint8_t* __restrict__ src_bits, const uint32_t* __restrict__ idx,
                                   const uint8_t* __restrict__ idx_valid, bool null_idx_bit, int64_t n,
                                   uint32_t* __restrict__ out_words) {
  int64_t nwarp_items = (n + 31) & ~int64_t(31);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nwarp_items;
       i += (int64_t)gridDim.x * blockDim.x) {
    bool bit = false;
    if (i < n) {
      bool iv = idx_valid == nullptr || ((idx_valid[i >> 3] >> (i & 7)) & 1);
      if (!iv) bit = null_idx_bit;
      else {
        uint32_t j = idx[i];
        bit = src_bits == nullptr || ((src_bits[j >> 3] >> (j & 7)) & 1);
      }
    }
    uint32_t w = __ballot_sync(0xffffffffu, bit);
    if ((threadIdx.x & 31) == 0) out_words[i >> 5] = w;
  }
}

__global__ void str_len_kernel(const int32_t* __restrict__ offs, const uint32_t* __restrict__ idx,
                               const uint8_t* __restrict__ idx_valid, int64_t n, uint32_t* __restrict__ len) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    bool ok = idx_valid == nullptr || ((idx_valid[i >> 3] >> (i & 7)) & 1);
    uint32_t j = ok ? idx[i] : 0;
    len[i] = ok ? (uint32_t)(offs[j + 1] - offs[j]) : 0u;
  }
}

__global__ void str_copy_kernel(const int32_t* __restrict__ offs, const uint8_t* __restrict__ data,
                                const uint32_t* __restrict__ idx, const uint8_t* __restrict__ idx_valid,
                                const uint64_t* __restrict__ out_off64, int64_t n, int32_t* __restrict__ out_offs,
                                uint8_t* __restrict__ out_data) {
  // one warp per string; lanes copy bytes
  int lane = threadIdx.x & 31;
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = warp; i < n; i += nwarps) {
    int64_t o = (int64_t)out_off64[i];
    if (lane == 0) out_offs[i] = (int32_t)o;
    bool ok = idx_valid == nullptr || ((idx_valid[i >> 3] >> (i & 7)) & 1);
    if (!ok) continue;
    uint32_t j = idx[i];
    int32_t a = offs[j], b = offs[j + 1];
    for (int32_t k = lane; k < b - a; k += 32) out_data[o + k] = data[a + k];
  }
}

__global__ void set_last_offset_kernel(int32_t* out_offs, int64_t n, uint64_t total) { out_offs[n] = (int32_t)total; }

__global__ void pack_bits_kernel(const uint8_t* bytes, int64_t n, uint32_t* out_words) {
  int64_t nwarp_items = (n + 31) & ~int64_t(31);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nwarp_items;
       i += (int64_t)gridDim.x * blockDim.x) {
    bool bit = i < n && bytes[i];
    uint32_t w = __ballot_sync(0xffffffffu, bit);
    if ((threadIdx.x & 31) == 0) out_words[i >> 5] = w;
  }
}

__global__ void scatter_bits_kernel(const uint32_t* idx, int64_t n, uint32_t* words) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t j = idx[i];
    atomicOr(&words[j >> 5], 1u << (j & 31));
  }
}

}  // namespace

static __global__ void copy_total_kernel(const uint64_t* src, uint64_t* dst) { *dst = *src; }

void scan_u32_async(Ctx& ctx, const uint32_t* in, uint64_t* out, int64_t n, uint64_t* total_dev) {
  if (n <= 0) {
    PRISM_CUDA(cudaMemsetAsync(total_dev, 0, 8, ctx.stream));
    return;
  }
  int64_t ntiles = ceil_div(n, ST);
  MemP ms;
  uint64_t* sums = ctx.alloc_t<uint64_t>((size_t)ntiles + 1, ms);
  tile_sum_kernel<<<(unsigned)ntiles, SB, 0, ctx.stream>>>(in, n, sums);
  ctx.check_launch("tile_sum_kernel");
  scan_sums_kernel<<<1, SB, 0, ctx.stream>>>(sums, ntiles);
  ctx.check_launch("scan_sums_kernel");
  tile_scan_kernel<<<(unsigned)ntiles, SB, 0, ctx.stream>>>(in, n, sums, out);
  ctx.check_launch("tile_scan_kernel");
  copy_total_kernel<<<1, 1, 0, ctx.stream>>>(sums + ntiles, total_dev);
  ctx.check_launch("copy_total_kernel");
}

uint64_t scan_u32(Ctx& ctx, const uint32_t* in, uint64_t* out, int64_t n) {
  if (n <= 0) return 0;
  int64_t ntiles = ceil_div(n, ST);
  MemP ms;
  uint64_t* sums = ctx.alloc_t<uint64_t>((size_t)ntiles + 1, ms);
  tile_sum_kernel<<<(unsigned)ntiles, SB, 0, ctx.stream>>>(in, n, sums);
  ctx.check_launch("tile_sum_kernel");
  scan_sums_kernel<<<1, SB, 0, ctx.stream>>>(sums, ntiles);
  ctx.check_launch("scan_sums_kernel");
  tile_scan_kernel<<<(unsigned)ntiles, SB, 0, ctx.stream>>>(in, n, sums, out);
  ctx.check_launch("tile_scan_kernel");
  uint64_t total = 0;
  PRISM_CUDA(cudaMemcpyAsync(&total, sums + ntiles, 8, cudaMemcpyDeviceToHost, ctx.stream));
  PRISM_CUDA(cudaStreamSynchronize(ctx.stream));
  return total;
}

MemP compact_bits(Ctx& ctx, const uint8_t* bitmap, int64_t n, bool invert, int64_t* count) {
  *count = 0;
  if (n <= 0) return ctx.alloc(4);
  int64_t nw = ceil_div(n, 32);
  MemP mc, mo;
  uint32_t* cnt = ctx.alloc_t<uint32_t>((size_t)nw, mc);
  uint64_t* off = ctx.alloc_t<uint64_t>((size_t)nw, mo);
  int g = grid_for(ctx, nw, 256);
  word_popc_kernel<<<g, 256, 0, ctx.stream>>>(bitmap, n, invert, cnt, nw);
  ctx.check_launch("word_popc_kernel");
  uint64_t total = scan_u32(ctx, cnt, off, nw);
  MemP out = ctx.alloc(std::max<uint64_t>(total, 1) * 4);
  if (total) {
    word_emit_kernel<<<g, 256, 0, ctx.stream>>>(bitmap, n, invert, off, nw, static_cast<uint32_t*>(out->ptr));
    ctx.check_launch("word_emit_kernel");
  }
  *count = (int64_t)total;
  return out;
}

void stable_sort_pairs_u32(Ctx& ctx, uint32_t* keys, uint32_t* vals, int64_t n, int bits) {
  if (n <= 1 || bits <= 0) return;
  MemP mk, mv, mz, mp;
  uint32_t* k2 = ctx.alloc_t<uint32_t>((size_t)n, mk);
  uint32_t* v2 = ctx.alloc_t<uint32_t>((size_t)n, mv);
  uint32_t* zf = ctx.alloc_t<uint32_t>((size_t)n, mz);
  uint64_t* zp = ctx.alloc_t<uint64_t>((size_t)n, mp);
  uint32_t *ka = keys, *va = vals, *kb = k2, *vb = v2;
  int g = grid_for(ctx, n, 256);
  for (int bit = 0; bit < bits; ++bit) {
    split_flags_kernel<<<g, 256, 0, ctx.stream>>>(ka, n, bit, zf);
    ctx.check_launch("split_flags_kernel");
    uint64_t zeros = scan_u32(ctx, zf, zp, n);
    split_scatter_kernel<<<g, 256, 0, ctx.stream>>>(ka, va, n, bit, zp, zeros, kb, vb);
    ctx.check_launch("split_scatter_kernel");
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    PRISM_CUDA(cudaMemcpyAsync(keys, ka, n * 4, cudaMemcpyDeviceToDevice, ctx.stream));
    PRISM_CUDA(cudaMemcpyAsync(vals, va, n * 4, cudaMemcpyDeviceToDevice, ctx.stream));
  }
}

ColP take(Ctx& ctx, const Column& col, const uint32_t* idx, const uint8_t* idx_valid, int64_t n,
          const std::string& name, bool nullable) {
  auto out = std::make_shared<Column>();
  out->type = col.type;
  out->index_type = col.index_type;
  out->name = name;
  out->nullable = nullable;
  out->length = n;
  out->precision = col.precision;
  out->scale = col.scale;
  out->dict = col.dict;
  out->dict_fingerprint = col.dict_fingerprint;
  if (col.type == TY_NULL) return out;
  int g = grid_for(ctx, std::max<int64_t>(n, 1), 256);
  if (col.validity || idx_valid) {
    MemP mvb;
    out->validity = ctx.alloc_t<uint8_t>((size_t)(n + 7) / 8 + 8, mvb);
    out->owners.push_back(mvb);
    if (n) {
      gather_bits_kernel<<<g, 256, 0, ctx.stream>>>(col.validity, idx, idx_valid, false, n,
                                                     reinterpret_cast<uint32_t*>(out->validity));
      ctx.check_launch("gather_bits_kernel(validity)");
    }
  }
  if (col.type == TY_UTF8) {
    MemP ml, mo;
    uint32_t* len = ctx.alloc_t<uint32_t>((size_t)std::max<int64_t>(n, 1), ml);
    uint64_t* off = ctx.alloc_t<uint64_t>((size_t)std::max<int64_t>(n, 1), mo);
    const int32_t* src_offs = col.offsets;
    const uint8_t* src_data = col.data - col.data_base;
    uint64_t total = 0;
    if (n) {
      str_len_kernel<<<g, 256, 0, ctx.stream>>>(src_offs, idx, idx_valid, n, len);
      ctx.check_launch("str_len_kernel");
      total = scan_u32(ctx, len, off, n);
    }
    if (total > (uint64_t)INT32_MAX) fail(PRISM_ERR_ARROW, "Utf8 output exceeds 2 GiB (i32 offsets)");
    MemP mof, md;
    out->offsets = ctx.alloc_t<int32_t>((size_t)n + 1, mof);
    out->data = ctx.alloc_t<uint8_t>((size_t)std::max<uint64_t>(total, 1) + 8, md);
    out->data_bytes = (int64_t)total;
    out->data_base = 0;
    out->owners.push_back(mof);
    out->owners.push_back(md);
    if (n) {
      int gw = grid_for(ctx, n * 32, 256);
      str_copy_kernel<<<gw, 256, 0, ctx.stream>>>(src_offs, src_data, idx, idx_valid, off, n, out->offsets, out->data);
      ctx.check_launch("str_copy_kernel");
    }
    set_last_offset_kernel<<<1, 1, 0, ctx.stream>>>(out->offsets, n, total);
    ctx.check_launch("set_last_offset_kernel");
    return out;
  }
  if (col.type == TY_BOOL) {
    MemP mb;
    out->values = ctx.alloc_t<uint8_t>((size_t)(n + 7) / 8 + 8, mb);
    out->owners.push_back(mb);
    if (n) {
      gather_bits_kernel<<<g, 256, 0, ctx.stream>>>(static_cast<const uint8_t*>(col.values), idx, idx_valid, false, n,
                                                     reinterpret_cast<uint32_t*>(out->values));
      ctx.check_launch("gather_bits_kernel(bool)");
    }
    return out;
  }
  int w = width_of(col.type == TY_DICT ? col.index_type : col.type);
  MemP mv = ctx.alloc((size_t)std::max<int64_t>(n, 1) * w + 16);
  out->values = mv->ptr;
  out->owners.push_back(mv);
  if (n) {
    switch (w) {
      case 1: gather_fixed_kernel<1><<<g, 256, 0, ctx.stream>>>((const Blob<1>*)col.values, idx, idx_valid, n, (Blob<1>*)out->values); break;
      case 2: gather_fixed_kernel<2><<<g, 256, 0, ctx.stream>>>((const Blob<2>*)col.values, idx, idx_valid, n, (Blob<2>*)out->values); break;
      case 4: gather_fixed_kernel<4><<<g, 256, 0, ctx.stream>>>((const Blob<4>*)col.values, idx, idx_valid, n, (Blob<4>*)out->values); break;
      case 8: gather_fixed_kernel<8><<<g, 256, 0, ctx.stream>>>((const Blob<8>*)col.values, idx, idx_valid, n, (Blob<8>*)out->values); break;
      case 16: gather_fixed_kernel<16><<<g, 256, 0, ctx.stream>>>((const Blob<16>*)col.values, idx, idx_valid, n, (Blob<16>*)out->values); break;
      default: fail(PRISM_ERR_INTERNAL, "bad gather width");
    }
    ctx.check_launch("gather_fixed_kernel");
  }
  return out;
}

ColP filter_column(Ctx& ctx, const Column& col, const uint32_t* kept_rows, int64_t n_kept) {
  return take(ctx, col, kept_rows, nullptr, n_kept, col.name, col.nullable);
}

void pack_bits(Ctx& ctx, const uint8_t* bytes, int64_t n, uint8_t* bitmap) {
  if (n <= 0) return;
  pack_bits_kernel<<<grid_for(ctx, n, 256), 256, 0, ctx.stream>>>(bytes, n, reinterpret_cast<uint32_t*>(bitmap));
  ctx.check_launch("pack_bits_kernel");
}

void scatter_bits(Ctx& ctx, const uint32_t* idx, int64_t n, uint8_t* bitmap) {
  if (n <= 0) return;
  scatter_bits_kernel<<<grid_for(ctx, n, 256), 256, 0, ctx.stream>>>(idx, n, reinterpret_cast<uint32_t*>(bitmap));
  ctx.check_launch("scatter_bits_kernel");
}

ColP u32_column(Ctx& ctx, const std::string& name, MemP mem, uint32_t* ptr, int64_t n) {
  (void)ctx;
  auto c = std::make_shared<Column>();
  c->type = TY_U32;
  c->name = name;
  c->nullable = false;
  c->length = n;
  c->values = ptr;
  c->owners.push_back(mem);
  return c;
}

}  // namespace prism
