// MatrixMarket text -> CSR on the GPU (the input side of the path): the
// reference's GraphCache::from_mtx_file (graph/cache/parser_mtx/mod.rs:34-162)
// parses entry lines with host threads (parser_mtx/producers.rs:139-240),
// counts degrees, scatters neighbours and sorts every row
// (graph/cache/impl_sort.rs:10-51).  Here the body of the file is one device
// buffer:
//   k_mtx_count_lines / k_mtx_fill_lines   line starts (a byte after '\n')
//   k_mtx_parse<false|true>                 per line: skip blank and '%' lines
//                                           and lines with fewer than two
//                                           tokens, parse i j (1-based), flag
//                                           0 or out-of-range indices; count,
//                                           then emit (i-1, j-1) and, for a
//                                           symmetric header and i != j, the
//                                           mirror, as keys row << 32 | column
//   k_radix_hist / k_radix_scatter          stable LSD radix sort of the keys
//                                           (8-bit digits): sorted keys are the
//                                           CSR rows in order, each ascending
//   k_mtx_rows                              row lengths -> offsets (scanned)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sparx {

enum : uint32_t {
  kMtxZeroIndex = 1u,    // an index of 0 (MatrixMarket is 1-based)
  kMtxOutOfRange = 2u,   // an index beyond the size line
  kMtxBadNumber = 4u,    // a token that is not an unsigned integer
};

// Rust's char::is_whitespace on ASCII (what str::trim and split_whitespace use)
__device__ __forceinline__ bool mtx_space(unsigned char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == 0x0B || c == 0x0C;
}

__device__ __forceinline__ bool line_start(const unsigned char* __restrict__ body, unsigned long long p) {
  return p == 0 || body[p - 1] == '\n';
}

// line starts per 16-byte chunk
struct MtxLineCount {
  const unsigned char* body;
  unsigned long long len;
  __device__ __forceinline__ unsigned long long operator()(unsigned long long c) const {
    const unsigned long long b = c * 16, e = min(b + 16, len);
    unsigned long long n = 0;
    for (unsigned long long p = b; p < e; ++p) n += line_start(body, p);
    return n;
  }
};

__global__ void __launch_bounds__(256) k_mtx_fill_lines(const unsigned char* __restrict__ body,
                                                        unsigned long long len,
                                                        const unsigned long long* __restrict__ chunk_pref,
                                                        unsigned long long* __restrict__ starts) {
  const unsigned long long chunks = (len + 15) / 16;
  for (unsigned long long c = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; c < chunks;
       c += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long at = chunk_pref[c];
    const unsigned long long b = c * 16, e = min(b + 16, len);
    for (unsigned long long p = b; p < e; ++p)
      if (line_start(body, p)) starts[at++] = p;
  }
}

// Unsigned decimal token at [p, e): Rust's usize::from_str (an optional '+',
// then digits; anything else, or a value past 64 bits, fails).
__device__ __forceinline__ bool mtx_number(const unsigned char* __restrict__ body, unsigned long long p,
                                           unsigned long long e, unsigned long long* out) {
  if (p < e && body[p] == '+') ++p;
  if (p >= e) return false;
  unsigned long long v = 0;
  for (; p < e; ++p) {
    const unsigned c = body[p] - '0';
    if (c > 9) return false;
    if (v > (~0ull - c) / 10) return false;
    v = v * 10 + c;
  }
  *out = v;
  return true;
}

// One thread per line.  kEmit false: edges per line into `count` and error
// flags (with the first failing line); kEmit true: the keys at `at[line]`.
template <bool kEmit>
__global__ void __launch_bounds__(256) k_mtx_parse(const unsigned char* __restrict__ body,
                                                   unsigned long long len,
                                                   const unsigned long long* __restrict__ starts,
                                                   unsigned long long lines, unsigned long long n, int symmetric,
                                                   uint32_t* __restrict__ count,
                                                   const unsigned long long* __restrict__ at,
                                                   unsigned long long* __restrict__ keys, uint32_t* __restrict__ err,
                                                   unsigned long long* __restrict__ bad_line) {
  for (unsigned long long l = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; l < lines;
       l += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long p = starts[l];
    unsigned long long end = p;
    while (end < len && body[end] != '\n') ++end;
    while (p < end && mtx_space(body[p])) ++p;  // trim
    uint32_t edges = 0, flags = 0;
    unsigned long long i = 0, j = 0;
    if (p < end && body[p] != '%') {
      unsigned long long t0 = p;
      while (p < end && !mtx_space(body[p])) ++p;
      const unsigned long long t0e = p;
      while (p < end && mtx_space(body[p])) ++p;
      const unsigned long long t1 = p;
      while (p < end && !mtx_space(body[p])) ++p;
      const unsigned long long t1e = p;
      if (t1 < t1e) {  // two tokens (fewer: the line is skipped)
        if (!mtx_number(body, t0, t0e, &i) || !mtx_number(body, t1, t1e, &j)) flags |= kMtxBadNumber;
        else if (i == 0 || j == 0) flags |= kMtxZeroIndex;
        else if (i > n || j > n) flags |= kMtxOutOfRange;
        else edges = (symmetric && i != j) ? 2u : 1u;
      }
    }
    if (!kEmit) {
      count[l] = edges;
      if (flags) {
        atomicOr(err, flags);
        atomicMin(bad_line, l);
      }
    } else if (edges) {
      const unsigned long long o = at[l];
      keys[o] = ((i - 1) << 32) | (j - 1);
      if (edges == 2) keys[o + 1] = ((j - 1) << 32) | (i - 1);
    }
  }
}

struct LoadCount {
  const uint32_t* p;
  __device__ __forceinline__ unsigned long long operator()(unsigned long long i) const { return p[i]; }
};

// ---------------------------------------------------------------------------
// Stable LSD radix sort of u64 keys, 8 bits per pass.  Each block owns a
// contiguous segment; hist[d * blocks + b] counts digit d in block b's segment,
// its exclusive scan (digit-major) gives every (digit, block) its output start,
// and the scatter places the segment's keys in order: items go through in
// rounds of 256 (one per thread, in item order), ranked among equal digits by
// warp (match + popcount of the lower lanes) and by the warps before.
constexpr int kRadixThreads = 256;
constexpr int kRadixWarps = kRadixThreads / 32;

__device__ __forceinline__ unsigned long long radix_segment(unsigned long long count, uint32_t blocks, uint32_t b) {
  const unsigned long long per = (count + blocks - 1) / blocks;
  return min(count, per * b);
}

__global__ void __launch_bounds__(kRadixThreads) k_radix_hist(const unsigned long long* __restrict__ keys,
                                                              unsigned long long count, int shift,
                                                              uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const unsigned long long b0 = radix_segment(count, gridDim.x, blockIdx.x);
  const unsigned long long b1 = radix_segment(count, gridDim.x, blockIdx.x + 1);
  for (unsigned long long i = b0 + threadIdx.x; i < b1; i += kRadixThreads)
    atomicAdd(&h[(keys[i] >> shift) & 0xFF], 1u);
  __syncthreads();
  hist[threadIdx.x * gridDim.x + blockIdx.x] = h[threadIdx.x];
}

// kPay: a u32 payload travels with each key (pin -> pout), in the same order.
template <bool kPay>
__global__ void __launch_bounds__(kRadixThreads) k_radix_scatter(const unsigned long long* __restrict__ in,
                                                                 unsigned long long* __restrict__ out,
                                                                 unsigned long long count, int shift,
                                                                 const uint32_t* __restrict__ start,
                                                                 const uint32_t* __restrict__ pin,
                                                                 uint32_t* __restrict__ pout) {
  __shared__ uint32_t warp_cnt[kRadixWarps][256];
  __shared__ uint32_t run[256];
  const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  run[threadIdx.x] = start[threadIdx.x * gridDim.x + blockIdx.x];
#pragma unroll
  for (int w = 0; w < kRadixWarps; ++w) warp_cnt[w][threadIdx.x] = 0;
  __syncthreads();
  const unsigned long long b0 = radix_segment(count, gridDim.x, blockIdx.x);
  const unsigned long long b1 = radix_segment(count, gridDim.x, blockIdx.x + 1);
  for (unsigned long long r = b0; r < b1; r += kRadixThreads) {
    const unsigned long long i = r + threadIdx.x;
    const bool valid = i < b1;
    const unsigned long long k = valid ? in[i] : 0ull;
    const uint32_t pl = kPay && valid ? pin[i] : 0u;
    const uint32_t d = valid ? (uint32_t)((k >> shift) & 0xFF) : 256u;
    const unsigned same = __match_any_sync(0xFFFFFFFFu, d);
    const uint32_t in_warp = __popc(same & ((1u << lane) - 1));
    if (valid && in_warp == 0) warp_cnt[wid][d] = __popc(same);
    __syncthreads();
    if (valid) {
      uint32_t before = 0;
      for (uint32_t w = 0; w < wid; ++w) before += warp_cnt[w][d];
      out[run[d] + before + in_warp] = k;
      if (kPay) pout[run[d] + before + in_warp] = pl;
    }
    __syncthreads();
    // advance the digit's running start, clear the counts for the next round
    uint32_t tot = 0;
#pragma unroll
    for (int w = 0; w < kRadixWarps; ++w) {
      tot += warp_cnt[w][threadIdx.x];
      warp_cnt[w][threadIdx.x] = 0;
    }
    run[threadIdx.x] += tot;
    __syncthreads();
  }
}

// row lengths from the sorted keys (rows are contiguous runs of equal high words)
__global__ void __launch_bounds__(256) k_mtx_rows(const unsigned long long* __restrict__ keys, unsigned long long count,
                                                  uint32_t* __restrict__ deg) {
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (unsigned long long)gridDim.x * blockDim.x)
    atomicAdd(&deg[keys[i] >> 32], 1u);
}

__global__ void __launch_bounds__(256) k_mtx_columns(const unsigned long long* __restrict__ keys,
                                                     unsigned long long count, unsigned long long* __restrict__ nbr) {
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (unsigned long long)gridDim.x * blockDim.x)
    nbr[i] = keys[i] & 0xFFFFFFFFull;
}

}  // namespace sparx
