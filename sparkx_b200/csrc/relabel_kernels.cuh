// Vertex relabelling for locality: vertices take new ids in (floor(log2
// degree), id) order, within their own graph's id range in a union, and the
// CSR is rebuilt on them; the caller's
// slot s maps to the new slot rmap[s].  Rows are sorted by id, and within a
// degree bucket the new ids keep the old order, so each new row is the old
// row stably partitioned by its neighbours' buckets: no sort of the slots is
// needed.  On R-MAT-22 the same engine ran the bucket-ordered copy of the
// graph 32 ms faster than the original (support 86.5 -> 80.6 ms, peel 340.6
// -> 315.1 ms): edges of similar-degree vertices sit together, so the peel's
// random state and row reads fall on far fewer lines.  Below 2^26 slots it
// costs more than it saves (R-MAT-20 and 21: peel 5-6 ms slower), so the
// tuning turns it on only for large skewed graphs.
//   k_vertex_keys       ((member << 5 | bucket) << 32 | id) per vertex, for the
//                       radix passes (one for a single graph)
//   k_vertex_order      new id and new degree per vertex
//   k_relabel_rows      a warp per row of at most kRelabelWarpRow entries
//   k_relabel_rows_big  a block per longer row (the listed big rows)
// Both row kernels count the row's entries per bucket, scan the 32 counts,
// then place the entries chunk by chunk in their order: an entry's place is
// its bucket's cursor plus the same-bucket entries before it in the chunk.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sparx {

constexpr uint32_t kRelabelWarpRow = 2048;  // longer rows: a block each (the orientation's big-row list)

__device__ __forceinline__ uint32_t degree_bucket(uint32_t d) { return d > 1 ? 31u - __clz(d) : 0u; }

// Keys ((member << 5 | bucket) << 32 | id): in a union of G graphs (members
// by ascending first vertex `vb`) every vertex keeps to its member's id range.
__global__ void __launch_bounds__(256) k_vertex_keys(const uint32_t* __restrict__ off, uint32_t n,
                                                     const uint32_t* __restrict__ member_vb, uint32_t G,
                                                     unsigned long long* __restrict__ keys,
                                                     uint8_t* __restrict__ bucket) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    const uint32_t b = degree_bucket(__ldg(off + u + 1) - __ldg(off + u));
    uint32_t lo = 0, hi = G - 1;  // the last member whose first vertex is <= u
    while (lo < hi) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      if (__ldg(member_vb + mid) <= u) lo = mid; else hi = mid - 1;
    }
    keys[u] = ((unsigned long long)((lo << 5) | b) << 32) | u;
    bucket[u] = (uint8_t)b;
  }
}

__global__ void __launch_bounds__(256) k_vertex_order(const unsigned long long* __restrict__ sorted,
                                                      const uint32_t* __restrict__ off, uint32_t n,
                                                      uint32_t* __restrict__ newid, uint32_t* __restrict__ deg_new) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    const uint32_t u = (uint32_t)sorted[p];
    newid[u] = p;
    deg_new[p] = __ldg(off + u + 1) - __ldg(off + u);
  }
}

// Rows of at most kRelabelWarpRow entries, a warp each (rows over it are
// skipped: k_relabel_rows_big places them).
__global__ void __launch_bounds__(256) k_relabel_rows(const uint32_t* __restrict__ off,
                                                      const uint32_t* __restrict__ nbr, uint32_t n,
                                                      const uint32_t* __restrict__ newid,
                                                      const uint8_t* __restrict__ bucket,
                                                      const uint32_t* __restrict__ off_new,
                                                      uint32_t* __restrict__ nbr_new, uint32_t* __restrict__ rmap) {
  __shared__ uint32_t s_cur[8][32];
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  uint32_t* cur = s_cur[wib];  // the row's bucket counts, then the buckets' cursors
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = warp; u < n; u += nwarps) {
    const uint32_t b = __ldg(off + u), e = __ldg(off + u + 1);
    if (e - b > kRelabelWarpRow) continue;
    // per-bucket counts of the row, then their exclusive scan (lane = bucket)
    cur[lane] = 0;
    __syncwarp();
    for (uint32_t s = b + lane; s < e; s += 32) atomicAdd(&cur[bucket[__ldg(nbr + s)]], 1u);
    __syncwarp();
    const uint32_t c = cur[lane];
    uint32_t x = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
      if (lane >= (uint32_t)d) x += y;
    }
    const uint32_t base = __ldg(off_new + __ldg(newid + u));
    __syncwarp();
    cur[lane] = base + x - c;
    __syncwarp();
    for (uint32_t s0 = b; s0 < e; s0 += 32) {
      const uint32_t s = s0 + lane;
      const bool valid = s < e;
      const uint32_t v = valid ? __ldg(nbr + s) : 0u;
      const uint32_t bk = valid ? bucket[v] : 32u;
      const unsigned same = __match_any_sync(0xFFFFFFFFu, bk);
      const uint32_t rank = __popc(same & ((1u << lane) - 1));
      uint32_t at = 0;
      if (valid) at = cur[bk] + rank;
      __syncwarp();
      if (valid) {
        nbr_new[at] = __ldg(newid + v);
        rmap[s] = at;
        if (rank == 0) cur[bk] += __popc(same);
      }
      __syncwarp();
    }
  }
}

// The listed rows longer than kRelabelWarpRow, a block of 256 each: chunks of
// 256 entries, ranked across the block's warps through per-warp bucket counts.
__global__ void __launch_bounds__(256) k_relabel_rows_big(const uint32_t* __restrict__ off,
                                                          const uint32_t* __restrict__ nbr,
                                                          const uint32_t* __restrict__ list,
                                                          const uint32_t* __restrict__ count,
                                                          const uint32_t* __restrict__ newid,
                                                          const uint8_t* __restrict__ bucket,
                                                          const uint32_t* __restrict__ off_new,
                                                          uint32_t* __restrict__ nbr_new, uint32_t* __restrict__ rmap) {
  __shared__ uint32_t s_cnt[32];
  __shared__ uint32_t s_cur[32];
  __shared__ uint32_t s_wc[8][32];
  const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t nbig = *count;
  for (uint32_t r = blockIdx.x; r < nbig; r += gridDim.x) {
    const uint32_t u = list[r];
    const uint32_t b = __ldg(off + u), e = __ldg(off + u + 1);
    if (threadIdx.x < 32) s_cnt[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t s = b + threadIdx.x; s < e; s += blockDim.x) atomicAdd(&s_cnt[bucket[__ldg(nbr + s)]], 1u);
    __syncthreads();
    if (threadIdx.x < 32) {
      const uint32_t c = s_cnt[threadIdx.x];
      uint32_t x = c;
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, d);
        if (lane >= (uint32_t)d) x += y;
      }
      s_cur[threadIdx.x] = __ldg(off_new + __ldg(newid + u)) + x - c;
    }
    __syncthreads();
    for (uint32_t s0 = b; s0 < e; s0 += blockDim.x) {
      const uint32_t s = s0 + threadIdx.x;
      const bool valid = s < e;
      const uint32_t v = valid ? __ldg(nbr + s) : 0u;
      const uint32_t bk = valid ? bucket[v] : 32u;
      const unsigned same = __match_any_sync(0xFFFFFFFFu, bk);
      const uint32_t rank = __popc(same & ((1u << lane) - 1));
      s_wc[wib][lane] = 0;
      __syncwarp();
      if (valid && rank == 0) s_wc[wib][bk] = __popc(same);
      __syncthreads();
      if (valid) {
        uint32_t before = 0;
        for (uint32_t w = 0; w < wib; ++w) before += s_wc[w][bk];
        const uint32_t at = s_cur[bk] + before + rank;
        nbr_new[at] = __ldg(newid + v);
        rmap[s] = at;
      }
      __syncthreads();
      if (threadIdx.x < 32) {
        uint32_t t = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) t += s_wc[w][threadIdx.x];
        s_cur[threadIdx.x] += t;
      }
      __syncthreads();
    }
  }
}

}  // namespace sparx
