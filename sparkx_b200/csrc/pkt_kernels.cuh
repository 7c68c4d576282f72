// Device kernels of the B200 PKT k-truss engine (sm_100a).
//
// One "union" CSR holds every graph of a launch as a disjoint union (vertex
// ids, slots and edge ids offset per member), so the preparation kernels
// (narrowing, orientation, support, finalize) see a single graph.  The peel
// runs a per-member state machine: each member has its own level, phase and
// frontier, and one device "wave" advances every member by one step (a level
// scan or one PKT sub-level).  A single graph is a union of one.
//
// Layout in HBM (u32 indices: width < 2^32, m < 2^28 per member):
//   off[n+1], nbr[width]        narrowed CSR, rows sorted ascending
//   row0[width] (u64)           the same rows as (id | edge id << 32) pairs, in
//                               slot order (edge id 0xFFFFFFFF: self-loop)
//   dplus[n], opos[n+1]         degree-ordered out-degree and its prefix
//   ocol[m], osrc[m]            oriented edge e = (osrc[e] -> ocol[e]); e is the
//                               undirected edge id; rank(osrc) < rank(ocol)
//   es[m] (int2)                per edge {support / PKT level, tag}: the tag is
//                               the wave at which the edge is processed
//                               (0xFFFFFFFF: not yet queued); one 8-byte word so
//                               a triangle's two other edges cost two sectors
//   act[2][m], q[2][m] (u64)    per-member active lists and frontier queues,
//   qd[2][m] (uint4)            with each queued edge's row descriptor;
//                               segment [eb_g, eb_g + m_g) for member g
//   working CSR (off, row)      the peel's view: row0 at first, then rebuilt
//                               without processed edges whenever the live
//                               edges fill at most 85% of it (two ping-pong
//                               buffers)
//   hub maps                    neighbour id -> edge id for the highest-degree
//                               vertices (each spans its own member's ids)
//   row hash tables (u64)       open-addressed (id | edge id << 32) entries,
//                               2^(1+ceil(log2 d)) of them at 4 * off[v] for
//                               rows of degree >= the tuning's floor
//   vinfo[n] (u64)              per vertex: hub base (kVinfoHub set) or the
//                               table's (log2 size << 32 | position), 0: none
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace sparx {

constexpr uint32_t kInvalid = 0xFFFFFFFFu;
constexpr uint32_t kTagActive = 0xFFFFFFFFu;
constexpr int kWorkBits = 36;  // packed queue counter: (count << 36) | work
constexpr unsigned long long kWorkMask = (1ull << kWorkBits) - 1;
constexpr int kEidBits = 28;   // queue entry: (wstart << 28) | local eid
constexpr uint32_t kEidMask = (1u << kEidBits) - 1;
constexpr unsigned kFull = 0xFFFFFFFFu;

// error flags (device bitmask)
enum : uint32_t {
  kErrRange = 1u,       // neighbour id >= n
  kErrUnsorted = 2u,    // row not ascending
  kErrMulti = 4u,       // duplicate slot
  kErrAsym = 8u,        // reverse slot missing
  kErrOverflowU8 = 16u, // truss > 255 with 8-bit output / level 255 in u8 mode
  kErrCapacity = 32u,   // packed counter or queue capacity exceeded
  kErrTimeout = 64u,    // device time budget exhausted
  kErrOffsets = 128u,   // offsets not monotone / wrong total
  kErrWaves = 256u,     // wave bound exceeded (no progress)
  kErrInternal = 512u,  // inconsistent wave layout (a device loop refused to spin)
};

enum : uint32_t { kPhaseScan0 = 0, kPhaseScan = 1, kPhaseProc = 2, kPhaseDone = 3 };

constexpr uint32_t kVinfoHub = 0x80000000u;  // Union::vinfo: the longer row's vertex has a hub map

struct Union {  // the prepared concatenated graph, as the peel sees it
  const uint32_t* off;             // working row offsets
  const unsigned long long* row;   // working rows: (id | edge id << 32)
  const uint32_t* opos;
  const uint32_t* ocol;
  const uint32_t* osrc;
  int2* es;
  uint32_t* act[2];
  unsigned long long* q[2];
  uint4* qd[2];                    // per queue entry {short row start, length, long row begin, end}
  const uint32_t* hub_slot;        // vertex -> hub map index or kInvalid; nullptr = no hub maps
  const uint32_t* hub_map;         // map pool: hub k's neighbour id w -> hub_map[hub_base[k] + w]
  const uint32_t* hub_base;        // per hub: its map's start in the pool minus its member's first
                                   // vertex id (u32 arithmetic, so base + w wraps into the map)
  const unsigned long long* hpool; // row hash tables (nullptr = none): vertex v's at 4 * off0[v]
  const uint32_t* off0;            // the rows' original offsets (hash table positions)
  uint2* qh[2];                    // per queue entry: {hash table position, log2 capacity} or 0
  const unsigned long long* vinfo; // per vertex, what a frontier edge's longer row offers (k_vinfo):
                                   // kVinfoHub | hub map base, or {table position, log2 capacity},
                                   // or 0; nullptr when there are neither hub maps nor tables
  uint32_t hash_min;               // rows of at least this degree have a hash table (0: none)
  uint32_t n;
  uint32_t m;
  uint32_t width;
  uint32_t G;
};

// The peel's arrays that stay where they are for a whole run.  The wave
// kernel takes them as a by-value parameter, so the compiler can re-read any
// of them from the parameter bank instead of holding (or spilling) it; only
// the working rows, which a compaction replaces, are read from the Union.
struct PeelArrays {
  const uint32_t* ocol;
  const uint32_t* osrc;
  int2* es;
  uint32_t* act0;
  uint32_t* act1;
  unsigned long long* q0;
  unsigned long long* q1;
  uint4* qd0;
  uint4* qd1;
  const uint32_t* hub_slot;
  const uint32_t* hub_map;
  const uint32_t* hub_base;
  const uint32_t* mu;    // multigraphs: multiplicity per edge id (nullptr: simple graph)
  const unsigned long long* hpool;
  const uint32_t* off0;
  uint2* qh0;
  uint2* qh1;
  uint32_t n;
  uint32_t merge_ratio;  // merge the rows when the longer is at most this many times the shorter
  uint32_t hash_min;
  uint32_t pad;
};

// Field-by-field copy of a device-resident Union into registers (a struct
// copy would land in local memory).
struct UnionRegs {
  const uint32_t* __restrict__ off;
  const unsigned long long* __restrict__ row;
  const uint32_t* __restrict__ ocol;
  const uint32_t* __restrict__ osrc;
  int2* es;
  uint32_t* act0;
  uint32_t* act1;
  unsigned long long* q0;
  unsigned long long* q1;
  uint4* qd0;
  uint4* qd1;
  const uint32_t* __restrict__ hub_slot;
  const uint32_t* __restrict__ hub_map;
  const uint32_t* __restrict__ hub_base;
  const uint32_t* __restrict__ mu;
  const unsigned long long* __restrict__ hpool;
  const uint32_t* __restrict__ off0;
  uint2* qh0;
  uint2* qh1;
  const unsigned long long* __restrict__ vinfo;
  uint32_t n;
  uint32_t hash_min;
  __device__ __forceinline__ explicit UnionRegs(const Union* p)
      : off(p->off), row(p->row), ocol(p->ocol), osrc(p->osrc), es(p->es),
        act0(p->act[0]), act1(p->act[1]), q0(p->q[0]), q1(p->q[1]),
        qd0(p->qd[0]), qd1(p->qd[1]), hub_slot(p->hub_slot), hub_map(p->hub_map), hub_base(p->hub_base),
        mu(nullptr), hpool(p->hpool), off0(p->off0), qh0(p->qh[0]), qh1(p->qh[1]), vinfo(p->vinfo), n(p->n),
        hash_min(p->hash_min) {}
  __device__ __forceinline__ UnionRegs(const Union* p, const PeelArrays& a)
      : off(p->off), row(p->row), ocol(a.ocol), osrc(a.osrc), es(a.es),
        act0(a.act0), act1(a.act1), q0(a.q0), q1(a.q1),
        qd0(a.qd0), qd1(a.qd1), hub_slot(a.hub_slot), hub_map(a.hub_map), hub_base(a.hub_base), mu(a.mu),
        hpool(a.hpool), off0(a.off0), qh0(a.qh0), qh1(a.qh1), vinfo(nullptr), n(a.n), hash_min(a.hash_min) {}
};

// Row hash tables: vertex v of original degree d >= hash_min (and no hub map)
// has an open-addressed table of its (neighbour id | edge id << 32) pairs with
// 2^(1 + ceil(log2 d)) entries (at most 4d, so at 4 * off0[v] the tables of
// consecutive vertices never overlap), probed linearly from a multiplicative
// hash of the id; an empty entry is all ones.
__device__ __forceinline__ uint32_t hash_log2cap(uint32_t d) { return 1u + (d > 1 ? 32u - __clz(d - 1) : 0u); }
__device__ __forceinline__ uint32_t hash_first(uint32_t w, uint32_t lg) { return (w * 0x9E3779B1u) >> (32 - lg); }

// A queue-entry descriptor whose longer row belongs to a hub carries kHubDesc
// in place of the longer row's begin and the hub's map base in place of its
// end (row positions stay below 2^31 whenever hub maps are built).
constexpr uint32_t kHubDesc = 0x80000000u;

struct Member {  // static per-member ranges
  uint32_t vb, n;   // vertices [vb, vb + n)
  uint32_t sb, w;   // slots [sb, sb + w)
  uint32_t eb, m;   // edge ids [eb, eb + m)
};

struct MemberState {  // dynamic per-member peel state
  uint32_t phase, level, act_sel, q_sel;
  uint32_t act_count;
  uint32_t kept;            // wave accumulator: active edges kept by a scan
  uint32_t min_kept;        // wave accumulator: min support among kept
  uint32_t processed;       // edges whose truss is fixed
  unsigned long long curr;  // packed (count << 36 | work) of the frontier being processed
  unsigned long long next;  // wave accumulator: frontier being built
  uint32_t levels, max_level, waves, pad;
};

struct Control {
  uint32_t G;
  uint32_t wave;       // current wave number (>= 1)
  uint32_t done;
  uint32_t err;
  unsigned long long total_work;
  unsigned long long max_waves;
  unsigned long long t_start;
  unsigned long long timeout_ns;
  unsigned long long waves_run;
  // work counters (roofline accounting)
  unsigned long long el_proc;     // frontier elements searched
  unsigned long long el_scan;     // active-list entries scanned
  unsigned long long hits;        // triangles found by frontier elements
  unsigned long long edges_proc;  // frontier edges processed
  unsigned long long csr_slots;   // entries in the working rows
  unsigned long long compact_min; // do not compact working rows smaller than this
  uint32_t exit_reason;           // why the loop stopped: kExit*
  uint32_t blocks_done;           // wave blocks finished (the last one plans the next wave)
  uint32_t compactions;
  uint32_t compact_pct;           // compact when live entries fill at most this % of the working rows
  uint32_t pad0;
  unsigned long long merge_iters; // warp iterations resolved by the row merge
  unsigned long long lane_iters;  // warp iterations resolved by per-lane searches
  unsigned long long merge_chunks;// 32-entry chunks of longer rows read by merges
  // optional wave trace: per planned wave {start time (ns), work, members in
  // a frontier step, members in a scan}; nullptr = off
  ulonglong4* trace;
  unsigned long long trace_cap;
  // served unions: stop when a member finishes (its result can go out at
  // once), and when the host-mapped word `admit` is set (requests wait to
  // join); nullptr / 0 = off
  const volatile uint32_t* admit;
  uint32_t notify_done;
  uint32_t pad1;
};

enum : uint32_t { kExitNone = 0, kExitDone = 1, kExitCompact = 2, kExitError = 3, kExitMember = 4, kExitAdmit = 5 };

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ uint32_t deg_of(const uint32_t* off, uint32_t v) {
  return __ldg(off + v + 1) - __ldg(off + v);
}

// degree order, ties by id: the orientation rank
__device__ __forceinline__ bool rank_less(uint32_t du, uint32_t u, uint32_t dv, uint32_t v) {
  return du < dv || (du == dv && u < v);
}

// lower_bound of x in sorted a[lo, hi)
__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t* __restrict__ a, uint32_t lo,
                                                    uint32_t hi, uint32_t x) {
  while (lo < hi) {
    uint32_t mid = lo + ((hi - lo) >> 1);
    if (__ldg(a + mid) < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// Position of id w in the sorted row pairs [lo, hi) or kInvalid.  Ids inside
// a row are spread close to uniformly (vertex ids carry no degree order), so
// up to three interpolation probes narrow a long row before the binary search:
// on a 160k-entry hub row that is ~6 dependent loads instead of ~17.
__device__ __forceinline__ uint32_t find_in_row(const unsigned long long* __restrict__ row, uint32_t lo,
                                                uint32_t hi, uint32_t w) {
#pragma unroll 1
  for (int it = 0; it < 3 && hi - lo > 48; ++it) {
    const uint32_t a = (uint32_t)__ldg(row + lo), b = (uint32_t)__ldg(row + hi - 1);
    if (w < a || w > b) return kInvalid;
    // fraction in [0, 1); the clamp keeps g in [lo, hi - 1] whatever the rounding
    const float frac = __fdividef((float)(w - a), (float)(b - a) + 1.0f);
    const uint32_t span = hi - 1 - lo;
    const uint32_t g = lo + min(span, (uint32_t)(frac * (float)span));
    const uint32_t x = (uint32_t)__ldg(row + g);
    if (x == w) return g;
    if (x < w) lo = g + 1; else hi = g;
  }
  const uint32_t end = hi;
  while (lo < hi) {
    const uint32_t mid = lo + ((hi - lo) >> 1);
    if ((uint32_t)__ldg(row + mid) < w) lo = mid + 1; else hi = mid;
  }
  return (lo < end && (uint32_t)__ldg(row + lo) == w) ? lo : kInvalid;
}

// Warp-cooperative searches over a non-decreasing key(x).  Each step gathers
// 32 evenly spaced keys with one load per lane and keeps the stretch between
// the two samples that bracket the target, so a span of n entries costs
// ceil(log32 n) + 1 dependent gathers instead of log2 n dependent loads.  All
// lanes must call them with the same arguments.

// largest x in [lo, hi] with key(x) <= t; requires key(lo) <= t
template <class KeyF>
__device__ __forceinline__ uint32_t warp_last_le(const KeyF& key, uint32_t lo, uint32_t hi,
                                                 unsigned long long t) {
  const uint32_t lane = lane_id();
  while (hi - lo >= 32) {
    const uint32_t step = (hi - lo) / 32 + 1;
    const unsigned long long s = (unsigned long long)lo + (unsigned long long)lane * step;
    const bool le = s <= hi && key((uint32_t)s) <= t;
    const uint32_t b = __ballot_sync(kFull, le) | 1u;  // key(lo) <= t
    const uint32_t tl = 31 - __clz(b);
    lo += tl * step;
    hi = min(hi, lo + step - 1);
  }
  const bool le = lo + lane <= hi && key(lo + lane) <= t;
  const uint32_t b = __ballot_sync(kFull, le) | 1u;
  return lo + 31 - __clz(b);
}

// first x in [lo, hi) with key(x) >= t, or hi
template <class KeyF>
__device__ __forceinline__ uint32_t warp_lower_bound(const KeyF& key, uint32_t lo, uint32_t hi,
                                                     unsigned long long t) {
  const uint32_t lane = lane_id();
  while (hi - lo > 32) {
    const uint32_t step = (hi - lo + 31) / 32;
    const unsigned long long s = (unsigned long long)lo + (unsigned long long)lane * step;
    const bool lt = s < hi && key((uint32_t)s) < t;
    const uint32_t b = __ballot_sync(kFull, lt);
    if (b == 0) return lo;
    const uint32_t tl = 31 - __clz(b);
    // key(lo + tl*step) < t <= key(lo + (tl+1)*step) (or past hi)
    const uint32_t nlo = lo + tl * step + 1;
    hi = min(hi, lo + (tl + 1) * step);
    lo = nlo;
  }
  const bool lt = lo + lane < hi && key(lo + lane) < t;
  return lo + __popc(__ballot_sync(kFull, lt));
}

struct PrefKey {
  const unsigned long long* p;
  __device__ __forceinline__ unsigned long long operator()(uint32_t x) const { return p[x]; }
};

struct RowIdKey {
  const unsigned long long* row;
  __device__ __forceinline__ unsigned long long operator()(uint32_t x) const {
    return (uint32_t)__ldg(row + x);
  }
};

__device__ __forceinline__ unsigned long long warp_incl_scan(unsigned long long v) {
  const uint32_t lane = lane_id();
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned long long o = __shfl_up_sync(kFull, v, d);
    if (lane >= (uint32_t)d) v += o;
  }
  return v;
}

// ---------------------------------------------------------------------------
// Kernel A: narrowing (u64 ids -> u32) with range check.  Grid-stride.
__global__ void k_narrow_ids(const unsigned long long* __restrict__ src, uint32_t* __restrict__ dst,
                             unsigned long long count, unsigned long long n_limit, uint32_t base,
                             uint32_t* __restrict__ err) {
  unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  bool bad = false;
  for (; i < count; i += stride) {
    unsigned long long x = src[i];
    bad |= x >= n_limit;
    dst[i] = (uint32_t)x + base;
  }
  if (bad) atomicOr(err, kErrRange);
}

// u32 ids: range check, optionally copying with a base shift (dst may be null)
__global__ void k_range_ids(const uint32_t* __restrict__ ids, uint32_t* __restrict__ dst,
                            unsigned long long count, uint32_t n_limit, uint32_t base,
                            uint32_t* __restrict__ err) {
  unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  bool bad = false;
  for (; i < count; i += stride) {
    uint32_t x = __ldg(ids + i);
    bad |= x >= n_limit;
    if (dst) dst[i] = x + base;
  }
  if (bad) atomicOr(err, kErrRange);
}

// offsets u64 -> u32 (+ a member's slot base), checking monotonicity inside
// this chunk; first/last values are checked when first_expect / last_expect
// are >= 0 (device inputs), else by the host.
__global__ void k_narrow_offsets(const unsigned long long* __restrict__ src, uint32_t* __restrict__ dst,
                                 uint32_t count, uint32_t slot_base, long long first_expect,
                                 long long last_expect, uint32_t* __restrict__ err) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t stride = gridDim.x * blockDim.x;
  bool bad = false;
  for (; i < count; i += stride) {
    const unsigned long long x = src[i];
    if (i == 0 && first_expect >= 0) bad |= x != (unsigned long long)first_expect;
    if (i + 1 == count && last_expect >= 0) bad |= x != (unsigned long long)last_expect;
    if (i + 1 < count) bad |= src[i + 1] < x;
    dst[i] = (uint32_t)x + slot_base;
  }
  if (bad) atomicOr(err, kErrOffsets);
}


// ---------------------------------------------------------------------------
// Exclusive scan across the block (all threads call it); `total` is the
// block sum.  smem_warp holds one value per warp.
template <class T>
__device__ __forceinline__ T block_exclusive_scan(T x, T* smem_warp, T& total) {
  const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
  T v = x;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    T o = __shfl_up_sync(kFull, v, d);
    if (lane >= (uint32_t)d) v += o;
  }
  if (lane == 31) smem_warp[wid] = v;
  __syncthreads();
  if (wid == 0) {
    const int nw = blockDim.x >> 5;
    T w = lane < (uint32_t)nw ? smem_warp[lane] : T(0);
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      T o = __shfl_up_sync(kFull, w, d);
      if (lane >= (uint32_t)d) w += o;
    }
    if (lane < (uint32_t)nw) smem_warp[lane] = w;
  }
  __syncthreads();
  T warp_off = wid ? smem_warp[wid - 1] : T(0);
  total = smem_warp[(blockDim.x >> 5) - 1];
  __syncthreads();
  return warp_off + v - x;
}

// Row kernels take 32 consecutive vertices per warp: a row of at most
// kLaneRow entries is walked by its own lane, longer rows by the whole warp
// one at a time, so low-degree vertices (most of a skewed graph) keep all
// lanes busy.
constexpr uint32_t kLaneRow = 32;

// Rows longer than kWarpRow entries (by original degree) are oriented and
// compacted by a block each (the *_big kernels over the list k_big_rows
// builds); the others by their lane or their warp.
constexpr uint32_t kWarpRow = 2048;

__device__ __forceinline__ bool big_row(const uint32_t* __restrict__ off0, uint32_t u) {
  return __ldg(off0 + u + 1) - __ldg(off0 + u) > kWarpRow;
}

__global__ void __launch_bounds__(256) k_big_rows(const uint32_t* __restrict__ off0, uint32_t n,
                                                  uint32_t* __restrict__ list, uint32_t* __restrict__ count) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x)
    if (big_row(off0, u)) list[atomicAdd(count, 1u)] = u;
}

// Kernel B1: per-row validation + oriented out-degree.
//   rows strictly ascending (equal -> multigraph), counts self-loops, and
//   dplus[u] = #{v in N(u): v != u, rank(u) < rank(v)}.
__global__ void __launch_bounds__(256) k_orient_count(const uint32_t* __restrict__ off,
                                                      const uint32_t* __restrict__ nbr, uint32_t n,
                                                      uint32_t* __restrict__ dplus,
                                                      unsigned long long* __restrict__ self_loops,
                                                      uint32_t* __restrict__ err,
                                                      uint32_t* __restrict__ max_dplus,
                                                      const uint32_t* __restrict__ big_list,
                                                      const uint32_t* __restrict__ big_count) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  uint32_t flags = 0, mxd = 0;
  unsigned long long selfc = 0;
  for (uint32_t base = warp * 32; base < n; base += nwarps * 32) {
    const uint32_t u = base + lane;
    uint32_t b = 0, e = 0;
    if (u < n) { b = __ldg(off + u); e = __ldg(off + u + 1); }
    uint32_t cnt = 0;
    if (u < n && e - b <= kLaneRow) {
      uint32_t prev = 0;
      for (uint32_t s = b; s < e; ++s) {
        const uint32_t v = __ldg(nbr + s);
        if (s > b && prev < n) {  // the pair (prev, v), judged as the warp path does
          if (v == prev) flags |= kErrMulti;
          else if (v < prev) flags |= kErrUnsorted;
        }
        prev = v;
        if (v >= n) { flags |= kErrRange; continue; }
        if (v == u) { selfc++; continue; }
        cnt += rank_less(e - b, u, deg_of(off, v), v);
      }
    }
    const bool blk = u < n && e - b > kWarpRow;  // counted below, a block per row
    unsigned big = __ballot_sync(kFull, u < n && e - b > kLaneRow && !blk);
    while (big) {
      const int j = __ffs(big) - 1;
      big &= big - 1;
      const uint32_t bu = base + j, bb = __shfl_sync(kFull, b, j), be = __shfl_sync(kFull, e, j);
      const uint32_t du = be - bb;
      uint32_t c = 0;
      for (uint32_t s = bb + lane; s < be; s += 32) {
        const uint32_t v = __ldg(nbr + s);
        if (v >= n) { flags |= kErrRange; continue; }
        if (s + 1 < be) {
          const uint32_t nx = __ldg(nbr + s + 1);
          if (nx == v) flags |= kErrMulti;
          else if (nx < v) flags |= kErrUnsorted;
        }
        if (v == bu) { selfc++; continue; }
        c += rank_less(du, bu, deg_of(off, v), v);
      }
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) c += __shfl_xor_sync(kFull, c, d);
      if (lane == (uint32_t)j) cnt = c;
    }
    if (u < n && !blk) {
      dplus[u] = cnt;
      mxd = max(mxd, cnt);
    }
  }
  // rows longer than kWarpRow: block-wide, one row at a time
  __shared__ unsigned long long s_red[32];
  const uint32_t nbig = *big_count;
  for (uint32_t r = blockIdx.x; r < nbig; r += gridDim.x) {
    const uint32_t bu = big_list[r];
    const uint32_t bb = __ldg(off + bu), be = __ldg(off + bu + 1), du = be - bb;
    unsigned long long c = 0;
    for (uint32_t s = bb + threadIdx.x; s < be; s += blockDim.x) {
      const uint32_t v = __ldg(nbr + s);
      if (v >= n) { flags |= kErrRange; continue; }
      if (s + 1 < be) {
        const uint32_t nx = __ldg(nbr + s + 1);
        if (nx == v) flags |= kErrMulti;
        else if (nx < v) flags |= kErrUnsorted;
      }
      if (v == bu) { selfc++; continue; }
      c += rank_less(du, bu, deg_of(off, v), v);
    }
    unsigned long long total;
    block_exclusive_scan<unsigned long long>(c, s_red, total);
    if (threadIdx.x == 0) {
      dplus[bu] = (uint32_t)total;
      mxd = max(mxd, (uint32_t)total);
    }
  }
  if (flags) atomicOr(err, flags);
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    selfc += __shfl_down_sync(kFull, selfc, d);
    mxd = max(mxd, __shfl_down_sync(kFull, mxd, d));
  }
  if (lane == 0 && selfc) atomicAdd(self_loops, selfc);
  if (lane == 0 && mxd) atomicMax(max_dplus, mxd);
}

// Kernel B2: fill oriented lists (kept in id order) and, for each vertex's
// out-slots, the (id | edge id << 32) pair of row0; self-loop slots get edge id
// 0xFFFFFFFF.  In-slots are left to B3: owner[s] = u marks them (kInvalid for
// the others).
__device__ __forceinline__ unsigned long long make_pair(uint32_t id, uint32_t e) {
  return (unsigned long long)id | ((unsigned long long)e << 32);
}

__global__ void __launch_bounds__(256) k_orient_fill(const uint32_t* __restrict__ off,
                                                     const uint32_t* __restrict__ nbr, uint32_t n,
                                                     const uint32_t* __restrict__ opos,
                                                     uint32_t* __restrict__ ocol,
                                                     uint32_t* __restrict__ osrc,
                                                     unsigned long long* __restrict__ row0,
                                                     uint32_t* __restrict__ owner,
                                                     const uint32_t* __restrict__ big_list,
                                                     const uint32_t* __restrict__ big_count) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t base0 = warp * 32; base0 < n; base0 += nwarps * 32) {
    const uint32_t u = base0 + lane;
    uint32_t b = 0, e = 0;
    if (u < n) { b = __ldg(off + u); e = __ldg(off + u + 1); }
    if (u < n && e - b <= kLaneRow) {
      uint32_t p = __ldg(opos + u);
      for (uint32_t s = b; s < e; ++s) {
        const uint32_t v = __ldg(nbr + s);
        uint32_t own = kInvalid;
        if (v == u || v >= n) {
          row0[s] = make_pair(v, kInvalid);
        } else if (rank_less(e - b, u, deg_of(off, v), v)) {
          ocol[p] = v;
          osrc[p] = u;
          row0[s] = make_pair(v, p);
          ++p;
        } else {
          own = u;
        }
        owner[s] = own;
      }
    }
    unsigned big = __ballot_sync(kFull, u < n && e - b > kLaneRow && e - b <= kWarpRow);
    while (big) {
      const int j = __ffs(big) - 1;
      big &= big - 1;
      const uint32_t bu = base0 + j, bb = __shfl_sync(kFull, b, j), be = __shfl_sync(kFull, e, j);
      const uint32_t du = be - bb;
      uint32_t p0 = __ldg(opos + bu);
      for (uint32_t s0 = bb; s0 < be; s0 += 32) {
        const uint32_t s = s0 + lane;
        bool out = false;
        uint32_t v = 0;
        if (s < be) {
          v = __ldg(nbr + s);
          uint32_t own = kInvalid;
          if (v == bu || v >= n) row0[s] = make_pair(v, kInvalid);
          else if (rank_less(du, bu, deg_of(off, v), v)) out = true;
          else own = bu;
          owner[s] = own;
        }
        const unsigned bal = __ballot_sync(kFull, out);
        if (out) {
          const uint32_t p = p0 + __popc(bal & ((1u << lane) - 1));
          ocol[p] = v;
          osrc[p] = bu;
          row0[s] = make_pair(v, p);
        }
        p0 += __popc(bal);
      }
    }
  }
  // rows longer than kWarpRow: a block per row, out-slots placed in order by
  // a block-wide scan over chunks of four consecutive slots per thread
  __shared__ uint32_t s_scan[32];
  const uint32_t nbig = *big_count;
  for (uint32_t r = blockIdx.x; r < nbig; r += gridDim.x) {
    const uint32_t bu = big_list[r];
    const uint32_t bb = __ldg(off + bu), be = __ldg(off + bu + 1), du = be - bb;
    uint32_t p0 = __ldg(opos + bu);
    for (uint32_t base = bb; base < be; base += 4 * blockDim.x) {
      const uint32_t s0 = base + 4 * threadIdx.x;
      uint32_t v[4], outm = 0, nout = 0;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        v[i] = 0;
        const uint32_t s = s0 + i;
        if (s < be) {
          v[i] = __ldg(nbr + s);
          uint32_t own = kInvalid;
          if (v[i] == bu || v[i] >= n) row0[s] = make_pair(v[i], kInvalid);
          else if (rank_less(du, bu, deg_of(off, v[i]), v[i])) { outm |= 1u << i; ++nout; }
          else own = bu;
          owner[s] = own;
        }
      }
      uint32_t total;
      uint32_t p = p0 + block_exclusive_scan<uint32_t>(nout, s_scan, total);
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (outm & (1u << i)) {
          ocol[p] = v[i];
          osrc[p] = bu;
          row0[s0 + i] = make_pair(v[i], p);
          ++p;
        }
      p0 += total;
    }
  }
}

// Kernel B3: in-slots (owner[s] = u: rank(v) < rank(u)) take the id of v's
// out-slot to u, found by binary search in v's oriented list; slot-parallel.
// Missing -> asymmetric.
__global__ void __launch_bounds__(256) k_orient_reverse(const uint32_t* __restrict__ nbr,
                                                        const uint32_t* __restrict__ owner,
                                                        unsigned long long width,
                                                        const uint32_t* __restrict__ opos,
                                                        const uint32_t* __restrict__ ocol,
                                                        unsigned long long* __restrict__ row0,
                                                        uint32_t* __restrict__ err) {
  bool bad = false;
  for (unsigned long long s = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; s < width;
       s += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t u = __ldg(owner + s);
    if (u == kInvalid) continue;
    const uint32_t v = __ldg(nbr + s);
    const uint32_t lo = __ldg(opos + v), hi = __ldg(opos + v + 1);
    const uint32_t p = lower_bound_u32(ocol, lo, hi, u);
    if (p < hi && __ldg(ocol + p) == u) {
      row0[s] = make_pair(v, p);
    } else {
      row0[s] = make_pair(v, kInvalid);
      bad = true;
    }
  }
  if (bad) atomicOr(err, kErrAsym);
}

// ---------------------------------------------------------------------------
// Exclusive scans (reduce-then-scan, 3 kernels), with the input produced by a
// functor so work values need not be materialised.
constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;


template <class T, class F>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(F f, unsigned long long count, T* tile_sums) {
  __shared__ T sw[32];
  const unsigned long long base = (unsigned long long)blockIdx.x * kScanTile;
  T acc = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    unsigned long long i = base + (unsigned long long)j * kScanThreads + threadIdx.x;
    if (i < count) acc += f(i);
  }
  T total;
  block_exclusive_scan<T>(acc, sw, total);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

template <class T>
__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(T* tile_sums, unsigned long long tiles, T* grand_total) {
  __shared__ T sw[32];
  T carry = 0;
  for (unsigned long long b = 0; b < tiles; b += kScanThreads) {
    unsigned long long i = b + threadIdx.x;
    T x = i < tiles ? tile_sums[i] : T(0);
    T total;
    T ex = block_exclusive_scan<T>(x, sw, total);
    if (i < tiles) tile_sums[i] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) *grand_total = carry;
}

// out[i] = exclusive prefix; out[count] = total
template <class T, class F>
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(F f, unsigned long long count, const T* tile_offsets,
                                                             T* out) {
  __shared__ T sw[32];
  const unsigned long long base = (unsigned long long)blockIdx.x * kScanTile;
  // each thread owns kScanItems consecutive items
  const unsigned long long my = base + (unsigned long long)threadIdx.x * kScanItems;
  T vals[kScanItems];
  T acc = 0;
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    unsigned long long i = my + j;
    vals[j] = i < count ? f(i) : T(0);
    acc += vals[j];
  }
  T total;
  T ex = block_exclusive_scan<T>(acc, sw, total) + tile_offsets[blockIdx.x];
#pragma unroll
  for (int j = 0; j < kScanItems; ++j) {
    unsigned long long i = my + j;
    if (i < count) out[i] = ex;
    ex += vals[j];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[count] = ex;
}

struct LoadU32 {
  const uint32_t* p;
  __device__ __forceinline__ uint32_t operator()(unsigned long long i) const { return __ldg(p + i); }
};

// support work of oriented edge e = min(d+(src), d+(dst))
#ifndef SPARX_SAMPLED_LIST
#define SPARX_SAMPLED_LIST 64
#endif
// longer lists from this length on are searched through 32 samples
constexpr uint32_t kSampledList = SPARX_SAMPLED_LIST;

struct SupportWork {
  const uint32_t* opos;
  const uint32_t* osrc;
  const uint32_t* ocol;
  __device__ __forceinline__ unsigned long long operator()(unsigned long long e) const {
    uint32_t a = __ldg(osrc + e), b = __ldg(ocol + e);
    uint32_t da = __ldg(opos + a + 1) - __ldg(opos + a);
    uint32_t db = __ldg(opos + b + 1) - __ldg(opos + b);
    return min(da, db);
  }
};

// ---------------------------------------------------------------------------
// Kernel C (balanced form): per oriented edge e = (a -> b), each element of the
// shorter of N+(a), N+(b) is searched in the longer; a hit c closes the
// triangle (a, b, c), credited on e, (a -> c) and (b -> c).  Work elements are
// spread evenly over warps through the exclusive prefix `spref`; a warp owns a
// contiguous chunk and walks it 32 elements at a time.
struct PrefStart {
  const unsigned long long* p;
  __device__ __forceinline__ unsigned long long operator()(uint32_t x) const { return p[x]; }
};

template <class StartF>
__device__ __forceinline__ uint32_t window_find(const StartF& start, uint32_t i, uint32_t count,
                                                unsigned long long j, bool valid);

// 8 resident blocks per SM (32 registers): the pass is latency-bound and
// loses more to fewer warps than to the few spilled values.
//
// kMulti (multigraphs, `mu` = multiplicity per edge id): a triangle of pairs
// (e, f, h) stands for mu_e * mu_f * mu_h triangles of copies, so a copy of e
// is credited mu_f * mu_h (each hit lane adds its own product; the one-atomic
// run credit of the simple form is for unit weights only).
//
// kHash: out-lists of at least hash_min entries have an open-addressed table
// of (id | position << 32) at 4 * their start in `hpool` (k_table_fill with
// OutListSource, the same layout as the peel's row tables), probed instead of
// searched.
__device__ __forceinline__ uint32_t probe_list(const unsigned long long* __restrict__ hpool, uint32_t lb,
                                               uint32_t len, uint32_t c) {
  const uint32_t lg = hash_log2cap(len), mask = (1u << lg) - 1;
  const unsigned long long* tb = hpool + 4ull * lb;
  uint32_t at = hash_first(c, lg);
#pragma unroll 1
  for (uint32_t it = 0; it <= mask; ++it) {
    const unsigned long long en = __ldg(tb + at);
    const uint32_t id = (uint32_t)en;
    if (id == c) return (uint32_t)(en >> 32);
    if (id == kInvalid) return kInvalid;
    at = (at + 1) & mask;
  }
  return kInvalid;
}

#ifndef SPARX_SUP_SAMPLES
#define SPARX_SUP_SAMPLES 2  // samples of a long out-list per lane in the support fast path (2 or 4)
#endif
constexpr int kSupSamples = SPARX_SUP_SAMPLES;
static_assert(kSupSamples == 2 || kSupSamples == 4, "2 or 4 samples per lane");
constexpr int kSupSampleShift = kSupSamples == 4 ? 7 : 6;  // log2 of the sample count

template <bool kMulti, bool kHash>
__global__ void __launch_bounds__(256, 8) k_support_balanced(
    const uint32_t* __restrict__ opos, const uint32_t* __restrict__ ocol,
    const uint32_t* __restrict__ osrc, const unsigned long long* __restrict__ spref, uint32_t m,
    int2* __restrict__ es, unsigned long long* __restrict__ tri_total, uint32_t* __restrict__ err,
    const uint32_t* __restrict__ mu, uint32_t sample_min, const unsigned long long* __restrict__ hpool,
    uint32_t hash_min) {
  const uint32_t lane = lane_id();
  const unsigned long long total = spref[m];
  const unsigned long long warp = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nwarps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  unsigned long long ch = total / (nwarps * 4);
  ch = min(max((ch + 31) & ~31ull, 32ull), 4096ull);
  const PrefStart ps{spref};
  unsigned long long found_total = 0;
  for (unsigned long long c0 = warp * ch; c0 < total; c0 += nwarps * ch) {
    const unsigned long long kend = min(c0 + ch, total);
    uint32_t i = warp_last_le(PrefKey{spref}, 0, m - 1, c0);
    for (unsigned long long kb = c0; kb < kend; kb += 32) {
      const unsigned long long k = kb + lane;
      const bool valid = k < kend;
      const uint32_t e = window_find(ps, i, m, k, valid);
      const uint32_t last = (uint32_t)min(31ull, kend - 1 - kb);
      const uint32_t e_last = __shfl_sync(kFull, e, last);
      uint32_t o = 0, sb = 0, lb = 0, le = 0;
      if (valid) {
        o = (uint32_t)(k - spref[e]);
        const uint32_t a = __ldg(osrc + e), b = __ldg(ocol + e);
        const uint32_t ab = __ldg(opos + a), ae = __ldg(opos + a + 1);
        const uint32_t bb = __ldg(opos + b), be = __ldg(opos + b + 1);
        if (ae - ab <= be - bb) { sb = ab; lb = bb; le = be; }
        else { sb = bb; lb = ab; le = ae; }
      }
      uint32_t p = kInvalid;  // position of c in the longer list
      if (valid) {
        const uint32_t c = __ldg(ocol + sb + o);
        if (kHash && le - lb >= hash_min) {
          p = probe_list(hpool, lb, le - lb, c);
        } else {
          const uint32_t q = lower_bound_u32(ocol, lb, le, c);
          if (q < le && __ldg(ocol + q) == c) p = q;
        }
      }
      const bool hit = valid && p != kInvalid;
      if (kMulti) {
        if (hit) {
          const uint32_t me = __ldg(mu + e), mf = __ldg(mu + sb + o), mh = __ldg(mu + p);
          atomicAdd(&es[sb + o].x, (int)(me * mh));
          atomicAdd(&es[p].x, (int)(me * mf));
          atomicAdd(&es[e].x, (int)(mf * mh));
          found_total += (unsigned long long)me * mf * mh;
        }
      } else {
        if (hit) {
          atomicAdd(&es[sb + o].x, 1);
          atomicAdd(&es[p].x, 1);
          found_total++;
        }
        // credit e once per run of lanes sharing it
        const unsigned hits = __ballot_sync(kFull, hit);
        const unsigned grp = __match_any_sync(kFull, valid ? e : kInvalid);
        if (valid && lane == (uint32_t)(__ffs(grp) - 1)) {
          const int cnt = __popc(grp & hits);
          if (cnt) atomicAdd(&es[e].x, cnt);
        }
      }
      i = e_last;
      // fast path: while the next 32 elements all lie inside edge i, the
      // lists and the element offsets are the same for the whole warp
      const unsigned long long nb = kb + 32;
      const unsigned long long e_end = i + 1 < m ? spref[i + 1] : total;
      if (nb + 32 <= min(kend, e_end)) {
        const unsigned long long e_start = spref[i];
        const uint32_t a = __ldg(osrc + i), b = __ldg(ocol + i);
        const uint32_t ab = __ldg(opos + a), ae = __ldg(opos + a + 1);
        const uint32_t bb = __ldg(opos + b), be = __ldg(opos + b + 1);
        const bool a_short = ae - ab <= be - bb;
        const uint32_t fsb = a_short ? ab : bb, flb = a_short ? bb : ab, fle = a_short ? be : ae;
        const unsigned long long stop = min(kend, e_end);
        // a long list is narrowed first through 32 * kSupSamples evenly spaced
        // samples, kSupSamples per lane (gathered once per edge, then
        // shuffles), leaving that fraction of it to search
        const uint32_t flen = fle - flb;
        const bool hashed = kHash && flen >= hash_min;
        const bool sampled = !hashed && flen >= sample_min;
        uint32_t smp[kSupSamples];
#pragma unroll
        for (int x = 0; x < kSupSamples; ++x)
          smp[x] = sampled ? __ldg(ocol + flb + (uint32_t)(((unsigned long long)(kSupSamples * lane + x) * flen) >>
                                                          kSupSampleShift))
                           : 0u;
        do {
          kb += 32;
          const uint32_t fo = (uint32_t)(kb + lane - e_start);
          const uint32_t c = __ldg(ocol + fsb + fo);
          uint32_t lo = flb, hi = fle;
          if (hashed) {
            const uint32_t q = probe_list(hpool, flb, flen, c);
            const bool fh = q != kInvalid;
            if (kMulti) {
              if (fh) {
                const uint32_t me = __ldg(mu + i), mf = __ldg(mu + fsb + fo), mh = __ldg(mu + q);
                atomicAdd(&es[fsb + fo].x, (int)(me * mh));
                atomicAdd(&es[q].x, (int)(me * mf));
                atomicAdd(&es[i].x, (int)(mf * mh));
                found_total += (unsigned long long)me * mf * mh;
              }
            } else {
              if (fh) {
                atomicAdd(&es[fsb + fo].x, 1);
                atomicAdd(&es[q].x, 1);
                found_total++;
              }
              const int cnt = __popc(__ballot_sync(kFull, fh));
              if (lane == 0 && cnt) atomicAdd(&es[i].x, cnt);
            }
            continue;
          }
          if (sampled) {
            uint32_t t = 0;
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) {
              const uint32_t cand = __shfl_sync(kFull, smp[0], t + d);
              if (cand <= c) t += d;
            }
            // lane t's first sample is the last lane-first one <= c; its
            // other samples (ascending) decide how far past it c lies
            uint32_t kk = kSupSamples * t;
#pragma unroll
            for (int x = 1; x < kSupSamples; ++x) kk += __shfl_sync(kFull, smp[x], t) <= c ? 1u : 0u;
            lo = flb + (uint32_t)(((unsigned long long)kk * flen) >> kSupSampleShift);
            hi = kk == 32 * kSupSamples - 1
                     ? fle
                     : flb + (uint32_t)(((unsigned long long)(kk + 1) * flen) >> kSupSampleShift);
          }
          const uint32_t q = lower_bound_u32(ocol, lo, hi, c);
          const bool fh = q < hi && __ldg(ocol + q) == c;
          if (kMulti) {
            if (fh) {
              const uint32_t me = __ldg(mu + i), mf = __ldg(mu + fsb + fo), mh = __ldg(mu + q);
              atomicAdd(&es[fsb + fo].x, (int)(me * mh));
              atomicAdd(&es[q].x, (int)(me * mf));
              atomicAdd(&es[i].x, (int)(mf * mh));
              found_total += (unsigned long long)me * mf * mh;
            }
          } else {
            if (fh) {
              atomicAdd(&es[fsb + fo].x, 1);
              atomicAdd(&es[q].x, 1);
              found_total++;
            }
            const int cnt = __popc(__ballot_sync(kFull, fh));
            if (lane == 0 && cnt) atomicAdd(&es[i].x, cnt);
          }
        } while (kb + 64 <= stop);
      }
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) found_total += __shfl_down_sync(kFull, found_total, d);
  if (lane == 0 && found_total) atomicAdd(tri_total, found_total);
}

// ---------------------------------------------------------------------------
// Kernel C (vertex form).  Each triangle a < b < c (orientation rank) is found
// once, from its lowest vertex a: N+(a) is hashed into shared memory, then the
// out-lists N+(b) of every b in N+(a) are streamed with coalesced loads and
// probed against the table.  Of the three credits, (a -> b) and (a -> c) land
// in shared-memory counters for a's out-list, flushed once per vertex; only
// (b -> c) is a global atomic.  Light vertices (out-degree <= kLightMax) take
// one warp each; heavier ones one CTA each (k_support_heavy).
constexpr int kLightMax = 64;
constexpr int kLightSlots = 128;

__device__ __forceinline__ uint32_t hash_slot(uint32_t c, uint32_t shift) {
  return (c * 0x9E3779B1u) >> shift;
}

// insert key c -> j (table has >= 2x slots, so a free slot always exists)
__device__ __forceinline__ void table_insert(uint32_t* keys, uint16_t* vals, uint32_t mask, uint32_t shift,
                                             uint32_t c, uint32_t j) {
  uint32_t h = hash_slot(c, shift);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const uint32_t old = atomicCAS(keys + h, kInvalid, c);
    if (old == kInvalid) { vals[h] = (uint16_t)j; return; }
    h = (h + 1) & mask;
  }
}

__device__ __forceinline__ uint32_t table_find(const uint32_t* keys, const uint16_t* vals, uint32_t mask,
                                               uint32_t shift, uint32_t c) {
  uint32_t h = hash_slot(c, shift);
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const uint32_t k = keys[h];
    if (k == c) return vals[h];
    if (k == kInvalid) return kInvalid;
    h = (h + 1) & mask;
  }
  return kInvalid;
}

__device__ __forceinline__ uint32_t log2_pow2(uint32_t t) { return 31 - __clz(t); }

__global__ void __launch_bounds__(256) k_support_light(const uint32_t* __restrict__ opos,
                                                       const uint32_t* __restrict__ ocol, uint32_t n,
                                                       int2* __restrict__ es, unsigned long long* __restrict__ tri_total,
                                                       uint32_t* __restrict__ heavy_list,
                                                       uint32_t* __restrict__ heavy_count,
                                                       uint32_t* __restrict__ vcursor) {
  __shared__ uint32_t s_key[8][kLightSlots];
  __shared__ uint16_t s_val[8][kLightSlots];
  __shared__ uint32_t s_cnt[8][kLightMax];
  const uint32_t lane = lane_id(), wib = threadIdx.x >> 5;
  uint32_t* keys = s_key[wib];
  uint16_t* vals = s_val[wib];
  uint32_t* cnt = s_cnt[wib];
  unsigned long long tri = 0;
  for (;;) {
    uint32_t v0 = 0;
    if (lane == 0) v0 = atomicAdd(vcursor, 32u);
    v0 = __shfl_sync(kFull, v0, 0);
    if (v0 >= n) break;
    const uint32_t va = v0 + lane;
    const uint32_t dv = va < n ? __ldg(opos + va + 1) - __ldg(opos + va) : 0u;
    const bool heavy = dv > (uint32_t)kLightMax;
    const unsigned hb = __ballot_sync(kFull, heavy);
    if (hb) {
      uint32_t at = 0;
      if (lane == 0) at = atomicAdd(heavy_count, (uint32_t)__popc(hb));
      at = __shfl_sync(kFull, at, 0);
      if (heavy) heavy_list[at + __popc(hb & ((1u << lane) - 1))] = va;
    }
    unsigned todo = __ballot_sync(kFull, dv >= 2 && !heavy);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      const uint32_t a = v0 + src;
      const uint32_t da = __shfl_sync(kFull, dv, src);
      const uint32_t base = __ldg(opos + a);
      uint32_t T = 8;
      while (T < 2 * da) T <<= 1;
      const uint32_t mask = T - 1, shift = 32 - log2_pow2(T);
      for (uint32_t s = lane; s < T; s += 32) keys[s] = kInvalid;
      if (lane < da) cnt[lane] = 0;
      if (lane + 32 < da) cnt[lane + 32] = 0;
      __syncwarp();
      const uint32_t b0 = lane < da ? __ldg(ocol + base + lane) : kInvalid;
      const uint32_t b1 = lane + 32 < da ? __ldg(ocol + base + lane + 32) : kInvalid;
      if (b0 != kInvalid) table_insert(keys, vals, mask, shift, b0, lane);
      if (b1 != kInvalid) table_insert(keys, vals, mask, shift, b1, lane + 32);
      // out-lists of the b's: start and length, exclusive prefix over lengths
      const uint32_t p0 = b0 != kInvalid ? __ldg(opos + b0) : 0u;
      const uint32_t l0 = b0 != kInvalid ? __ldg(opos + b0 + 1) - p0 : 0u;
      const uint32_t p1 = b1 != kInvalid ? __ldg(opos + b1) : 0u;
      const uint32_t l1 = b1 != kInvalid ? __ldg(opos + b1 + 1) - p1 : 0u;
      const uint32_t i0 = (uint32_t)warp_incl_scan(l0), t0 = __shfl_sync(kFull, i0, 31);
      const uint32_t i1 = (uint32_t)warp_incl_scan(l1) + t0, total = __shfl_sync(kFull, i1, 31);
      // exclusive starts; entries past the list never match (start = max)
      const uint32_t x0 = lane < da ? i0 - l0 : kInvalid;
      const uint32_t x1 = lane + 32 < da ? i1 - l1 : kInvalid;
      __syncwarp();
      for (uint32_t f0 = 0; f0 < total; f0 += 32) {
        const uint32_t f = f0 + lane;
        // entry owning f: largest index with start <= f, over 64 entries
        uint32_t t = 0;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
          const uint32_t cand = __shfl_sync(kFull, x0, t + d);
          if (cand <= f) t += d;
        }
        uint32_t u = 0;
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
          const uint32_t cand = __shfl_sync(kFull, x1, u + d);
          if (cand <= f) u += d;
        }
        const uint32_t x1_0 = __shfl_sync(kFull, x1, 0);
        const uint32_t xt = __shfl_sync(kFull, x0, t), pt = __shfl_sync(kFull, p0, t);
        const uint32_t xu = __shfl_sync(kFull, x1, u), pu = __shfl_sync(kFull, p1, u);
        const bool hi = x1_0 <= f;  // entry index >= 32
        const uint32_t i = hi ? 32 + u : t;
        const uint32_t start = hi ? xu : xt, pos = hi ? pu : pt;
        bool hit = false;
        if (f < total) {
          const uint32_t at = pos + (f - start);
          const uint32_t c = __ldg(ocol + at);
          const uint32_t j = table_find(keys, vals, mask, shift, c);
          if (j != kInvalid) {
            hit = true;
            atomicAdd(cnt + j, 1u);    // a -> c
            atomicAdd(cnt + i, 1u);    // a -> b
            atomicAdd(&es[at].x, 1);   // b -> c
          }
        }
        tri += hit;
      }
      __syncwarp();
      if (lane < da && cnt[lane]) atomicAdd(&es[base + lane].x, (int)cnt[lane]);
      if (lane + 32 < da && cnt[lane + 32]) atomicAdd(&es[base + lane + 32].x, (int)cnt[lane + 32]);
      __syncwarp();
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) tri += __shfl_down_sync(kFull, tri, d);
  if (lane == 0 && tri) atomicAdd(tri_total, tri);
}

// Heavy vertices: one CTA each, table of `slots` entries in dynamic shared
// memory (slots >= 2 * max out-degree), lists of the b's staged in shared memory.
__global__ void __launch_bounds__(256) k_support_heavy(const uint32_t* __restrict__ opos,
                                                       const uint32_t* __restrict__ ocol,
                                                       int2* __restrict__ es, unsigned long long* __restrict__ tri_total,
                                                       const uint32_t* __restrict__ heavy_list,
                                                       const uint32_t* __restrict__ heavy_count,
                                                       uint32_t* __restrict__ hcursor, uint32_t slots,
                                                       uint32_t max_deg) {
  extern __shared__ __align__(16) unsigned char smem[];
  uint32_t* keys = (uint32_t*)smem;                       // slots
  uint32_t* cnt = keys + slots;                           // max_deg
  uint32_t* pre = cnt + max_deg;                          // max_deg + 1 exclusive starts
  uint32_t* bpos = pre + max_deg + 1;                     // max_deg list starts
  uint16_t* vals = (uint16_t*)(bpos + max_deg);           // slots
  __shared__ uint32_t s_a, s_sum[32];
  const uint32_t lane = lane_id(), wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t nheavy = *heavy_count;
  unsigned long long tri = 0;
  for (;;) {
    if (threadIdx.x == 0) {
      const uint32_t h = atomicAdd(hcursor, 1u);
      s_a = h < nheavy ? heavy_list[h] : kInvalid;
    }
    __syncthreads();
    const uint32_t a = s_a;
    if (a == kInvalid) break;
    const uint32_t base = __ldg(opos + a), d = __ldg(opos + a + 1) - base;
    uint32_t T = 8;
    while (T < 2 * d) T <<= 1;
    const uint32_t mask = T - 1, shift = 32 - log2_pow2(T);
    for (uint32_t s = threadIdx.x; s < T; s += blockDim.x) keys[s] = kInvalid;
    for (uint32_t i = threadIdx.x; i < d; i += blockDim.x) cnt[i] = 0;
    __syncthreads();
    // insert N+(a), record the b lists, exclusive prefix of their lengths
    uint32_t carry = 0;
    for (uint32_t i0 = 0; i0 < d; i0 += blockDim.x) {
      const uint32_t i = i0 + threadIdx.x;
      uint32_t len = 0;
      if (i < d) {
        const uint32_t b = __ldg(ocol + base + i);
        table_insert(keys, vals, mask, shift, b, i);
        const uint32_t pb = __ldg(opos + b);
        len = __ldg(opos + b + 1) - pb;
        bpos[i] = pb;
      }
      uint32_t total;
      const uint32_t ex = block_exclusive_scan<uint32_t>(len, s_sum, total);
      if (i < d) pre[i] = carry + ex;
      carry += total;
    }
    if (threadIdx.x == 0) pre[d] = carry;
    __syncthreads();
    const uint32_t total = carry;
    for (uint32_t f0 = wid * 32; f0 < total; f0 += nw * 32) {
      const uint32_t f = f0 + lane;
      if (f < total) {
        // entry owning f: largest i with pre[i] <= f (entries with no out-list
        // share their start with the next entry and are skipped)
        uint32_t lo = 0, hi = d - 1;
        while (lo < hi) {
          const uint32_t mid = (lo + hi + 1) >> 1;
          if (pre[mid] <= f) lo = mid; else hi = mid - 1;
        }
        const uint32_t at = bpos[lo] + (f - pre[lo]);
        const uint32_t c = __ldg(ocol + at);
        const uint32_t j = table_find(keys, vals, mask, shift, c);
        if (j != kInvalid) {
          atomicAdd(cnt + j, 1u);
          atomicAdd(cnt + lo, 1u);
          atomicAdd(&es[at].x, 1);
          ++tri;
        }
      }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < d; i += blockDim.x)
      if (cnt[i]) atomicAdd(&es[base + i].x, (int)cnt[i]);
    __syncthreads();
  }
#pragma unroll
  for (int dd = 16; dd > 0; dd >>= 1) tri += __shfl_down_sync(kFull, tri, dd);
  if (lane == 0 && tri) atomicAdd(tri_total, tri);
}

// dynamic shared memory of k_support_heavy for a given max out-degree
__host__ __device__ inline size_t heavy_smem_bytes(uint32_t slots, uint32_t max_deg) {
  return (size_t)slots * 4 + (size_t)max_deg * 4 * 3 + 4 + (size_t)slots * 2;
}

// ---------------------------------------------------------------------------
// Peel setup: u8 wrap (u8 mode), per-member triangle sums and max support,
// tags cleared, identity active lists (local ids inside each member's segment).
// Per-lane running sums are flushed when the member changes, then reduced per
// warp, so a single member costs one atomic per warp.
__device__ __forceinline__ void flush_member_stats(uint32_t g, unsigned long long sum, uint32_t mx,
                                                   unsigned long long* mem_tri, uint32_t* mem_maxsup) {
  if (g == kInvalid) return;
  if (sum) atomicAdd(mem_tri + g, sum);
  if (mx) atomicMax(mem_maxsup + g, mx);
}

// Multigraphs (mu != nullptr): a pair's support is per copy, so its triangle
// credits are support * mu; a support that wrapped past 2^31 is a capacity error.
// Edges [e_begin, m): all of them, or those of members that join a served union.
__global__ void __launch_bounds__(256) k_peel_setup(const Union* __restrict__ Up, const Member* __restrict__ mem,
                                                    int u8mode, unsigned long long* __restrict__ mem_tri,
                                                    uint32_t* __restrict__ mem_maxsup,
                                                    const uint32_t* __restrict__ mu, uint32_t* __restrict__ err,
                                                    uint32_t e_begin = 0) {
  const Union U = *Up;
  const uint32_t G = U.G;
  uint32_t cur = kInvalid;
  unsigned long long sum = 0;
  uint32_t mx = 0;
  for (uint32_t e = e_begin + blockIdx.x * blockDim.x + threadIdx.x; e < U.m; e += gridDim.x * blockDim.x) {
    uint32_t g = 0;
    if (G > 1) {
      uint32_t lo = 0, hi = G - 1;
      while (lo < hi) {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (mem[mid].eb <= e) lo = mid; else hi = mid - 1;
      }
      g = lo;
    }
    if (g != cur) {
      flush_member_stats(cur, sum, mx, mem_tri, mem_maxsup);
      cur = g; sum = 0; mx = 0;
    }
    int32_t s = U.es[e].x;
    if (mu) {
      if (s < 0) atomicOr(err, kErrCapacity);
      sum += (unsigned long long)(uint32_t)s * __ldg(mu + e);
    } else {
      sum += (unsigned long long)s;
    }
    if (u8mode) s &= 0xFF;
    U.es[e] = make_int2(s, (int)kTagActive);
    mx = max(mx, (uint32_t)s);
    U.act[0][e] = e - mem[g].eb;
  }
  // warp reduction when every lane ends on the same member
  const unsigned same = __match_any_sync(kFull, cur);
  if (same == kFull) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      sum += __shfl_down_sync(kFull, sum, d);
      mx = max(mx, __shfl_down_sync(kFull, mx, d));
    }
    if (lane_id() == 0) flush_member_stats(cur, sum, mx, mem_tri, mem_maxsup);
  } else {
    flush_member_stats(cur, sum, mx, mem_tri, mem_maxsup);
  }
}

// first wave: every member scans all its edges at level 0
__global__ void k_peel_init(const Member* __restrict__ mem, MemberState* __restrict__ st, Control* ctl,
                            unsigned long long* __restrict__ wpref, uint32_t G) {
  // single block: prefix of m_g
  __shared__ unsigned long long sw[32];
  unsigned long long carry = 0;
  for (uint32_t b = 0; b < G; b += blockDim.x) {
    const uint32_t g = b + threadIdx.x;
    unsigned long long w = 0;
    if (g < G) {
      MemberState s{};
      s.phase = mem[g].m ? kPhaseScan0 : kPhaseDone;
      s.act_count = mem[g].m;
      s.min_kept = 0xFFFFFFFFu;
      st[g] = s;
      w = s.phase == kPhaseDone ? 0 : mem[g].m;
    }
    unsigned long long total;
    unsigned long long ex = block_exclusive_scan<unsigned long long>(w, sw, total);
    if (g < G) wpref[g] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) {
    wpref[G] = carry;
    ctl->total_work = carry;
    ctl->wave = 1;
    ctl->done = carry == 0;
    ctl->waves_run = 0;
    ctl->el_scan = carry;
    ctl->t_start = globaltimer();
  }
}

struct WaveArgs {
  const Union* Up;     // working rows (replaced by compactions)
  PeelArrays arr;      // everything else the wave reads, by value
  const Member* mem;
  MemberState* st;
  Control* ctl;
  unsigned long long* wpref;
  uint32_t* err;
  cudaGraphConditionalHandle handle;  // WHILE condition of the peel graph
  int use_handle;                     // 0: waves are launched by the host
};

// Rows of frontier edge x in the working CSR: {shorter row start, its length,
// longer row begin, longer row end}, or {.., .., kHubDesc, hub map base} when
// the longer row's vertex has a hub map.  The length is the edge's work.
// *hq: the longer row's hash table {position, log2 capacity}, or {0, 0}.
__device__ __forceinline__ uint4 edge_desc(const UnionRegs& U, uint32_t x, uint2* hq) {
  const uint32_t u = __ldg(U.osrc + x), v = __ldg(U.ocol + x);
  // row bounds and both vertices' longer-row offers, all in one round of loads
  const uint32_t ub = __ldg(U.off + u), ue = __ldg(U.off + u + 1);
  const uint32_t vb = __ldg(U.off + v), ve = __ldg(U.off + v + 1);
  const unsigned long long iu = U.vinfo ? __ldg(U.vinfo + u) : 0ull, iv = U.vinfo ? __ldg(U.vinfo + v) : 0ull;
  const bool u_short = ue - ub <= ve - vb;
  const unsigned long long li = u_short ? iv : iu;
  const uint32_t lo = (uint32_t)li, hi = (uint32_t)(li >> 32);
  *hq = make_uint2(0, 0);
  if (hi & kVinfoHub)
    return u_short ? make_uint4(ub, ue - ub, kHubDesc, lo) : make_uint4(vb, ve - vb, kHubDesc, lo);
  if (hi) *hq = make_uint2(lo, hi);
  return u_short ? make_uint4(ub, ue - ub, vb, ve) : make_uint4(vb, ve - vb, ub, ue);
}

// What each vertex's row offers when it is a frontier edge's longer row: its
// hub map (kVinfoHub | the map's base), else its hash table (log2 capacity <<
// 32 | the table's position), else nothing.
__global__ void __launch_bounds__(256) k_vinfo(uint32_t n, const uint32_t* __restrict__ hub_slot,
                                               const uint32_t* __restrict__ hub_base,
                                               const uint32_t* __restrict__ off0, uint32_t hash_min,
                                               unsigned long long* __restrict__ vinfo) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    unsigned long long info = 0;
    const uint32_t hs = hub_slot ? __ldg(hub_slot + v) : kInvalid;
    if (hs != kInvalid) {
      info = ((unsigned long long)kVinfoHub << 32) | __ldg(hub_base + hs);
    } else if (hash_min) {
      const uint32_t b0 = __ldg(off0 + v), d0 = __ldg(off0 + v + 1) - b0;
      if (d0 >= hash_min) info = ((unsigned long long)hash_log2cap(d0) << 32) | (4u * b0);
    }
    vinfo[v] = info;
  }
}

// PKT sub-level rule for one triangle (e, f, h) of frontier edge e at level l,
// wave W (pkt.rs:409-479 restated on undirected edge ids):
//   f or h processed (tag < W)         -> nothing
//   both above l                        -> charge both
//   only f above l                      -> charge f unless h is in this frontier
//                                          with a smaller id than e
//   only h above l                      -> symmetric
// A charge that takes the support from above l to l or below queues the edge
// for the next sub-level; a charge that goes below l is restored to l.
//
// A charge is 1 in a simple graph.  In a multigraph (kMulti) a triangle of
// pairs stands for mu_e * mu_f * mu_h triangles of copies, and peeling e
// removes mu_e * mu_h of them from each copy of f (mu_e * mu_f from h): the
// charge is that product, applied at once.
template <bool kMulti>
__device__ __forceinline__ void pkt_rule(const UnionRegs& U, uint32_t e, uint32_t f, int2 es_f, uint32_t h,
                                         uint32_t l, uint32_t W, bool& pf, bool& ph) {
  pf = ph = false;
  const int2 es_h = U.es[h];
  const uint32_t tf = (uint32_t)es_f.y, th = (uint32_t)es_h.y;
  if (tf < W || th < W) return;
  const int32_t sf = es_f.x, sh = es_h.x;
  const int32_t L = (int32_t)l;
  bool df = false, dh = false;
  if (sf > L && sh > L) { df = true; dh = true; }
  else if (sf > L) df = (e < h) || (th != W);
  else if (sh > L) dh = (e < f) || (tf != W);
  int32_t cf = 1, ch = 1;
  if (kMulti && (df || dh)) {
    const int32_t me = (int32_t)__ldg(U.mu + e), mf = (int32_t)__ldg(U.mu + f), mh = (int32_t)__ldg(U.mu + h);
    cf = me * mh;
    ch = me * mf;
  }
  if (df) {
    int32_t prev = atomicSub(&U.es[f].x, cf);
    if (prev > L && prev - cf <= L) pf = true;
    if (prev - cf < L) atomicMax(&U.es[f].x, L);
  }
  if (dh) {
    int32_t prev = atomicSub(&U.es[h].x, ch);
    if (prev > L && prev - ch <= L) ph = true;
    if (prev - ch < L) atomicMax(&U.es[h].x, L);
  }
}

// Entry lookup for a warp iteration over consecutive work indices.  `start(x)`
// is the (non-decreasing) first work index of entry x; entry `i` owns the
// iteration's first element.  Each lane finds the largest x with
// start(x) <= j among entries i .. i+31 with a 5-step shuffle search; a lane
// whose entry lies beyond the window (only possible when entries own no work)
// falls back to a binary search in memory.
template <class StartF>
__device__ __forceinline__ uint32_t window_find(const StartF& start, uint32_t i, uint32_t count,
                                                unsigned long long j, bool valid) {
  const uint32_t lane = lane_id();
  const unsigned long long st = (i + lane < count) ? start(i + lane) : ~0ull;
  uint32_t t = 0;
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    const unsigned long long cand = __shfl_sync(kFull, st, t + d);
    if (cand <= j) t += d;
  }
  uint32_t x = i + t;
  if (valid && t == 31 && x + 1 < count && start(x + 1) <= j) {
    uint32_t lo = x + 1, hi = count - 1;
    while (lo < hi) {
      uint32_t mid = lo + ((hi - lo + 1) >> 1);
      if (start(mid) <= j) lo = mid; else hi = mid - 1;
    }
    x = lo;
  }
  return x;
}

struct QueueStart {
  const unsigned long long* q;
  __device__ __forceinline__ unsigned long long operator()(uint32_t x) const { return q[x] >> kEidBits; }
};

// Per-warp staging of frontier pushes in shared memory: edge ids are gathered
// across iterations and published with one 64-bit atomic (count and work) per
// kPushBuf entries, instead of one per iteration on a single hot counter.  The
// row descriptors of the staged edges are looked up at publication, all lanes
// at once, so those dependent loads stay off the per-iteration path.
constexpr int kPushBuf = 64;
constexpr int kWaveThreads = 256;
#ifndef SPARX_WAVE_MINB
#define SPARX_WAVE_MINB 7  // resident 256-thread blocks per SM the register budget targets
#endif
constexpr int kWaveWarps = kWaveThreads / 32;
// slots of the per-warp loop state in shared memory (k_wave)
enum : int { kCtxJb = 0, kCtxSegEnd = 1, kCtxKend = 2 };
enum : int { kCtxEb = 0, kCtxM, kCtxLevel, kCtxQsel, kCtxQcount, kCtxSegLen, kCtxG, kCtxW };
// kept active-list entries staged per warp before one atomic reserves their
// place: every kept entry of a large scan goes through one counter per member
constexpr int kKeepBuf = 256;
#ifndef SPARX_MERGE_CHUNKS
#define SPARX_MERGE_CHUNKS 2  // long-row chunks of 32 entries loaded per merge round
#endif
constexpr int kMergeChunks = SPARX_MERGE_CHUNKS;
#ifndef SPARX_STATE_AFTER_SEARCH
#define SPARX_STATE_AFTER_SEARCH 1  // read the other edges' states after the search, on hits only
#endif

struct PushStage {
  uint32_t* eid;  // this warp's kPushBuf staged edges
  uint32_t n;     // warp-uniform fill
};

// Publication of a warp's staged pushes.  Not inlined: it runs once per
// kPushBuf pushes, and as a call its temporaries (two row descriptors, hash
// descriptors, scans) stay out of the element loop's register budget.  It
// reads the union's arrays from the device-resident Union.
__device__ __noinline__ void push_flush_cold(const uint32_t* eid, uint32_t n, const Union* Up, uint32_t eb,
                                             uint32_t m, MemberState* st, uint32_t* err, uint32_t q_sel) {
  const UnionRegs U(Up);
  // the queue being built (q_sel names the one being processed)
  unsigned long long* qnext = q_sel ? U.q0 : U.q1;
  uint4* qdnext = q_sel ? U.qd0 : U.qd1;
  uint2* qhnext = q_sel ? U.qh0 : U.qh1;
  const Member M{0, 0, 0, 0, eb, m};
  const uint32_t lane = lane_id();
  const uint32_t x0 = lane < n ? eid[lane] : 0u, x1 = lane + 32 < n ? eid[lane + 32] : 0u;
  uint2 h0 = make_uint2(0, 0), h1 = make_uint2(0, 0);
  const uint4 d0 = lane < n ? edge_desc(U, x0, &h0) : make_uint4(0, 0, 0, 0);
  const uint4 d1 = lane + 32 < n ? edge_desc(U, x1, &h1) : make_uint4(0, 0, 0, 0);
  const unsigned long long p0 = warp_incl_scan(d0.y), p1 = warp_incl_scan(d1.y);
  const unsigned long long t0 = __shfl_sync(kFull, p0, 31), t1 = __shfl_sync(kFull, p1, 31);
  unsigned long long old = 0;
  if (lane == 0) {
    old = atomicAdd(&st->next, ((unsigned long long)n << kWorkBits) | (t0 + t1));
    if ((old & kWorkMask) + t0 + t1 > kWorkMask) atomicOr(err, kErrCapacity);
  }
  old = __shfl_sync(kFull, old, 0);
  const unsigned long long pos = old >> kWorkBits, ws = old & kWorkMask;
  if (lane < n) {
    if (pos + lane < M.m) {
      qnext[M.eb + pos + lane] = ((ws + p0 - d0.y) << kEidBits) | (x0 - M.eb);
      qdnext[M.eb + pos + lane] = d0;
      if (U.hash_min) qhnext[M.eb + pos + lane] = h0;
    } else {
      atomicOr(err, kErrCapacity);
    }
  }
  if (lane + 32 < n) {
    if (pos + 32 + lane < M.m) {
      qnext[M.eb + pos + 32 + lane] = ((ws + t0 + p1 - d1.y) << kEidBits) | (x1 - M.eb);
      qdnext[M.eb + pos + 32 + lane] = d1;
      if (U.hash_min) qhnext[M.eb + pos + 32 + lane] = h1;
    } else {
      atomicOr(err, kErrCapacity);
    }
  }
}

__device__ __forceinline__ void push_flush(PushStage& ps, const Union* Up, uint32_t eb, uint32_t m, MemberState* st,
                                           uint32_t* err, uint32_t q_sel) {
  __syncwarp();
  if (ps.n == 0) return;
  push_flush_cold(ps.eid, ps.n, Up, eb, m, st, err, q_sel);
  ps.n = 0;
  __syncwarp();
}

// Queue edge x (union eid) for wave W + 1.  All lanes call it.
__device__ __forceinline__ void push_edge(PushStage& ps, const UnionRegs& U, const Union* Up, uint32_t eb,
                                          uint32_t m, MemberState* st, uint32_t* err, uint32_t q_sel, bool want,
                                          uint32_t x, uint32_t W) {
  const unsigned bal = __ballot_sync(kFull, want);
  if (!bal) return;
  const uint32_t k = __popc(bal);
  if (ps.n + k > kPushBuf) push_flush(ps, Up, eb, m, st, err, q_sel);
  if (want) {
    U.es[x].y = (int)(W + 1);
    ps.eid[ps.n + __popc(bal & ((1u << lane_id()) - 1))] = x;
  }
  ps.n += k;
}

// Member state read past L1: the planner runs in the wave kernel's last
// block, whose L1 may hold lines that other blocks changed by atomics.
__device__ __forceinline__ MemberState load_state_cg(const MemberState* p) {
  static_assert(sizeof(MemberState) % 16 == 0, "MemberState is read as uint4 words");
  MemberState s;
  const uint4* src = reinterpret_cast<const uint4*>(p);
  uint4* dst = reinterpret_cast<uint4*>(&s);
#pragma unroll
  for (int i = 0; i < (int)(sizeof(MemberState) / 16); ++i) dst[i] = __ldcg(src + i);
  return s;
}

struct PlanShared {
  unsigned long long sw[32];
  uint32_t live;
  uint32_t newly_done;  // members that finished in this wave
  unsigned long long proc, scan, edges, live_edges;
};

// Planner: one block advances every member's state machine after a wave and
// lays out the next wave's work; sets the CUDA-graph loop condition.  Runs in
// the last block of each wave (see k_wave), after every other block's writes.
__device__ __forceinline__ void plan_wave(const Member* __restrict__ mem, MemberState* __restrict__ st,
                                          Control* ctl, unsigned long long* __restrict__ wpref,
                                          uint32_t* __restrict__ err, cudaGraphConditionalHandle handle,
                                          int use_handle, PlanShared& ps) {
  unsigned long long* sw = ps.sw;
  uint32_t& s_live = ps.live;
  unsigned long long &s_proc = ps.proc, &s_scan = ps.scan, &s_edges = ps.edges, &s_live_edges = ps.live_edges;
  const uint32_t G = ctl->G;
  if (threadIdx.x == 0) { s_live = 0; s_proc = 0; s_scan = 0; s_edges = 0; s_live_edges = 0; ps.newly_done = 0; }
  __syncthreads();
  const bool was_done = ctl->done;
  if (was_done) {
    // the loop is stopped (host-launched waves keep coming until the host
    // looks): the planned wave must survive untouched for a resume
    if (threadIdx.x == 0 && use_handle) cudaGraphSetConditional(handle, 0u);
    return;
  }
  unsigned long long carry = 0;
  for (uint32_t b = 0; b < G; b += blockDim.x) {
    const uint32_t g = b + threadIdx.x;
    unsigned long long w = 0;
    if (g < G && !was_done) {
      MemberState s = load_state_cg(st + g);
      const uint32_t m = mem[g].m;
      const uint32_t phase_before = s.phase;
      switch (s.phase) {
        case kPhaseScan0:
          s.act_sel ^= 1u;
          s.act_count = s.kept;
          s.kept = 0;
          if (s.processed >= m) s.phase = kPhaseDone;
          else { s.level = s.min_kept; s.min_kept = 0xFFFFFFFFu; s.phase = kPhaseScan; }
          break;
        case kPhaseScan: {
          s.act_sel ^= 1u;
          s.act_count = s.kept;
          s.kept = 0;
          const unsigned long long cnt = s.next >> kWorkBits;
          if (cnt) {
            s.curr = s.next;
            s.next = 0;
            s.q_sel ^= 1u;
            s.phase = kPhaseProc;
            s.levels++;
            s.max_level = s.level;
          } else if (s.act_count == 0) {
            s.phase = kPhaseDone;
          } else {
            s.level = s.min_kept;  // no edge at this level: jump to the next occupied one
          }
          s.min_kept = 0xFFFFFFFFu;
          break;
        }
        case kPhaseProc: {
          s.processed += (uint32_t)(s.curr >> kWorkBits);
          const unsigned long long cnt = s.next >> kWorkBits;
          if (cnt) {
            s.curr = s.next;
            s.next = 0;
            s.q_sel ^= 1u;
          } else {
            s.curr = 0;
            if (s.processed >= m) s.phase = kPhaseDone;
            else { s.level += 1; s.phase = kPhaseScan; s.min_kept = 0xFFFFFFFFu; }
          }
          break;
        }
        default:
          break;
      }
      if (s.phase != kPhaseDone) s.waves++;
      else if (phase_before != kPhaseDone) atomicAdd(&ps.newly_done, 1u);
      st[g] = s;
      if (s.phase == kPhaseScan0 || s.phase == kPhaseScan) {
        w = s.act_count;
        if (w) atomicAdd(&s_scan, w);
      } else if (s.phase == kPhaseProc) {
        w = s.curr & kWorkMask;
        atomicAdd(&s_proc, w);
        atomicAdd(&s_edges, s.curr >> kWorkBits);
      }
      if (s.phase != kPhaseDone) {
        atomicAdd(&s_live, 1u);
        atomicAdd(&s_live_edges, (unsigned long long)(m - s.processed));
      }
    }
    unsigned long long total;
    unsigned long long ex = block_exclusive_scan<unsigned long long>(w, sw, total);
    if (g < G) wpref[g] = carry + ex;
    carry += total;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    wpref[G] = carry;
    uint32_t done = was_done;
    if (!was_done) {
      if (ctl->trace && ctl->waves_run < ctl->trace_cap)
        ctl->trace[ctl->waves_run] = make_ulonglong4(globaltimer(), carry, s_proc, s_scan);
      ctl->el_proc += s_proc;
      ctl->el_scan += s_scan;
      ctl->edges_proc += s_edges;
      ctl->total_work = carry;
      ctl->wave += 1;
      ctl->waves_run += 1;
      const uint32_t e = __ldcg(err);
      uint32_t reason = kExitNone;
      if (s_live == 0) { done = 1; reason = kExitDone; }
      if (e) { done = 1; reason = kExitError; }
      if (ctl->waves_run > ctl->max_waves) { atomicOr(err, kErrWaves); done = 1; reason = kExitError; }
      if (globaltimer() - ctl->t_start > ctl->timeout_ns) { atomicOr(err, kErrTimeout); done = 1; reason = kExitError; }
      // live edges fill at most compact_pct % of the working rows (85 unless
      // tuned): stop so the host can compact them (a compaction is a few passes
      // over the rows, which the shorter rows repay at this fill; 78% and 90%
      // measured slower on R-MAT-22)
      if (!done && ctl->csr_slots >= ctl->compact_min &&
          200 * s_live_edges <= (unsigned long long)ctl->compact_pct * ctl->csr_slots) {
        done = 1;
        reason = kExitCompact;
      }
      if (!done && ctl->notify_done && ps.newly_done) { done = 1; reason = kExitMember; }
      if (!done && ctl->admit && *ctl->admit) { done = 1; reason = kExitAdmit; }
      ctl->done = done;
      ctl->exit_reason = reason;
    }
    if (use_handle) cudaGraphSetConditional(handle, done ? 0u : 1u);
  }
}

// One member's segment of a level scan (kPhaseScan0 / kPhaseScan): active
// entry j of the segment is kept (support above the level), queued for this
// level, or dropped (processed).  Not inlined: its staging state stays out of
// the frontier loop's register budget.  Publishes its pushes before returning.
__device__ __noinline__ void wave_scan_segment(const Union* Up, MemberState* st, uint32_t eb, uint32_t m,
                                               uint32_t phase, uint32_t level, uint32_t act_sel, uint32_t q_sel,
                                               uint32_t W, uint32_t a0, uint32_t seg_len, uint32_t* keepbuf,
                                               uint32_t* push_eid, uint32_t* err) {
  const UnionRegs U(Up);
  const uint32_t lane = lane_id();
  PushStage ps{push_eid, 0};
  const uint32_t* act = act_sel ? U.act1 : U.act0;
  uint32_t* act_out = act_sel ? U.act0 : U.act1;
  uint32_t nkeep = 0, nzero = 0, mn = 0xFFFFFFFFu;
  for (uint32_t r = 0; r < seg_len; r += 32) {
    const bool valid = r + lane < seg_len;
    bool keep = false, zero = false, queue = false;
    uint32_t le = 0, e = 0;
    if (valid) {
      le = act[eb + a0 + r + lane];
      e = eb + le;
      const int2 st_e = U.es[e];
      const int32_t s = st_e.x;
      if (phase == kPhaseScan0) {
        if (s == 0) { U.es[e].y = 0; zero = true; }
        else { keep = true; mn = min(mn, (uint32_t)s); }
      } else if ((uint32_t)st_e.y == kTagActive) {  // processed edges leave the active list
        if (s <= (int32_t)level) queue = true;
        else { keep = true; mn = min(mn, (uint32_t)s); }
      }
    }
    push_edge(ps, U, Up, eb, m, st, err, q_sel, queue, e, W);
    const unsigned kb_bal = __ballot_sync(kFull, keep);
    if (kb_bal) {
      const uint32_t kc = __popc(kb_bal);
      if (nkeep + kc > kKeepBuf) {
        __syncwarp();
        uint32_t old = 0;
        if (lane == 0) old = atomicAdd(&st->kept, nkeep);
        old = __shfl_sync(kFull, old, 0);
        for (uint32_t t = lane; t < nkeep; t += 32) act_out[eb + old + t] = keepbuf[t];
        nkeep = 0;
        __syncwarp();
      }
      if (keep) keepbuf[nkeep + __popc(kb_bal & ((1u << lane) - 1))] = le;
      nkeep += kc;
    }
    nzero += __popc(__ballot_sync(kFull, zero));
  }
  __syncwarp();
  if (nkeep) {
    uint32_t old = 0;
    if (lane == 0) old = atomicAdd(&st->kept, nkeep);
    old = __shfl_sync(kFull, old, 0);
    for (uint32_t t = lane; t < nkeep; t += 32) act_out[eb + old + t] = keepbuf[t];
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) mn = min(mn, __shfl_xor_sync(kFull, mn, d));
  if (lane == 0) {
    if (mn != 0xFFFFFFFFu) atomicMin(&st->min_kept, mn);
    if (nzero) atomicAdd(&st->processed, nzero);
  }
  __syncwarp();
  push_flush(ps, Up, eb, m, st, err, q_sel);
}

// Kernel D: one peel wave.  The wave's work (all members' scan elements and
// frontier elements, laid out by `wpref`) is cut into warp-sized chunks; a
// warp walks its chunk member by member, 32 consecutive elements per
// iteration, so every iteration belongs to one member.
//   scan element j      active-list entry j: processed -> dropped; support
//                       <= level -> queued for this level; else kept
//   frontier element j  element o of the shorter working row of frontier
//                       edge e, searched in the longer row; a hit is a triangle
template <bool kMulti>
__global__ void __launch_bounds__(kWaveThreads, SPARX_WAVE_MINB) k_wave(WaveArgs a) {
  __shared__ uint32_t s_push_eid[kWaveWarps][kPushBuf];
  __shared__ uint32_t s_keep[kWaveWarps][kKeepBuf];
  const Control* ctl = a.ctl;
  // a stopped loop (host-launched waves run on until the host looks) does no
  // work, but its blocks still hand over to the planner
  const unsigned long long total = ctl->done ? 0ull : ctl->total_work;
  const uint32_t W = ctl->wave;
  const uint32_t G = ctl->G;
  const uint32_t lane = lane_id();
  const uint32_t wib = threadIdx.x >> 5;
  const unsigned long long warp = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nwarps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  const UnionRegs U(a.Up, a.arr);
  const bool hubs = U.hub_map != nullptr;  // descriptors carry kHubDesc only when maps exist
  // one chunk per warp: finer chunks (and any cap on their size) measured
  // slower, the search for a chunk's first entry is paid once per warp;
  // ch * nwarps >= total, so the chunk below is the warp's only one
  const unsigned long long ch = max(((total + nwarps - 1) / nwarps + 31) & ~31ull, 32ull);
  // work counters live in shared memory (per warp: hits, merge iterations,
  // lane iterations, merge chunks) rather than in four registers held across
  // the loop; lane 0 adds to them
  __shared__ uint32_t s_cnt[4][kWaveWarps];
  if (lane < 4) s_cnt[lane][wib] = 0;
  __syncwarp();
  PushStage ps{s_push_eid[wib], 0};
  // Warp-uniform state of the frontier loop lives in shared memory and is read
  // back where it is used: held in registers it was spilled to local memory,
  // whose lines the loop's random row and state loads evict from L1.
  __shared__ unsigned long long s_w64[kWaveWarps][3];  // kCtxJb, kCtxSegEnd, kCtxKend
  __shared__ uint32_t s_w32[kWaveWarps][8];            // kCtxEb .. kCtxW
  volatile unsigned long long* const w64 = s_w64[wib];
  volatile uint32_t* const w32 = s_w32[wib];

  if (warp * ch < total) {
    const unsigned long long c0 = warp * ch;
    if (lane == 0) w64[kCtxKend] = min(c0 + ch, total);
    __syncwarp();
    unsigned long long k = c0;
    uint32_t g = G > 1 ? warp_last_le(PrefKey{a.wpref}, 0, G - 1, k) : 0;
    while (k < w64[kCtxKend]) {
      const unsigned long long kend = w64[kCtxKend];
      while (g + 1 < G && a.wpref[g + 1] <= k) ++g;
      const unsigned long long mbeg = a.wpref[g];
      // a segment spans < 2^31 elements, so offsets inside it are 32-bit
      const unsigned long long seg_end = min(min(kend, a.wpref[g + 1]), k + (1ull << 31));
      if (seg_end <= k || mbeg > k) {  // layout does not cover k: stop rather than spin
        if (lane == 0) atomicOr(a.err, kErrInternal);
        break;
      }
      const Member M = a.mem[g];
      MemberState* st = a.st + g;
      const uint32_t phase = st->phase, level = st->level, act_sel = st->act_sel, q_sel = st->q_sel;
      if (phase == kPhaseProc) {
        const uint32_t qcount0 = (uint32_t)(st->curr >> kWorkBits);
        if (qcount0 == 0) {
          if (lane == 0) atomicOr(a.err, kErrInternal);
          k = seg_end;
          continue;
        }
        const uint32_t i0 =
            warp_last_le(QueueStart{(q_sel ? U.q1 : U.q0) + M.eb}, 0, qcount0 - 1, k - mbeg);
        __syncwarp();
        if (lane == 0) {
          // element j (member-relative) = jb + r + lane; r counts the segment
          w64[kCtxJb] = k - mbeg;
          w64[kCtxSegEnd] = seg_end;
          w32[kCtxEb] = M.eb;
          w32[kCtxM] = M.m;
          w32[kCtxLevel] = level;
          w32[kCtxQsel] = q_sel;
          w32[kCtxQcount] = qcount0;
          w32[kCtxSegLen] = (uint32_t)(seg_end - k);
          w32[kCtxG] = g;
          w32[kCtxW] = W;
        }
        __syncwarp();
        uint32_t i = i0;
        // merge cursor carried across iterations that continue the same edge
        uint32_t m_e = kInvalid, m_next_o = 0, m_cur = 0;
        for (uint32_t r = 0; r < w32[kCtxSegLen]; r += 32) {
          const uint32_t seg_len = w32[kCtxSegLen];
          const uint32_t qcount = w32[kCtxQcount];
          const unsigned long long* q = (w32[kCtxQsel] ? U.q1 : U.q0) + w32[kCtxEb];
          const bool valid = r + lane < seg_len;
          // the window's entries, loaded once: each lane picks its own by a
          // shuffle search on the work starts (entries own >= 1 element, so
          // 32 consecutive elements span at most 32 entries).  The search runs
          // on 32-bit distances from the iteration's first element jr: the
          // window's first entry owns element jr - 1 or jr and an entry's work
          // is below 2^31, so every distance lies in (-2^31, 2^31); entries
          // past the queue's end clamp to the most negative.  Lane l's
          // element jr + l lies in entry x iff jr - start(x) >= -l.
          const unsigned long long jr = w64[kCtxJb] + r;
          const unsigned long long qv = (i + lane < qcount) ? q[i + lane] : ~0ull;
          const int32_t dq = (int32_t)max((long long)(jr - (qv >> kEidBits)), (long long)INT32_MIN);
          uint32_t t = 0;
#pragma unroll
          for (int d = 16; d > 0; d >>= 1) {
            const int32_t cand = __shfl_sync(kFull, dq, t + d);
            if (cand >= -(int32_t)lane) t += d;
          }
          const int32_t dt = __shfl_sync(kFull, dq, t);
          const uint32_t eid_t = __shfl_sync(kFull, (uint32_t)qv & kEidMask, t);
          const uint32_t x = i + t;
          const uint32_t last = min(31u, seg_len - 1 - r);
          const uint32_t x_last = __shfl_sync(kFull, x, last);
          uint32_t e = 0, o = 0, sb = 0, slen = 0, lb = 0, le = 0;
          if (valid) {
            e = w32[kCtxEb] + eid_t;
            o = (uint32_t)(dt + (int32_t)lane);
            const uint4 dsc = ((w32[kCtxQsel] ? U.qd1 : U.qd0) + w32[kCtxEb])[x];
            sb = dsc.x;
            slen = dsc.y;
            lb = dsc.z;
            le = dsc.w;
          }
          // rows may have been compacted since the entry's work was counted
          const bool el = valid && o < slen;
          unsigned long long pr = el ? __ldg(U.row + sb + o) : 0ull;
          const uint32_t w = (uint32_t)pr;
          uint32_t f = (uint32_t)(pr >> 32), h = kInvalid, p = kInvalid;
          // f == kInvalid: a self-loop entry; f == e: the frontier edge itself
          bool look = el && f != kInvalid && f != e;
          int2 es_f = make_int2(0, 0);
#if !SPARX_STATE_AFTER_SEARCH
          // the other edge of the short row: already processed -> nothing to resolve
          if (look) {
            es_f = U.es[f];
            look = (uint32_t)es_f.y >= w32[kCtxW];
          }
#endif
          // lane 0 is always valid: its rows decide, so the branch and the
          // merge below are warp-uniform
          const uint32_t e0 = __shfl_sync(kFull, e, 0);
          const uint32_t L_beg = __shfl_sync(kFull, lb, 0), L_end = __shfl_sync(kFull, le, 0);
          const uint32_t s_len0 = __shfl_sync(kFull, slen, 0);
          const bool one_edge = __all_sync(kFull, !valid || e == e0);
          const bool hub0 = hubs && (L_beg & kHubDesc);
          if (one_edge && !hub0 && (L_end - L_beg) <= a.arr.merge_ratio * s_len0) {
            // similar row lengths: walk the longer row with a warp-wide cursor;
            // every chunk of 32 entries is matched against the 32 sorted
            // elements by a shuffle search
            const unsigned elb = __ballot_sync(kFull, el);
            if (elb) {
              const uint32_t o0 = __shfl_sync(kFull, o, 0);
              const uint32_t wmax = __shfl_sync(kFull, w, 31 - __clz(elb));
              uint32_t cur;
              if (m_e == e0 && m_next_o == o0) {
                cur = m_cur;
              } else {
                const uint32_t wmin = __shfl_sync(kFull, w, __ffs(elb) - 1);
                cur = warp_lower_bound(RowIdKey{U.row}, L_beg, L_end, wmin);
              }
              // kMergeChunks chunks are loaded per round, so most rows cost
              // one dependent load instead of one per chunk
              const uint32_t cap = (L_end - L_beg) / 32 + 2;
              uint32_t nch = 0;  // chunks matched (work counter)
              for (uint32_t it = 0;; ++it) {
                if (it > cap) {
                  if (lane == 0) atomicOr(a.err, kErrInternal);
                  break;
                }
                unsigned long long lp[kMergeChunks];
#pragma unroll
                for (int c = 0; c < kMergeChunks; ++c) {
                  const uint32_t idx = cur + 32 * c + lane;
                  lp[c] = idx < L_end ? __ldg(U.row + idx) : ~0ull;
                }
                uint32_t adv = 0;
#pragma unroll
                for (int c = 0; c < kMergeChunks; ++c) {
                  if (c > 0 && adv < 32u * c) break;  // the row passed wmax in an earlier chunk
                  const uint32_t lv = (uint32_t)lp[c];
                  uint32_t tt = 0;
#pragma unroll
                  for (int d = 16; d > 0; d >>= 1) {
                    const uint32_t cv = __shfl_sync(kFull, lv, tt + d);
                    if (cv <= w) tt += d;
                  }
                  const uint32_t lvt = __shfl_sync(kFull, lv, tt);
                  const uint32_t ht = (uint32_t)(__shfl_sync(kFull, lp[c], tt) >> 32);
                  if (look && lvt == w) { p = cur + 32 * c + tt; h = ht; }
                  adv += __popc(__ballot_sync(kFull, lv <= wmax));
                  ++nch;
                }
                cur += adv;
                if (adv < 32u * kMergeChunks) break;
              }
              if (lane == 0) s_cnt[3][wib] += nch;
              m_e = e0;
              m_next_o = o0 + 32;
              m_cur = cur;
            }
            if (lane == 0) s_cnt[1][wib]++;
          } else {
            if (lane == 0) s_cnt[2][wib]++;
            m_e = kInvalid;
            if (look) {
              const uint2 hq = U.hash_min ? (w32[kCtxQsel] ? U.qh1 : U.qh0)[w32[kCtxEb] + x] : make_uint2(0, 0);
              if (hubs && (lb & kHubDesc)) {
                // the longer row's vertex has a hub map: one lookup
                h = __ldg(U.hub_map + (uint32_t)(le + w));
                p = h != kInvalid ? 0u : kInvalid;
              } else if (hq.y) {
                // the longer row has a hash table: probe from the id's hash
                const unsigned long long* tb = U.hpool + hq.x;
                const uint32_t mask = (1u << hq.y) - 1;
                uint32_t at = hash_first(w, hq.y);
#pragma unroll 1
                for (uint32_t it = 0; it <= mask; ++it) {
                  const unsigned long long en = __ldg(tb + at);
                  const uint32_t id = (uint32_t)en;
                  if (id == w) { h = (uint32_t)(en >> 32); p = 0; break; }
                  if (id == kInvalid) break;
                  at = (at + 1) & mask;
                }
              } else {
                p = find_in_row(U.row, lb, le, w);
                if (p != kInvalid) h = (uint32_t)(__ldg(U.row + p) >> 32);
              }
            }
          }
          bool pf = false, ph = false;
          // h == kInvalid: w was the long row's own vertex (a self-loop entry)
          const bool hit = look && p != kInvalid && h != kInvalid;
          const uint32_t nhit = __popc(__ballot_sync(kFull, hit));
          if (lane == 0) s_cnt[0][wib] += nhit;
#if SPARX_STATE_AFTER_SEARCH
          // both other edges' states are read only for a found triangle (a
          // quarter of the elements on R-MAT); the search may run for an f
          // that is already processed, which pkt_rule then skips
          if (hit) es_f = U.es[f];
#endif
          if (hit) pkt_rule<kMulti>(U, e, f, es_f, h, w32[kCtxLevel], w32[kCtxW], pf, ph);
          push_edge(ps, U, a.Up, w32[kCtxEb], w32[kCtxM], a.st + w32[kCtxG], a.err, w32[kCtxQsel], pf, f,
                    w32[kCtxW]);
          push_edge(ps, U, a.Up, w32[kCtxEb], w32[kCtxM], a.st + w32[kCtxG], a.err, w32[kCtxQsel], ph, h,
                    w32[kCtxW]);
          i = x_last;
        }
        // entries belong to this member: publish before moving on
        push_flush(ps, a.Up, w32[kCtxEb], w32[kCtxM], a.st + w32[kCtxG], a.err, w32[kCtxQsel]);
        k = w64[kCtxSegEnd];
        g = w32[kCtxG];
        continue;
      } else if (phase == kPhaseScan0 || phase == kPhaseScan) {
        // active-list positions are below the member's edge count (< 2^28)
        wave_scan_segment(a.Up, st, M.eb, M.m, phase, level, act_sel, q_sel, W, (uint32_t)(k - mbeg),
                          (uint32_t)(seg_end - k), s_keep[wib], ps.eid, a.err);
      }
      push_flush(ps, a.Up, M.eb, M.m, st, a.err, q_sel);  // entries belong to this member: publish before moving on
      k = seg_end;
    }
  }
  // work counters: summed per block, then one atomic per counter and block
  // (per-warp atomics on four addresses serialise on large waves)
  __syncthreads();
  if (threadIdx.x < 4) {
    unsigned long long sum = 0;
#pragma unroll
    for (int w = 0; w < kWaveWarps; ++w) sum += s_cnt[threadIdx.x][w];
    unsigned long long* dst = threadIdx.x == 0 ? &a.ctl->hits
                              : threadIdx.x == 1 ? &a.ctl->merge_iters
                              : threadIdx.x == 2 ? &a.ctl->lane_iters
                                                 : &a.ctl->merge_chunks;
    if (sum) atomicAdd(dst, sum);
  }
  // the last block to finish plans the next wave (threadfence-reduction
  // pattern: every thread fences its writes, the block takes a ticket; the
  // block holding the last ticket sees every other block's writes)
  __shared__ uint32_t s_last;
  __shared__ PlanShared s_plan;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&a.ctl->blocks_done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (s_last) {
    __threadfence();
    plan_wave(a.mem, a.st, a.ctl, a.wpref, a.err, a.handle, a.use_handle, s_plan);
    if (threadIdx.x == 0) a.ctl->blocks_done = 0;
  }
}

// Hub maps: the vertices of highest degree (at least `min_deg`, at most the
// reserved number of maps) get a dense map from neighbour id to edge id, so a
// frontier element whose longer row is a hub's resolves its triangle with one
// load instead of a search of the long row.  A hub's map covers its own
// member's vertex range only, so maps are as small as their graph, and unions
// of many graphs get maps for the hubs of each.
//   k_hub_hist    vertices and slots per floor(log2(degree)) (also the
//                 degree signature the tuning is keyed on)
//   k_hub_assign  hub index per vertex (kInvalid below the chosen degree)
//   k_hub_layout  each hub's map base in the pool (a prefix over its member's
//                 vertex count); hubs past the pool lose their map
//   k_hub_fill    scatter each hub's row into its map (block per hub)
__global__ void __launch_bounds__(256) k_hub_hist(const uint32_t* __restrict__ off, uint32_t n,
                                                  uint32_t* __restrict__ hist,
                                                  unsigned long long* __restrict__ hist_slots) {
  __shared__ uint32_t sh[33];
  __shared__ unsigned long long sl[33];
  if (threadIdx.x < 33) { sh[threadIdx.x] = 0; sl[threadIdx.x] = 0; }
  __syncthreads();
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    const uint32_t d = __ldg(off + u + 1) - __ldg(off + u);
    if (d) {
      atomicAdd(&sh[32 - __clz(d)], 1u);
      atomicAdd(&sl[32 - __clz(d)], (unsigned long long)d);
    }
  }
  __syncthreads();
  if (threadIdx.x < 33 && sh[threadIdx.x]) {
    atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
    atomicAdd(&hist_slots[threadIdx.x], sl[threadIdx.x]);
  }
}

__global__ void __launch_bounds__(256) k_hub_assign(const uint32_t* __restrict__ off, uint32_t n,
                                                    uint32_t min_deg, uint32_t max_hubs,
                                                    uint32_t* __restrict__ hub_slot,
                                                    uint32_t* __restrict__ hub_vertex,
                                                    uint32_t* __restrict__ hub_count) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    const uint32_t d = __ldg(off + u + 1) - __ldg(off + u);
    uint32_t slot = kInvalid;
    if (d >= min_deg) {
      slot = atomicAdd(hub_count, 1u);
      if (slot < max_hubs) hub_vertex[slot] = u;
      else slot = kInvalid;  // cannot happen: the host sized max_hubs from the histogram
    }
    hub_slot[u] = slot;
  }
}

// One block: base of each hub's map = exclusive prefix of its member's vertex
// count, minus the member's first vertex; a hub whose map would end past
// `pool` entries gets none (hub_slot back to kInvalid).
__global__ void __launch_bounds__(1024) k_hub_layout(const uint32_t* __restrict__ hub_vertex, uint32_t hubs,
                                                     const Member* __restrict__ mem, uint32_t G,
                                                     unsigned long long pool, uint32_t* __restrict__ hub_base,
                                                     uint32_t* __restrict__ hub_slot) {
  __shared__ unsigned long long sw[32];
  unsigned long long carry = 0;
  for (uint32_t b = 0; b < hubs; b += blockDim.x) {
    const uint32_t k = b + threadIdx.x;
    unsigned long long size = 0;
    uint32_t u = 0, vb = 0;
    if (k < hubs) {
      u = hub_vertex[k];
      uint32_t lo = 0, hi = G - 1;
      while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (mem[mid].vb <= u) lo = mid; else hi = mid - 1;
      }
      vb = mem[lo].vb;
      size = mem[lo].n;
    }
    unsigned long long total;
    const unsigned long long at = carry + block_exclusive_scan<unsigned long long>(size, sw, total);
    if (k < hubs) {
      if (at + size <= pool) hub_base[k] = (uint32_t)at - vb;
      else hub_slot[u] = kInvalid;
    }
    carry += total;
  }
}

__global__ void __launch_bounds__(256) k_hub_fill(const uint32_t* __restrict__ off,
                                                  const unsigned long long* __restrict__ row0,
                                                  const uint32_t* __restrict__ hub_vertex, uint32_t hubs,
                                                  const uint32_t* __restrict__ hub_slot,
                                                  const uint32_t* __restrict__ hub_base,
                                                  uint32_t* __restrict__ hub_map) {
  for (uint32_t k = blockIdx.x; k < hubs; k += gridDim.x) {
    const uint32_t u = hub_vertex[k];
    if (__ldg(hub_slot + u) != k) continue;  // no room in the pool
    const uint32_t b = __ldg(off + u), e = __ldg(off + u + 1), base = __ldg(hub_base + k);
    for (uint32_t s = b + threadIdx.x; s < e; s += blockDim.x) {
      const unsigned long long pr = __ldg(row0 + s);
      const uint32_t id = (uint32_t)pr, eid = (uint32_t)(pr >> 32);
      if (eid != kInvalid) hub_map[(uint32_t)(base + id)] = eid;
    }
  }
}

// Working-row compaction (between waves): keep the entries whose edge is not
// processed (tag >= the next wave).  The edges' states are first condensed
// into a bitmap (one bit per edge, small enough to stay in L2), so the row
// passes look up a bit instead of a random 8-byte state.  Mark, count, scan
// (host), fill; 32 vertices per warp for the row passes.
__global__ void __launch_bounds__(256) k_compact_mark(const int2* __restrict__ es, uint32_t m,
                                                      const Control* ctl, uint32_t* __restrict__ alive) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  const uint32_t W = ctl->wave;
  const uint32_t words = (m + 31) / 32;
  for (uint32_t i = warp; i < words; i += nwarps) {
    const uint32_t x = i * 32 + lane;
    const bool live = x < m && (uint32_t)__ldg(&es[x].y) >= W;
    const uint32_t bits = __ballot_sync(kFull, live);
    if (lane == 0) alive[i] = bits;
  }
}

__device__ __forceinline__ bool is_alive(const uint32_t* __restrict__ alive, uint32_t x) {
  return x != kInvalid && ((__ldg(alive + (x >> 5)) >> (x & 31)) & 1u);
}

__global__ void __launch_bounds__(256) k_compact_count(const uint32_t* __restrict__ off,
                                                       const unsigned long long* __restrict__ row, uint32_t n,
                                                       const uint32_t* __restrict__ alive,
                                                       uint32_t* __restrict__ cnt,
                                                       const uint32_t* __restrict__ off0) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t base = warp * 32; base < n; base += nwarps * 32) {
    const uint32_t u = base + lane;
    uint32_t b = 0, e = 0;
    if (u < n) { b = __ldg(off + u); e = __ldg(off + u + 1); }
    uint32_t c = 0;
    if (u < n && e - b <= kLaneRow)
      for (uint32_t s = b; s < e; ++s) c += is_alive(alive, (uint32_t)(__ldg(row + s) >> 32));
    const bool blk = u < n && e - b > kLaneRow && big_row(off0, u);
    unsigned big = __ballot_sync(kFull, u < n && e - b > kLaneRow && !blk);
    while (big) {
      const int j = __ffs(big) - 1;
      big &= big - 1;
      const uint32_t bb = __shfl_sync(kFull, b, j), be = __shfl_sync(kFull, e, j);
      uint32_t cc = 0;
      for (uint32_t s = bb + lane; s < be; s += 32) cc += is_alive(alive, (uint32_t)(__ldg(row + s) >> 32));
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) cc += __shfl_xor_sync(kFull, cc, d);
      if (lane == (uint32_t)j) c = cc;
    }
    if (u < n && !blk) cnt[u] = c;
  }
}

__global__ void __launch_bounds__(256) k_compact_fill(const uint32_t* __restrict__ off,
                                                      const unsigned long long* __restrict__ row, uint32_t n,
                                                      const uint32_t* __restrict__ alive,
                                                      const uint32_t* __restrict__ off2,
                                                      unsigned long long* __restrict__ row2,
                                                      const uint32_t* __restrict__ off0) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t base = warp * 32; base < n; base += nwarps * 32) {
    const uint32_t u = base + lane;
    uint32_t b = 0, e = 0;
    if (u < n) { b = __ldg(off + u); e = __ldg(off + u + 1); }
    if (u < n && e - b <= kLaneRow) {
      uint32_t at = __ldg(off2 + u);
      for (uint32_t s = b; s < e; ++s) {
        const unsigned long long pr = __ldg(row + s);
        if (is_alive(alive, (uint32_t)(pr >> 32))) row2[at++] = pr;
      }
    }
    unsigned big = __ballot_sync(kFull, u < n && e - b > kLaneRow && !big_row(off0, u));
    while (big) {
      const int j = __ffs(big) - 1;
      big &= big - 1;
      const uint32_t bb = __shfl_sync(kFull, b, j), be = __shfl_sync(kFull, e, j);
      uint32_t at = __ldg(off2 + base + j);
      for (uint32_t s0 = bb; s0 < be; s0 += 32) {
        const uint32_t s = s0 + lane;
        unsigned long long pr = 0;
        bool keep = false;
        if (s < be) {
          pr = __ldg(row + s);
          keep = is_alive(alive, (uint32_t)(pr >> 32));
        }
        const unsigned bal = __ballot_sync(kFull, keep);
        if (keep) row2[at + __popc(bal & ((1u << lane) - 1))] = pr;
        at += __popc(bal);
      }
    }
  }
}

// Big rows, a block of 1024 threads each.  Count: block sum.  Fill: chunks of
// 4096 entries, four consecutive per thread, placed by a block-wide exclusive
// scan so the row keeps its order.
__global__ void __launch_bounds__(1024) k_compact_count_big(const uint32_t* __restrict__ off,
                                                           const unsigned long long* __restrict__ row,
                                                           const uint32_t* __restrict__ alive,
                                                           uint32_t* __restrict__ cnt,
                                                           const uint32_t* __restrict__ list,
                                                           const uint32_t* __restrict__ count) {
  __shared__ unsigned long long sw[32];
  const uint32_t nbig = *count;
  for (uint32_t r = blockIdx.x; r < nbig; r += gridDim.x) {
    const uint32_t u = list[r];
    const uint32_t b = __ldg(off + u), e = __ldg(off + u + 1);
    unsigned long long c = 0;
#pragma unroll 4
    for (uint32_t s = b + threadIdx.x; s < e; s += blockDim.x) c += is_alive(alive, (uint32_t)(__ldg(row + s) >> 32));
    unsigned long long total;
    block_exclusive_scan<unsigned long long>(c, sw, total);
    if (threadIdx.x == 0) cnt[u] = (uint32_t)total;
  }
}

__global__ void __launch_bounds__(1024) k_compact_fill_big(const uint32_t* __restrict__ off,
                                                          const unsigned long long* __restrict__ row,
                                                          const uint32_t* __restrict__ alive,
                                                          const uint32_t* __restrict__ off2,
                                                          unsigned long long* __restrict__ row2,
                                                          const uint32_t* __restrict__ list,
                                                          const uint32_t* __restrict__ count) {
  __shared__ uint32_t sw[32];
  const uint32_t nbig = *count;
  for (uint32_t r = blockIdx.x; r < nbig; r += gridDim.x) {
    const uint32_t u = list[r];
    const uint32_t b = __ldg(off + u), e = __ldg(off + u + 1);
    uint32_t at = __ldg(off2 + u);
    for (uint32_t base = b; base < e; base += 4 * blockDim.x) {
      const uint32_t s0 = base + 4 * threadIdx.x;
      unsigned long long pr[4];
      uint32_t keep = 0, nk = 0;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        pr[i] = s0 + i < e ? __ldg(row + s0 + i) : 0ull;
        const bool k = s0 + i < e && is_alive(alive, (uint32_t)(pr[i] >> 32));
        keep |= (uint32_t)k << i;
        nk += k;
      }
      uint32_t total;
      uint32_t pos = at + block_exclusive_scan<uint32_t>(nk, sw, total);
#pragma unroll
      for (int i = 0; i < 4; ++i)
        if (keep & (1u << i)) row2[pos++] = pr[i];
      at += total;
    }
  }
}

// After a compaction the rows moved: rebuild the descriptors of every queued
// frontier.  `per` blocks share a member (block b serves member b / per), so
// one large frontier is spread over the whole GPU.
__global__ void __launch_bounds__(256) k_refresh_desc(const Union* __restrict__ Up,
                                                      const Member* __restrict__ mem,
                                                      const MemberState* __restrict__ st, uint32_t G,
                                                      uint32_t per) {
  const UnionRegs U(Up);
  const uint32_t g = blockIdx.x / per, part = blockIdx.x % per;
  if (g >= G) return;
  const MemberState s = st[g];
  if (s.phase != kPhaseProc) return;
  const uint32_t cnt = (uint32_t)(s.curr >> kWorkBits);
  const Member M = mem[g];
  const unsigned long long* q = (s.q_sel ? U.q1 : U.q0) + M.eb;
  uint4* qd = (s.q_sel ? U.qd1 : U.qd0) + M.eb;
  uint2* qh = U.hash_min ? (s.q_sel ? U.qh1 : U.qh0) + M.eb : nullptr;
  for (uint32_t x = part * blockDim.x + threadIdx.x; x < cnt; x += per * blockDim.x) {
    uint2 hq;
    qd[x] = edge_desc(U, M.eb + (uint32_t)(q[x] & kEidMask), &hq);
    if (qh) qh[x] = hq;
  }
}

// Publish the compacted rows and resume the loop.
__global__ void k_compact_commit(Union* U, const uint32_t* off2, const unsigned long long* row2,
                                 const uint32_t* new_slots, Control* ctl) {
  U->off = off2;
  U->row = row2;
  ctl->csr_slots = *new_slots;
  ctl->compactions += 1;
  ctl->exit_reason = kExitNone;
  ctl->done = 0;
}


// Kernel E: truss per slot = level + 2 (pkt.rs:524-526); self-loop slots 2.
// Multigraphs: `smap` takes each slot of the caller's CSR to its pair's slot
// in the deduplicated rows (nullptr: the rows are the caller's).
template <typename OutT>
__global__ void k_finalize(const unsigned long long* __restrict__ row0, const int2* __restrict__ es,
                           unsigned long long width, OutT* __restrict__ out, int u8mode, int out8,
                           uint32_t* __restrict__ kmax, uint32_t* __restrict__ err,
                           const uint32_t* __restrict__ smap) {
  unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  uint32_t mx = 0;
  bool ovf = false;
  for (; i < width; i += stride) {
    const uint32_t e = (uint32_t)(__ldg(row0 + (smap ? __ldg(smap + i) : i)) >> 32);
    uint32_t t = 2;
    if (e != kInvalid) {
      const uint32_t s = (uint32_t)__ldg(&es[e].x);
      t = s + 2;
      if (u8mode) { ovf |= s >= 255; t &= 0xFFu; }
      else if (out8) ovf |= t > 255;
    }
    mx = max(mx, t);
    out[i] = (OutT)t;
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) mx = max(mx, __shfl_down_sync(__activemask(), mx, d));
  if ((threadIdx.x & 31) == 0) atomicMax(kmax, mx);
  if (ovf) atomicOr(err, kErrOverflowU8);
}

// support per slot (Triangles::new layout): sup of the slot's edge, 0 for self-loops
// ---------------------------------------------------------------------------
// k-core decomposition (the peel of liu_et_al.rs:190-420, level-synchronous):
// degree = row length (mod 256 in u8 mode, the reference's AtomicU8); vertices
// with degree 0 get core 0; at level k every live vertex with degree <= k is
// peeled with core k, and peeling it decrements each neighbour's degree only
// while that degree exceeds k; a neighbour whose degree drops from k + 1 to k
// joins the next sub-level.  The result does not depend on the order.
__global__ void __launch_bounds__(256) k_kcore_init(const uint32_t* __restrict__ off, uint32_t n, int u8mode,
                                                    uint32_t* __restrict__ deg, uint32_t* __restrict__ alive,
                                                    uint32_t* __restrict__ core,
                                                    unsigned long long* __restrict__ remaining) {
  uint32_t live = 0;
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    const uint32_t d = __ldg(off + u + 1) - __ldg(off + u);
    deg[u] = u8mode ? (d & 0xFFu) : d;
    alive[u] = d != 0;
    core[u] = 0;
    live += d != 0;
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) live += __shfl_xor_sync(kFull, live, d);
  if (lane_id() == 0 && live) atomicAdd(remaining, (unsigned long long)live);
}

// Level k: live vertices with degree <= k form the first sub-level; the
// smallest degree left is recorded so that empty levels are skipped.
__global__ void __launch_bounds__(256) k_kcore_scan(const uint32_t* __restrict__ deg, uint32_t* __restrict__ alive,
                                                    uint32_t n, uint32_t k, uint32_t* __restrict__ frontier,
                                                    uint32_t* __restrict__ count, uint32_t* __restrict__ min_left) {
  const uint32_t lane = lane_id();
  uint32_t mn = 0xFFFFFFFFu;
  for (uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; b < n; b += gridDim.x * blockDim.x) {
    const uint32_t u = b + lane;
    bool take = false;
    if (u < n && alive[u]) {
      const uint32_t d = deg[u];
      if (d <= k) {
        take = true;
        alive[u] = 0;
      } else {
        mn = min(mn, d);
      }
    }
    const unsigned bal = __ballot_sync(kFull, take);
    if (bal) {
      uint32_t at = 0;
      if (lane == 0) at = atomicAdd(count, (uint32_t)__popc(bal));
      at = __shfl_sync(kFull, at, 0);
      if (take) frontier[at + __popc(bal & ((1u << lane) - 1))] = u;
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) mn = min(mn, __shfl_xor_sync(kFull, mn, d));
  if (lane == 0 && mn != 0xFFFFFFFFu) atomicMin(min_left, mn);
}

// One sub-level: a warp per frontier vertex.  The decrement-while-above-k is a
// compare-and-swap loop; each failed swap means the degree dropped, so the
// loop ends after at most (degree - k) tries.
__global__ void __launch_bounds__(256) k_kcore_peel(const uint32_t* __restrict__ off,
                                                    const uint32_t* __restrict__ nbr,
                                                    const uint32_t* __restrict__ frontier, uint32_t count,
                                                    uint32_t k, uint32_t* __restrict__ deg,
                                                    uint32_t* __restrict__ alive, uint32_t* __restrict__ core,
                                                    uint32_t* __restrict__ next, uint32_t* __restrict__ next_count) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = warp; i < count; i += nwarps) {
    const uint32_t u = frontier[i];
    if (lane == 0) core[u] = k;
    const uint32_t b = __ldg(off + u), e = __ldg(off + u + 1);
    for (uint32_t s0 = b; s0 < e; s0 += 32) {
      const uint32_t s = s0 + lane;
      bool push = false;
      uint32_t v = 0;
      if (s < e) {
        v = __ldg(nbr + s);
        uint32_t x = *(volatile uint32_t*)(deg + v);
        while (x > k) {
          const uint32_t old = atomicCAS(deg + v, x, x - 1);
          if (old == x) {
            push = x == k + 1 && atomicExch(alive + v, 0u) == 1u;
            break;
          }
          x = old;
        }
      }
      const unsigned bal = __ballot_sync(kFull, push);
      if (bal) {
        uint32_t at = 0;
        if (lane == 0) at = atomicAdd(next_count, (uint32_t)__popc(bal));
        at = __shfl_sync(kFull, at, 0);
        if (push) next[at + __popc(bal & ((1u << lane) - 1))] = v;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// The k-core level loop on the device: one wave kernel runs either the scan of
// level k (live vertices of degree <= k join the frontier, the smallest degree
// left is recorded) or one sub-level (a warp per frontier vertex, as
// k_kcore_peel); the last block of each wave advances the state (the next
// sub-level, the next level, or a jump past empty levels to the smallest degree
// left) and sets the CUDA-graph loop condition.  Bounded by a wave count and
// the device clock, like the PKT peel.
struct KcState {
  uint32_t phase;        // 0 scan, 1 sub-level, 2 done
  uint32_t k;
  uint32_t count;        // frontier size of the sub-level to run
  uint32_t next_count;   // wave accumulator: frontier being built
  uint32_t min_left;     // wave accumulator (scan): smallest degree above k
  uint32_t sel;          // queue holding the frontier
  uint32_t levels, subs, kmax;
  uint32_t blocks_done;
  uint32_t err;
  uint32_t pad;
  unsigned long long remaining;  // live vertices
  unsigned long long waves_run, max_waves, t_start, timeout_ns;
};

__global__ void k_kcore_start(KcState* st, unsigned long long max_waves, unsigned long long timeout_ns) {
  st->phase = st->remaining ? 0u : 2u;
  st->k = 1;
  st->count = 0;
  st->next_count = 0;
  st->min_left = 0xFFFFFFFFu;
  st->sel = 0;
  st->max_waves = max_waves;
  st->timeout_ns = timeout_ns;
  st->t_start = globaltimer();
}

__global__ void __launch_bounds__(256) k_kcore_wave(const uint32_t* __restrict__ off,
                                                    const uint32_t* __restrict__ nbr, uint32_t n,
                                                    uint32_t* __restrict__ deg, uint32_t* __restrict__ alive,
                                                    uint32_t* __restrict__ core, uint32_t* __restrict__ q0,
                                                    uint32_t* __restrict__ q1, KcState* st,
                                                    cudaGraphConditionalHandle handle, int use_handle) {
  const uint32_t phase = st->phase, k = st->k, sel = st->sel, count = st->count;
  const uint32_t lane = lane_id();
  if (phase == 0) {
    uint32_t* frontier = sel ? q1 : q0;
    uint32_t mn = 0xFFFFFFFFu;
    for (uint32_t b = (blockIdx.x * blockDim.x + threadIdx.x) & ~31u; b < n; b += gridDim.x * blockDim.x) {
      const uint32_t u = b + lane;
      bool take = false;
      if (u < n && alive[u]) {
        const uint32_t d = deg[u];
        if (d <= k) {
          take = true;
          alive[u] = 0;
        } else {
          mn = min(mn, d);
        }
      }
      const unsigned bal = __ballot_sync(kFull, take);
      if (bal) {
        uint32_t at = 0;
        if (lane == 0) at = atomicAdd(&st->next_count, (uint32_t)__popc(bal));
        at = __shfl_sync(kFull, at, 0);
        if (take) frontier[at + __popc(bal & ((1u << lane) - 1))] = u;
      }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) mn = min(mn, __shfl_xor_sync(kFull, mn, d));
    if (lane == 0 && mn != 0xFFFFFFFFu) atomicMin(&st->min_left, mn);
  } else if (phase == 1) {
    const uint32_t* frontier = sel ? q1 : q0;
    uint32_t* next = sel ? q0 : q1;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = warp; i < count; i += nwarps) {
      const uint32_t u = frontier[i];
      if (lane == 0) core[u] = k;
      const uint32_t b = __ldg(off + u), e = __ldg(off + u + 1);
      for (uint32_t s0 = b; s0 < e; s0 += 32) {
        const uint32_t s = s0 + lane;
        bool push = false;
        uint32_t v = 0;
        if (s < e) {
          v = __ldg(nbr + s);
          uint32_t x = *(volatile uint32_t*)(deg + v);
          while (x > k) {
            const uint32_t old = atomicCAS(deg + v, x, x - 1);
            if (old == x) {
              push = x == k + 1 && atomicExch(alive + v, 0u) == 1u;
              break;
            }
            x = old;
          }
        }
        const unsigned bal = __ballot_sync(kFull, push);
        if (bal) {
          uint32_t at = 0;
          if (lane == 0) at = atomicAdd(&st->next_count, (uint32_t)__popc(bal));
          at = __shfl_sync(kFull, at, 0);
          if (push) next[at + __popc(bal & ((1u << lane) - 1))] = v;
        }
      }
    }
  }
  // the last block to finish plans the next wave
  __shared__ uint32_t s_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&st->blocks_done, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  st->blocks_done = 0;
  uint32_t done = phase == 2;
  if (!done) {
    const uint32_t found = *(volatile uint32_t*)&st->next_count;
    if (phase == 0) {
      if (found) {
        st->count = found;
        st->phase = 1;
        st->levels += 1;
        st->kmax = k;
      } else {
        const uint32_t ml = *(volatile uint32_t*)&st->min_left;
        if (ml == 0xFFFFFFFFu) { st->err |= kErrInternal; done = 1; }  // live vertices, none found
        else st->k = max(k + 1, ml);
      }
    } else {
      st->remaining -= min(st->remaining, (unsigned long long)count);
      st->subs += 1;
      if (found) {
        st->count = found;
        st->sel = sel ^ 1u;
      } else {
        st->count = 0;
        st->k = k + 1;
        st->phase = 0;
      }
    }
    st->next_count = 0;
    st->min_left = 0xFFFFFFFFu;
    st->waves_run += 1;
    if (st->remaining == 0 && st->phase == 0) done = 1;
    if (st->waves_run > st->max_waves) { st->err |= kErrWaves; done = 1; }
    if (globaltimer() - st->t_start > st->timeout_ns) { st->err |= kErrTimeout; done = 1; }
    if (done) st->phase = 2;
  }
  if (use_handle) cudaGraphSetConditional(handle, done ? 0u : 1u);
}

template <typename OutT>
__global__ void k_kcore_out(const uint32_t* __restrict__ core, uint32_t n, OutT* __restrict__ out) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x)
    out[u] = (OutT)core[u];
}

// Local clustering coefficient per vertex, and the sums behind the average and
// the transitivity, from the edge supports (clustering_coefficient.rs:93-190
// restated): with d = |N(u)| (distinct neighbours; a self-loop counts),
// possible(u) = d(d - 1)/2 for d > 1, t(u) = ceil(sum of u's slot supports /
// 2) = triangles at u, local(u) = t(u) / possible(u) or 0.  Slot supports are
// reduced mod 256 in u8 mode, as the reference's AtomicU8 counts are.  Rows
// of up to kLaneRow entries per lane, longer rows per warp.
__device__ __forceinline__ uint32_t slot_support(unsigned long long pr, const int2* __restrict__ es,
                                                 int u8mode) {
  const uint32_t e = (uint32_t)(pr >> 32);
  const uint32_t s = e == kInvalid ? 0u : (uint32_t)__ldg(&es[e].x);
  return u8mode ? (s & 0xFFu) : s;
}

// Multigraphs: the rows are the deduplicated ones (so d counts distinct
// neighbours, the reference's HashSet) and `mult` gives each slot's copies,
// every copy carrying the pair's support.
__global__ void __launch_bounds__(256) k_clustering(const uint32_t* __restrict__ off,
                                                    const unsigned long long* __restrict__ row0,
                                                    const int2* __restrict__ es, uint32_t n, int u8mode,
                                                    double* __restrict__ local, double* __restrict__ sum_possible,
                                                    double* __restrict__ sum_local,
                                                    unsigned long long* __restrict__ sum_slots,
                                                    const uint32_t* __restrict__ mult) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  double acc_p = 0.0, acc_l = 0.0;
  unsigned long long acc_s = 0;
  for (uint32_t base = warp * 32; base < n; base += nwarps * 32) {
    const uint32_t u = base + lane;
    uint32_t b = 0, e = 0;
    if (u < n) { b = __ldg(off + u); e = __ldg(off + u + 1); }
    unsigned long long ts = 0;
    if (u < n && e - b <= kLaneRow)
      for (uint32_t s = b; s < e; ++s)
        ts += (unsigned long long)slot_support(__ldg(row0 + s), es, u8mode) * (mult ? __ldg(mult + s) : 1u);
    unsigned big = __ballot_sync(kFull, u < n && e - b > kLaneRow);
    while (big) {
      const int j = __ffs(big) - 1;
      big &= big - 1;
      const uint32_t bb = __shfl_sync(kFull, b, j), be = __shfl_sync(kFull, e, j);
      unsigned long long c = 0;
      for (uint32_t s = bb + lane; s < be; s += 32)
        c += (unsigned long long)slot_support(__ldg(row0 + s), es, u8mode) * (mult ? __ldg(mult + s) : 1u);
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) c += __shfl_xor_sync(kFull, c, d);
      if (lane == (uint32_t)j) ts = c;
    }
    if (u < n) {
      const uint32_t d = e - b;
      const double possible = d > 1 ? (double)d * (double)(d - 1) / 2.0 : 0.0;
      const double tri = (double)((ts + 1) / 2);
      const double loc = possible > 0.0 ? tri / possible : 0.0;
      local[u] = loc;
      acc_p += possible;
      acc_l += loc;
      acc_s += ts;
    }
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    acc_p += __shfl_xor_sync(kFull, acc_p, d);
    acc_l += __shfl_xor_sync(kFull, acc_l, d);
    acc_s += __shfl_xor_sync(kFull, acc_s, d);
  }
  if (lane == 0) {
    if (acc_p != 0.0) atomicAdd(sum_possible, acc_p);
    if (acc_l != 0.0) atomicAdd(sum_local, acc_l);
    if (acc_s) atomicAdd(sum_slots, acc_s);
  }
}

__global__ void k_support_slots(const unsigned long long* __restrict__ row0, const int2* __restrict__ es,
                                unsigned long long width, uint32_t* __restrict__ out, int u8mode,
                                const uint32_t* __restrict__ smap) {
  unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (; i < width; i += stride) {
    const uint32_t e = (uint32_t)(__ldg(row0 + (smap ? __ldg(smap + i) : i)) >> 32);
    uint32_t s = e == kInvalid ? 0u : (uint32_t)__ldg(&es[e].x);
    out[i] = u8mode ? (s & 0xFFu) : s;
  }
}

// ---------------------------------------------------------------------------
// Multigraphs (the reference's OneOrMany paths, impl_csc.rs:154-215,
// triangles.rs:172-224, pkt.rs:373-395): parallel edges are equal neighbour
// ids side by side in a row.  All copies of a pair are interchangeable, so
// they share one truss number; the engine reduces each row to its distinct
// neighbours with a multiplicity per slot, runs the weighted support and peel
// on those rows, and maps every caller slot back to its pair.  A warp per row
// (cold path: only multigraphs take it).
//   k_dedupe_count  distinct neighbours per row
//   k_dedupe_fill   deduplicated rows, copies per slot, caller slot -> slot
//   k_mult_out      multiplicity per edge id, from each pair's out-slot
//   k_mult_check    an in-slot must agree (else the CSR is not symmetric)
__global__ void __launch_bounds__(256) k_dedupe_count(const uint32_t* __restrict__ off,
                                                      const uint32_t* __restrict__ nbr, uint32_t n,
                                                      uint32_t* __restrict__ dcount) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = warp; u < n; u += nwarps) {
    const uint32_t b = __ldg(off + u), e = __ldg(off + u + 1);
    uint32_t c = 0;
    for (uint32_t s0 = b; s0 < e; s0 += 32) {
      const uint32_t s = s0 + lane;
      const bool head = s < e && (s == b || __ldg(nbr + s) != __ldg(nbr + s - 1));
      c += __popc(__ballot_sync(kFull, head));
    }
    if (lane == 0) dcount[u] = c;
  }
}

__global__ void __launch_bounds__(256) k_dedupe_fill(const uint32_t* __restrict__ off,
                                                     const uint32_t* __restrict__ nbr, uint32_t n,
                                                     const uint32_t* __restrict__ off2,
                                                     uint32_t* __restrict__ nbr2, uint32_t* __restrict__ mult2,
                                                     uint32_t* __restrict__ smap, uint32_t* __restrict__ err) {
  const uint32_t lane = lane_id();
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t u = warp; u < n; u += nwarps) {
    const uint32_t b = __ldg(off + u), e = __ldg(off + u + 1);
    uint32_t p0 = __ldg(off2 + u);  // slot of the run before this chunk's first head, + 1
    for (uint32_t s0 = b; s0 < e; s0 += 32) {
      const uint32_t s = s0 + lane;
      const uint32_t v = s < e ? __ldg(nbr + s) : 0u;
      const bool head = s < e && (s == b || v != __ldg(nbr + s - 1));
      const unsigned hb = __ballot_sync(kFull, head);
      // the run holding slot s: heads up to and including this lane
      const uint32_t pos = p0 + __popc(hb & (0xFFFFFFFFu >> (31 - lane))) - 1;
      if (s < e) {
        if (head) nbr2[pos] = v;
        smap[s] = pos;
        const uint32_t c = atomicAdd(mult2 + pos, 1u);
        if (c == 0xFFFFu) atomicOr(err, kErrCapacity);  // more than 65535 copies of one pair
      }
      p0 += __popc(hb);
    }
  }
}

__global__ void __launch_bounds__(256) k_mult_out(const unsigned long long* __restrict__ row0,
                                                  const uint32_t* __restrict__ owner,
                                                  const uint32_t* __restrict__ mult2, unsigned long long width,
                                                  uint32_t* __restrict__ mu) {
  for (unsigned long long s = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; s < width;
       s += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t e = (uint32_t)(__ldg(row0 + s) >> 32);
    if (e != kInvalid && __ldg(owner + s) == kInvalid) mu[e] = __ldg(mult2 + s);
  }
}

__global__ void __launch_bounds__(256) k_mult_check(const unsigned long long* __restrict__ row0,
                                                    const uint32_t* __restrict__ owner,
                                                    const uint32_t* __restrict__ mult2, unsigned long long width,
                                                    const uint32_t* __restrict__ mu, uint32_t* __restrict__ err) {
  bool bad = false;
  for (unsigned long long s = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; s < width;
       s += (unsigned long long)gridDim.x * blockDim.x) {
    const uint32_t e = (uint32_t)(__ldg(row0 + s) >> 32);
    if (e != kInvalid && __ldg(owner + s) != kInvalid) bad |= __ldg(mu + e) != __ldg(mult2 + s);
  }
  if (bad) atomicOr(err, kErrAsym);
}

// ---------------------------------------------------------------------------
// Served unions: members join a running peel between graph launches.  Their
// graphs are prepared (narrowed, oriented, supported) as a union of their own,
// then copied behind the running union's vertices, slots and edge ids with
// the ids shifted; their states start at the level-0 scan.
__global__ void k_shift_u32(uint32_t* __restrict__ dst, const uint32_t* __restrict__ src,
                            unsigned long long count, uint32_t add) {
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (unsigned long long)gridDim.x * blockDim.x)
    dst[i] = src[i] + add;
}

// row pairs (id | edge id << 32): id + id_add, edge id + eid_add (self-loops keep kInvalid)
__global__ void k_shift_pairs(unsigned long long* __restrict__ dst, const unsigned long long* __restrict__ src,
                              unsigned long long count, uint32_t id_add, uint32_t eid_add) {
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const unsigned long long pr = src[i];
    const uint32_t id = (uint32_t)pr + id_add, e = (uint32_t)(pr >> 32);
    dst[i] = make_pair(id, e == kInvalid ? kInvalid : e + eid_add);
  }
}

// rows longer than kWarpRow among vertices [v0, v1), appended to the list
__global__ void __launch_bounds__(256) k_big_rows_range(const uint32_t* __restrict__ off0, uint32_t v0, uint32_t v1,
                                                        uint32_t* __restrict__ list, uint32_t* __restrict__ count) {
  for (uint32_t u = v0 + blockIdx.x * blockDim.x + threadIdx.x; u < v1; u += gridDim.x * blockDim.x)
    if (big_row(off0, u)) list[atomicAdd(count, 1u)] = u;
}

// new members' states (the first wave of a member is its level-0 scan)
__global__ void k_member_init(const Member* __restrict__ mem, MemberState* __restrict__ st, uint32_t g0,
                              uint32_t g1) {
  for (uint32_t g = g0 + blockIdx.x * blockDim.x + threadIdx.x; g < g1; g += gridDim.x * blockDim.x) {
    MemberState s{};
    s.phase = mem[g].m ? kPhaseScan0 : kPhaseDone;
    s.act_count = mem[g].m;
    s.min_kept = 0xFFFFFFFFu;
    st[g] = s;
  }
}

// members joined: the union's member count, wave bound and working-row size grow
__global__ void k_ctl_join(Control* ctl, uint32_t G, unsigned long long add_waves, unsigned long long add_slots) {
  ctl->G = G;
  ctl->max_waves += add_waves;
  ctl->csr_slots += add_slots;
}

// One block: the pending wave's layout again (after members joined), no state
// transitions; restarts the time budget and the loop.
__global__ void k_replan(const Member* __restrict__ mem, const MemberState* __restrict__ st, Control* ctl,
                         unsigned long long* __restrict__ wpref) {
  __shared__ unsigned long long sw[32];
  const uint32_t G = ctl->G;
  unsigned long long carry = 0;
  for (uint32_t b = 0; b < G; b += blockDim.x) {
    const uint32_t g = b + threadIdx.x;
    unsigned long long w = 0;
    if (g < G) {
      const MemberState s = st[g];
      if (s.phase == kPhaseScan0 || s.phase == kPhaseScan) w = s.act_count;
      else if (s.phase == kPhaseProc) w = s.curr & kWorkMask;
    }
    unsigned long long total;
    const unsigned long long ex = block_exclusive_scan<unsigned long long>(w, sw, total);
    if (g < G) wpref[g] = carry + ex;
    carry += total;
  }
  if (threadIdx.x == 0) {
    wpref[G] = carry;
    ctl->total_work = carry;
    ctl->t_start = globaltimer();
    ctl->done = 0;
    ctl->exit_reason = kExitNone;
  }
}

// Hash tables per row (see hash_log2cap): the rows of at least `min_len`
// entries (the peel: original rows without a hub map; the support pass:
// oriented out-lists) get an open-addressed table of 2^(1+ceil(log2 d)) 8-byte
// entries at 4 * the row's start in `pool`.  A warp reads the lengths of 32
// consecutive rows at once and builds each qualifying row's table in turn in
// its own slice of shared memory (cleared, filled by compare-and-swap, then
// stored coalesced).  Rows whose table is larger than the slice are listed
// for k_table_fill_big, a block per row, which builds them in place: one warp
// issuing a long row's global compare-and-swaps one round trip at a time took
// milliseconds on R-MAT's largest non-hub rows.  Every table is written whole,
// so the pool needs no clearing beforehand; entries outside the tables are
// never read.
constexpr uint32_t kTableSmem = 1024;  // entries per warp (8 KB)
constexpr int kTableWarps = 4;

// peel: (column id | edge id << 32) from the original rows; self-loop slots
// (edge id kInvalid) stay out
struct RowPairSource {
  const unsigned long long* row0;
  __device__ __forceinline__ unsigned long long operator()(uint32_t s) const {
    const unsigned long long pr = __ldg(row0 + s);
    return (uint32_t)(pr >> 32) == kInvalid ? ~0ull : pr;
  }
};
// support: (column id | position << 32) from the oriented out-lists
struct OutListSource {
  const uint32_t* ocol;
  __device__ __forceinline__ unsigned long long operator()(uint32_t j) const {
    return (unsigned long long)__ldg(ocol + j) | ((unsigned long long)j << 32);
  }
};

template <class Source>
__global__ void __launch_bounds__(kTableWarps * 32) k_table_fill(const uint32_t* __restrict__ off, uint32_t n,
                                                                  uint32_t min_len,
                                                                  const uint32_t* __restrict__ hub_slot,
                                                                  Source src, unsigned long long* __restrict__ pool,
                                                                  uint32_t* __restrict__ big, uint32_t* big_count) {
  __shared__ unsigned long long s_tab[kTableWarps][kTableSmem];
  const uint32_t lane = lane_id();
  unsigned long long* st = s_tab[threadIdx.x >> 5];
  const unsigned long long warp = ((unsigned long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const unsigned long long nwarps = ((unsigned long long)gridDim.x * blockDim.x) >> 5;
  for (unsigned long long u0 = warp * 32; u0 < n; u0 += nwarps * 32) {
    const unsigned long long u = u0 + lane;
    uint32_t b = 0, d = 0;
    bool want = false;
    if (u < n) {
      b = __ldg(off + u);
      d = __ldg(off + u + 1) - b;
      want = d >= min_len && !(hub_slot && __ldg(hub_slot + u) != kInvalid);
    }
    const bool large = want && hash_log2cap(d) > 31 - __clz(kTableSmem);
    if (large) big[atomicAdd(big_count, 1u)] = (uint32_t)u;
    unsigned todo = __ballot_sync(kFull, want && !large);
    while (todo) {
      const int r = __ffs(todo) - 1;
      todo &= todo - 1;
      const uint32_t rb = __shfl_sync(kFull, b, r), rd = __shfl_sync(kFull, d, r);
      const uint32_t lg = hash_log2cap(rd), cap = 1u << lg, mask = cap - 1;
      for (uint32_t i = lane; i < cap; i += 32) st[i] = ~0ull;
      __syncwarp();
      for (uint32_t x = rb + lane; x < rb + rd; x += 32) {
        const unsigned long long en = src(x);
        if (en == ~0ull) continue;
        uint32_t at = hash_first((uint32_t)en, lg);
        for (uint32_t it = 0; it <= mask; ++it) {
          if (atomicCAS(st + at, ~0ull, en) == ~0ull) break;
          at = (at + 1) & mask;
        }
      }
      __syncwarp();
      unsigned long long* tb = pool + 4ull * rb;
      for (uint32_t i = lane; i < cap; i += 32) tb[i] = st[i];
      __syncwarp();
    }
  }
}

// The listed rows (tables larger than a warp's slice): a block per row, the
// table cleared and filled in place by all its threads.
template <class Source>
__global__ void __launch_bounds__(256) k_table_fill_big(const uint32_t* __restrict__ off,
                                                        const uint32_t* __restrict__ big,
                                                        const uint32_t* __restrict__ big_count, Source src,
                                                        unsigned long long* __restrict__ pool) {
  const uint32_t nb = *big_count;
  for (uint32_t i = blockIdx.x; i < nb; i += gridDim.x) {
    const uint32_t u = big[i];
    const uint32_t rb = __ldg(off + u), rd = __ldg(off + u + 1) - rb;
    const uint32_t lg = hash_log2cap(rd), cap = 1u << lg, mask = cap - 1;
    unsigned long long* tb = pool + 4ull * rb;
    for (uint32_t j = threadIdx.x; j < cap; j += blockDim.x) tb[j] = ~0ull;
    __syncthreads();
    for (uint32_t x = rb + threadIdx.x; x < rb + rd; x += blockDim.x) {
      const unsigned long long en = src(x);
      if (en == ~0ull) continue;
      uint32_t at = hash_first((uint32_t)en, lg);
      for (uint32_t it = 0; it <= mask; ++it) {
        if (atomicCAS(tb + at, ~0ull, en) == ~0ull) break;
        at = (at + 1) & mask;
      }
    }
    __syncthreads();
  }
}

}  // namespace sparx
