// Host side of the B200 PKT k-truss engine: C ABI (include/sparx_pkt.h),
// device workspace, pinned-staging upload, kernel sequencing and the
// device-resident peel loop (a CUDA graph with a conditional WHILE node whose
// body is four wave kernels; the last block of each wave plans the next).
#include <algorithm>
#include <cctype>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include <omp.h>

#include "../../include/sparx_pkt.h"
#include "pkt_kernels.cuh"
#include "mtx_kernels.cuh"
#include "relabel_kernels.cuh"

using namespace sparx;

namespace {

thread_local std::string g_last_error;

void set_error(const std::string& s) { g_last_error = s; }

#define CU(call)                                                                      \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess) {                                                          \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                 \
      return e_ == cudaErrorMemoryAllocation ? SPARX_E_OOM : SPARX_E_CUDA;            \
    }                                                                                 \
  } while (0)

inline size_t align_up(size_t x, size_t a = 256) { return (x + a - 1) / a * a; }

constexpr size_t kStageBytes = 64ull << 20;  // per staging buffer (pinned and device)
constexpr unsigned long long kDefaultTimeoutMs = 600000ull;
// working rows below this many entries are never compacted (not worth a pass)
constexpr unsigned long long kCompactMinSlots = 1ull << 20;

int status_from_flags(uint32_t f) {
  if (!f) return SPARX_OK;
  if (f & kErrMulti) return SPARX_E_MULTIGRAPH;
  if (f & (kErrRange | kErrUnsorted | kErrAsym | kErrOffsets)) return SPARX_E_INVALID_CSR;
  if (f & kErrCapacity) return SPARX_E_TOO_LARGE;
  if (f & (kErrTimeout | kErrWaves)) return SPARX_E_TIMEOUT;
  if (f & kErrInternal) return SPARX_E_CUDA;
  if (f & kErrOverflowU8) return SPARX_E_OVERFLOW_U8;
  return SPARX_E_CUDA;
}

// ---------------------------------------------------------------------------
// Tuning: the engine's performance knobs, picked per launch from a cache keyed
// on the graph's degree distribution (filled by the autotuner, sparx_autotune;
// defaults otherwise).  None of them changes a result, only the time.
struct Tuning {
  uint32_t merge_ratio = 8;        // peel: merge the rows when the longer is <= ratio x the shorter
  uint32_t hub_min_degree = 1024;  // dense hub maps for vertices of at least this degree (0: none)
  uint32_t sample_min = 64;        // support: longer out-lists from this length go through 64 samples
  uint32_t support_kernel = 1;     // 1 balanced edge form, 2 vertex form
  uint32_t compact_pct = 85;       // rebuild the peel's rows when live entries fill <= this % of them
  uint32_t hash_min_degree = 128;  // rows of at least this degree get a hash table for the per-lane search (0: none)
  uint32_t sup_hash_min = 0;       // support: out-lists of at least this length are probed in a hash table (0: none)
  uint32_t relabel = 0;            // rebuild the CSR on degree-ordered vertex ids first (0/1)
};

// Degree-distribution signature: log2 of the slot count, log2 bucket of the
// largest degree, and the share (in eighths) of slots in rows of degree >= 256.
// hist_cnt[b] / hist_slots[b]: vertices / slots with degree in [2^(b-1), 2^b).
struct TuneKey {
  uint32_t log_w = 0, log_dmax = 0, skew8 = 0;
  bool operator<(const TuneKey& o) const {
    return std::tie(log_w, log_dmax, skew8) < std::tie(o.log_w, o.log_dmax, o.skew8);
  }
};

TuneKey tune_key(const uint32_t* hist_cnt, const unsigned long long* hist_slots, uint64_t W) {
  TuneKey k;
  k.log_w = W ? 63 - __builtin_clzll(W) : 0;
  unsigned long long heavy = 0, total = 0;
  for (int b = 1; b <= 32; ++b) {
    if (hist_cnt[b]) k.log_dmax = (uint32_t)b;
    total += hist_slots[b];
    if (b >= 9) heavy += hist_slots[b];
  }
  k.skew8 = total ? (uint32_t)std::min<unsigned long long>(7, 8 * heavy / total) : 0;
  return k;
}

// The knobs a key gets without a cached choice: the defaults, with the vertex
// form of the support pass for unskewed graphs whose largest degree is 64..255
// (no slots in rows of degree >= 256).  Measured on one B200 with both forms:
// ER n = 4.2 M, m = 67 M support 5.4 vs 7.8 ms, mix members of that class
// 0.86-1.56 vs 1.09-2.56 ms; smaller largest degrees (de Bruijn graphs, sparse
// ER) and skewed graphs (R-MAT) are faster with the edge form.
Tuning default_tuning(const TuneKey& k) {
  Tuning t;
  if (k.skew8 == 0 && k.log_dmax >= 7 && k.log_dmax <= 8) t.support_kernel = 2;
  // large skewed graphs (2^26 slots or more, a quarter of them or more in rows
  // of degree >= 256) run on the degree-bucket relabelled CSR: R-MAT-22 / 23 /
  // 24 437 -> 409, 963 -> 883, 2179 -> 1962 ms; below 2^26 slots the state
  // fits the cache well enough that the relabelling costs more than it saves
  // (R-MAT-16 .. 21 and R-MAT-22 with edge factor 8: 4-25% slower)
  if (k.skew8 >= 2 && k.log_w >= 26) t.relabel = 1;
  return t;
}

std::mutex g_tune_mu;
std::map<TuneKey, Tuning> g_tune;
bool g_tune_loaded = false;
thread_local const Tuning* g_tune_force = nullptr;  // the autotuner's candidate under test
thread_local Tuning g_tune_last;                    // what the last launch on this thread used
thread_local TuneKey g_tune_last_key;

bool valid_tuning(const Tuning& t) {
  return t.merge_ratio >= 1 && t.merge_ratio <= 1024 && (t.hub_min_degree == 0 || t.hub_min_degree >= 256) &&
         t.sample_min >= 2 && (t.support_kernel == 1 || t.support_kernel == 2) && t.compact_pct >= 10 &&
         t.compact_pct <= 100 && (t.hash_min_degree == 0 || t.hash_min_degree >= 8) &&
         (t.sup_hash_min == 0 || t.sup_hash_min >= 4) && t.relabel <= 1;
}

// Text cache: one line per key,
// "log_w log_dmax skew8 merge hub sample kernel compact hash sup_hash relabel".
int tune_load_locked(const char* path) {
  FILE* f = std::fopen(path, "r");
  if (!f) return SPARX_E_NOT_FOUND;
  unsigned a, b, c, d, e, g, h, i, j, k, r;
  while (std::fscanf(f, "%u %u %u %u %u %u %u %u %u %u %u", &a, &b, &c, &d, &e, &g, &h, &i, &j, &k, &r) == 11) {
    Tuning t{d, e, g, h, i, j, k, r};
    if (valid_tuning(t)) g_tune[TuneKey{a, b, c}] = t;
  }
  std::fclose(f);
  return SPARX_OK;
}

int tune_save_locked(const char* path) {
  FILE* f = std::fopen(path, "w");
  if (!f) return SPARX_E_ARG;
  for (const auto& kv : g_tune)
    std::fprintf(f, "%u %u %u %u %u %u %u %u %u %u %u\n", kv.first.log_w, kv.first.log_dmax, kv.first.skew8,
                 kv.second.merge_ratio, kv.second.hub_min_degree, kv.second.sample_min, kv.second.support_kernel,
                 kv.second.compact_pct, kv.second.hash_min_degree, kv.second.sup_hash_min, kv.second.relabel);
  std::fclose(f);
  return SPARX_OK;
}

// The tuning a launch uses: the autotuner's candidate, else the cached choice
// for the key (the file named by SPARX_TUNE_FILE is read on first use), else
// the key's defaults.
Tuning resolve_tuning(const TuneKey& key) {
  Tuning t = default_tuning(key);
  if (g_tune_force) {
    t = *g_tune_force;
  } else {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    if (!g_tune_loaded) {
      g_tune_loaded = true;
      const char* path = std::getenv("SPARX_TUNE_FILE");
      if (path && *path) tune_load_locked(path);
    }
    auto it = g_tune.find(key);
    if (it != g_tune.end()) t = it->second;
  }
  g_tune_last = t;
  g_tune_last_key = key;
  return t;
}

struct Counters {  // device scalars
  uint32_t err;
  uint32_t kmax;
  unsigned long long self_loops;
  unsigned long long tri;
  unsigned long long grand;
  uint32_t max_dplus;    // largest oriented out-degree
  uint32_t vcursor;      // vertex-form support: next light vertex batch
  uint32_t hcursor;      //                      next heavy vertex
  uint32_t heavy_count;  //                      heavy vertices listed
  uint32_t hub_count;    // hub maps assigned
  uint32_t big_count;    // rows compacted by a block each
  uint32_t fin_err;      // served unions: error flags of one member's finalize
  uint32_t table_big;    // hash tables: rows listed for the block-per-row fill
  double cc_possible;    // clustering: sum of d(d - 1)/2 over vertices
  double cc_local;       //             sum of local coefficients
  unsigned long long cc_slots;  //      sum of slot supports
};



struct Layout {
  size_t off, nbr, row0, dplus, opos, ocol, osrc, es, act0, act1, q0, q1, qd0, qd1, out, stage0, stage1;
  size_t offA, offB, rowA, rowB;  // compaction ping-pong buffers (0 when compaction is off)
  size_t vinfo;                   // per vertex: what its row offers as a longer row (hub map / hash table)
  size_t alive;                   // compaction: one bit per edge, set while it is unprocessed
  size_t big;                     // compaction: rows longer than kWarpRow (a block each)
  size_t hub_slot, hub_vertex, hub_base, hub_hist, hub_map;  // hub maps (hub_cap == 0: none)
  uint32_t hub_cap;
  unsigned long long hub_pool;    // map entries reserved for all hubs together
  size_t tiles, ctl, mem, st, wpref, cnt, mem_tri, mem_maxsup, uni;
  size_t total;
};

// Hub maps: at most kHubMaxCount maps, each of its member's vertex count in
// u32 entries, within kHubBudgetBytes, for vertices of degree >= the tuned
// floor (never below kHubFloor, so never more than W / kHubFloor of them).
constexpr uint64_t kHubBudgetBytes = 4ull << 30;
constexpr uint32_t kHubFloor = 256;
constexpr uint32_t kHubMaxCount = 1024;

// maps reserved for a union whose largest member has `max_n` vertices
uint32_t hub_capacity(uint64_t max_n, uint64_t W) {
  if (max_n == 0 || W >= (1ull << 31)) return 0;
  const uint64_t k = std::min<uint64_t>({kHubMaxCount, W / kHubFloor, kHubBudgetBytes / (4 * max_n)});
  return (uint32_t)k;
}

Layout make_layout(uint64_t N, uint64_t W, uint32_t G, bool own_nbr, size_t out_bytes, uint64_t max_n = 0) {
  Layout L{};
  size_t p = 0;
  auto take = [&](size_t bytes) {
    size_t r = p;
    p = align_up(p + std::max<size_t>(bytes, 1));
    return r;
  };
  const uint64_t M = std::max<uint64_t>(W / 2, 1);
  L.off = take(4 * (N + 1));
  L.nbr = own_nbr ? take(4 * W) : 0;
  L.row0 = take(8 * W);
  L.dplus = take(4 * N);
  L.opos = take(4 * (N + 1));
  L.ocol = take(4 * M);
  L.osrc = take(4 * M);
  L.es = take(8 * M);
  L.act0 = take(4 * M);
  L.act1 = take(4 * M);
  L.q0 = take(16 * M + 16);  // q0 and q1 back to back; also the support prefix (M + 1 u64)
  L.q1 = L.q0 + 8 * M;
  L.qd0 = take(16 * M);
  L.qd1 = take(16 * M);
  L.out = take(out_bytes);
  L.offA = take(4 * (N + 1));
  L.offB = take(4 * (N + 1));
  L.rowA = take(8 * W);
  L.rowB = take(8 * W);
  L.alive = take(4 * ((M + 31) / 32));
  L.big = take(4 * (W / kWarpRow + 1));
  if (max_n == 0) max_n = N;
  L.hub_cap = hub_capacity(max_n, W);
  L.hub_hist = take(4 * 34 + 8 * 34);  // vertices, then slots, per log2 degree (always: the tuning key)
  L.vinfo = take(8ull * N);              // per vertex: its row's hub map or hash table (k_vinfo)
  if (L.hub_cap) {
    L.hub_pool = std::min<unsigned long long>(4ull * L.hub_cap * max_n, kHubBudgetBytes) / 4;
    L.hub_slot = take(4 * N);
    L.hub_vertex = take(4ull * L.hub_cap);
    L.hub_base = take(4ull * L.hub_cap);
    L.hub_map = take(4ull * L.hub_pool);
  }
  L.stage0 = take(kStageBytes);
  L.stage1 = take(kStageBytes);
  const uint64_t tiles = (std::max<uint64_t>(N + 1, M + 1) + kScanTile - 1) / kScanTile + 2;
  L.tiles = take(8 * tiles);
  L.ctl = take(sizeof(Control));
  L.mem = take(sizeof(Member) * G);
  L.st = take(sizeof(MemberState) * G);
  L.wpref = take(8ull * (G + 1));
  L.cnt = take(sizeof(Counters));
  L.mem_tri = take(8ull * G);
  L.mem_maxsup = take(4ull * G);
  L.uni = take(sizeof(Union));
  L.total = p;
  return L;
}

struct PeelGraph {
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  std::vector<size_t> key;
};

struct Engine {
  int device = 0;
  int sm_count = 148;
  cudaStream_t stream = nullptr;
  cudaStream_t capture = nullptr;
  char* ws = nullptr;
  size_t ws_cap = 0;
  void* pinned[2] = {nullptr, nullptr};
  cudaEvent_t pin_ev[2] = {nullptr, nullptr};
  cudaEvent_t tev[8] = {};
  void* pinned_small = nullptr;  // 4 KB for scalar read-backs
  PeelGraph peel;
  int wave_blocks = 0;        // k_wave<false> grid (resident blocks per SM x SMs)
  int wave_blocks_multi = 0;  // k_wave<true> grid (multigraphs)
  char* ws2 = nullptr;        // multigraph rows, multiplicities and slot map (allocated on first use)
  size_t ws2_cap = 0;
  char* ws3 = nullptr;        // row hash tables and their queue descriptors (allocated on first use)
  size_t ws3_cap = 0;
  ulonglong4* trace = nullptr;  // wave trace records (SPARX_TRACE_FILE set)
  std::mutex mu;
};

constexpr unsigned long long kTraceRecords = 1ull << 20;

std::mutex g_engines_mu;
std::map<int, Engine*> g_engines;

int engine_init(Engine& E, int device) {
  E.device = device;
  CU(cudaSetDevice(device));
  CU(cudaDeviceGetAttribute(&E.sm_count, cudaDevAttrMultiProcessorCount, device));
  CU(cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking));
  CU(cudaStreamCreateWithFlags(&E.capture, cudaStreamNonBlocking));
  for (int i = 0; i < 2; ++i) {
    CU(cudaHostAlloc(&E.pinned[i], kStageBytes, cudaHostAllocDefault));
    CU(cudaEventCreateWithFlags(&E.pin_ev[i], cudaEventDisableTiming));
    CU(cudaEventRecord(E.pin_ev[i], E.stream));
  }
  for (auto& e : E.tev) CU(cudaEventCreate(&e));
  CU(cudaHostAlloc(&E.pinned_small, 4096, cudaHostAllocDefault));
  int per_sm = 0;
  CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wave<false>, 256, 0));
  E.wave_blocks = std::max(1, per_sm) * E.sm_count;
  CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wave<true>, 256, 0));
  E.wave_blocks_multi = std::max(1, per_sm) * E.sm_count;
  return SPARX_OK;
}

int get_engine(int device, Engine** out) {
  if (device < 0) {
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) {
      set_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
      return SPARX_E_CUDA;
    }
  }
  std::lock_guard<std::mutex> lk(g_engines_mu);
  auto it = g_engines.find(device);
  if (it != g_engines.end()) { *out = it->second; return SPARX_OK; }
  Engine* E = new Engine();
  int rc = engine_init(*E, device);
  if (rc) { delete E; return rc; }
  g_engines[device] = E;
  *out = E;
  return SPARX_OK;
}

int ensure_ws(Engine& E, size_t bytes, bool slack = true) {
  if (E.ws_cap >= bytes) return SPARX_OK;
  if (E.peel.exec) {
    cudaGraphExecDestroy(E.peel.exec);
    cudaGraphDestroy(E.peel.graph);
    E.peel = PeelGraph{};
  }
  if (E.ws) { CU(cudaStreamSynchronize(E.stream)); CU(cudaFree(E.ws)); E.ws = nullptr; E.ws_cap = 0; }
  size_t cap = align_up(slack ? bytes + bytes / 8 : bytes, 1 << 21);
  cudaError_t e = cudaMalloc(&E.ws, cap);
  if (e != cudaSuccess) {
    cudaGetLastError();
    e = cudaMalloc(&E.ws, bytes);
    cap = bytes;
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error(std::string("workspace of ") + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e));
      E.ws = nullptr;
      return SPARX_E_OOM;
    }
  }
  E.ws_cap = cap;
  return SPARX_OK;
}

int ensure_ws3(Engine& E, size_t bytes) {
  if (E.ws3_cap >= bytes) return SPARX_OK;
  if (E.ws3) { CU(cudaStreamSynchronize(E.stream)); CU(cudaFree(E.ws3)); E.ws3 = nullptr; E.ws3_cap = 0; }
  cudaError_t e = cudaMalloc(&E.ws3, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(std::string("hash table workspace of ") + std::to_string(bytes) + " bytes: " + cudaGetErrorString(e));
    E.ws3 = nullptr;
    return SPARX_E_OOM;
  }
  E.ws3_cap = bytes;
  return SPARX_OK;
}

int ensure_ws2(Engine& E, size_t bytes) {
  if (E.ws2_cap >= bytes) return SPARX_OK;
  if (E.ws2) { CU(cudaStreamSynchronize(E.stream)); CU(cudaFree(E.ws2)); E.ws2 = nullptr; E.ws2_cap = 0; }
  cudaError_t e = cudaMalloc(&E.ws2, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(std::string("second workspace (deduplicated or relabelled rows) of ") + std::to_string(bytes) + " bytes: " +
              cudaGetErrorString(e));
    E.ws2 = nullptr;
    return SPARX_E_OOM;
  }
  E.ws2_cap = bytes;
  return SPARX_OK;
}

void parallel_copy(void* dst, const void* src, size_t bytes) {
  const size_t piece = 4ull << 20;
  const long pieces = (long)((bytes + piece - 1) / piece);
  if (pieces <= 1) { std::memcpy(dst, src, bytes); return; }
  int nt = std::min<int>(omp_get_max_threads(), 16);
#pragma omp parallel for num_threads(nt) schedule(static)
  for (long i = 0; i < pieces; ++i) {
    size_t o = (size_t)i * piece;
    std::memcpy((char*)dst + o, (const char*)src + o, std::min(piece, bytes - o));
  }
}

inline int grid_for(unsigned long long items, int threads, int cap_blocks) {
  unsigned long long b = (items + threads - 1) / threads;
  return (int)std::max<unsigned long long>(1, std::min<unsigned long long>(b, (unsigned long long)cap_blocks));
}

// host ids (u64 or u32) -> device u32 (+ base), chunked through pinned staging:
// host threads narrow each chunk to u32 and check id < n while copying it into
// the pinned buffer (so 4 bytes per slot cross PCIe, not 8), and the chunk goes
// straight to its place in HBM.  A bad id sets kErrRange in *d_err's host twin.
int upload_ids(Engine& E, const void* host, int bits, uint64_t count, uint32_t* dst, uint64_t n_limit,
               uint32_t base, cudaStream_t s, char* stage[2], uint32_t* d_err) {
  (void)stage;
  const uint64_t chunk = kStageBytes / 4;
  bool bad = false;
  for (uint64_t c = 0, at = 0; at < count; ++c, at += chunk) {
    const int slot = (int)(c & 1);
    const uint64_t k = std::min<uint64_t>(chunk, count - at);
    CU(cudaEventSynchronize(E.pin_ev[slot]));
    uint32_t* buf = (uint32_t*)E.pinned[slot];
    const long long pieces = (long long)((k + (1u << 18) - 1) >> 18);
    bool chunk_bad = false;
#pragma omp parallel for schedule(static) reduction(|| : chunk_bad) num_threads(std::min<int>(omp_get_max_threads(), 16))
    for (long long pi = 0; pi < pieces; ++pi) {
      const uint64_t lo = (uint64_t)pi << 18, hi = std::min<uint64_t>(k, lo + (1u << 18));
      bool b = false;
      if (bits == 64) {
        const uint64_t* src = (const uint64_t*)host + at;
        for (uint64_t i = lo; i < hi; ++i) {
          const uint64_t x = src[i];
          b |= x >= n_limit;
          buf[i] = (uint32_t)x + base;
        }
      } else {
        const uint32_t* src = (const uint32_t*)host + at;
        for (uint64_t i = lo; i < hi; ++i) {
          const uint32_t x = src[i];
          b |= x >= n_limit;
          buf[i] = x + base;
        }
      }
      chunk_bad = chunk_bad || b;
    }
    bad = bad || chunk_bad;
    CU(cudaMemcpyAsync(dst + at, buf, k * 4, cudaMemcpyHostToDevice, s));
    CU(cudaEventRecord(E.pin_ev[slot], s));
  }
  if (bad) {
    const uint32_t flag = kErrRange;
    CU(cudaMemcpyAsync(d_err, &flag, 4, cudaMemcpyHostToDevice, s));  // pageable: copied before return
  }
  return SPARX_OK;
}

int download(Engine& E, void* host, const void* dev, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return SPARX_OK;
  const size_t chunk = kStageBytes;
  const size_t nchunks = (bytes + chunk - 1) / chunk;
  // issue chunk 0, then overlap copy-out of chunk c with the D2H of chunk c + 1
  auto issue = [&](size_t c) -> int {
    const int slot = (int)(c & 1);
    const size_t at = c * chunk, k = std::min(chunk, bytes - at);
    CU(cudaMemcpyAsync(E.pinned[slot], (const char*)dev + at, k, cudaMemcpyDeviceToHost, s));
    CU(cudaEventRecord(E.pin_ev[slot], s));
    return SPARX_OK;
  };
  CU(cudaEventSynchronize(E.pin_ev[0]));
  CU(cudaEventSynchronize(E.pin_ev[1]));
  int rc = issue(0);
  if (rc) return rc;
  for (size_t c = 0; c < nchunks; ++c) {
    const int slot = (int)(c & 1);
    if (c + 1 < nchunks) {
      rc = issue(c + 1);
      if (rc) return rc;
    }
    CU(cudaEventSynchronize(E.pin_ev[slot]));
    const size_t at = c * chunk, k = std::min(chunk, bytes - at);
    parallel_copy((char*)host + at, E.pinned[slot], k);
  }
  return SPARX_OK;
}

template <class T, class F>
void exclusive_scan(F f, unsigned long long count, T* out, T* tiles, T* grand, cudaStream_t s) {
  const unsigned long long ntiles = std::max<unsigned long long>(1, (count + kScanTile - 1) / kScanTile);
  k_scan_reduce<T, F><<<(unsigned)ntiles, kScanThreads, 0, s>>>(f, count, tiles);
  k_scan_tiles<T><<<1, kScanThreads, 0, s>>>(tiles, ntiles, grand);
  k_scan_apply<T, F><<<(unsigned)ntiles, kScanThreads, 0, s>>>(f, count, tiles, out);
}

// Triangle support per oriented edge into es[].x (zeroed by the caller).
// The vertex form needs a shared-memory table of 2x the largest out-degree;
// beyond what a CTA can hold the balanced form runs instead.
constexpr size_t kHeavySmemLimit = 160u << 10;

int launch_support(int sm_count, uint32_t support_kernel, uint32_t n, uint64_t m, uint32_t max_dplus,
                   const uint32_t* opos, const uint32_t* ocol, const uint32_t* osrc, int2* es,
                   unsigned long long* spref, unsigned long long* tiles, Counters* cnt, uint32_t* heavy_list,
                   cudaStream_t s, uint32_t* launches, unsigned long long* support_elements,
                   const uint32_t* mu = nullptr, uint32_t sample_min = Tuning{}.sample_min,
                   const unsigned long long* hpool = nullptr, uint32_t hash_min = 0) {
  if (m == 0) return SPARX_OK;
  uint32_t slots = 8;
  while (slots < 2 * max_dplus) slots <<= 1;
  const size_t hsmem = heavy_smem_bytes(slots, max_dplus);
  // auto picks the balanced form: on R-MAT-22 it runs in 131 ms against 221 ms
  // for the vertex form (B200, measured)
  const bool vertex_form = support_kernel == 2 && !mu;  // multigraph weights: the balanced form only
  if (vertex_form && hsmem <= kHeavySmemLimit) {
    k_support_light<<<sm_count * 8, 256, 0, s>>>(opos, ocol, n, es, &cnt->tri, heavy_list, &cnt->heavy_count,
                                                 &cnt->vcursor);
    CU(cudaFuncSetAttribute(k_support_heavy, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsmem));
    k_support_heavy<<<sm_count * 4, 256, hsmem, s>>>(opos, ocol, es, &cnt->tri, heavy_list, &cnt->heavy_count,
                                                     &cnt->hcursor, slots, max_dplus);
    *launches += 2;
    *support_elements = 0;
    return SPARX_OK;
  }
  exclusive_scan<unsigned long long>(SupportWork{opos, osrc, ocol}, m, spref, tiles, &cnt->grand, s);
  const int g = sm_count * 8;
  const uint32_t mm = (uint32_t)m;
  if (hpool && hash_min) {
    if (mu)
      k_support_balanced<true, true><<<g, 256, 0, s>>>(opos, ocol, osrc, spref, mm, es, &cnt->tri, &cnt->err, mu,
                                                       sample_min, hpool, hash_min);
    else
      k_support_balanced<false, true><<<g, 256, 0, s>>>(opos, ocol, osrc, spref, mm, es, &cnt->tri, &cnt->err,
                                                        nullptr, sample_min, hpool, hash_min);
  } else if (mu) {
    k_support_balanced<true, false><<<g, 256, 0, s>>>(opos, ocol, osrc, spref, mm, es, &cnt->tri, &cnt->err, mu,
                                                      sample_min, nullptr, 0);
  } else {
    k_support_balanced<false, false><<<g, 256, 0, s>>>(opos, ocol, osrc, spref, mm, es, &cnt->tri, &cnt->err,
                                                       nullptr, sample_min, nullptr, 0);
  }
  *launches += 4;
  CU(cudaMemcpyAsync(support_elements, spref + m, 8, cudaMemcpyDeviceToHost, s));
  return SPARX_OK;
}

__global__ void k_member_edges(Member* mem, uint32_t G, const uint32_t* opos) {
  for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < G; g += gridDim.x * blockDim.x) {
    const uint32_t eb = opos[mem[g].vb];
    mem[g].eb = eb;
    mem[g].m = opos[mem[g].vb + mem[g].n] - eb;
  }
}

struct Opts {
  uint32_t support_mode = SPARX_SUPPORT_WIDE;
  uint32_t out_bits = 8;
  int device = -1;
  uint32_t loop = SPARX_LOOP_GRAPH;
  uint32_t support_kernel = 0;
  unsigned long long timeout_ms = kDefaultTimeoutMs;
};

int read_opts(const sparx_pkt_opts* o, Opts* out) {
  Opts d;
  if (o) {
    if (o->struct_size && o->struct_size < sizeof(sparx_pkt_opts)) { set_error("opts.struct_size too small"); return SPARX_E_ARG; }
    d.support_mode = o->support_mode;
    d.out_bits = o->out_bits ? o->out_bits : 8;
    d.device = o->device;
    d.loop = o->loop;
    d.support_kernel = o->support_kernel;
    d.timeout_ms = o->timeout_ms ? o->timeout_ms : kDefaultTimeoutMs;
  }
  if (d.support_mode > 1 || (d.out_bits != 8 && d.out_bits != 32) || d.loop > 1) {
    set_error("bad option value");
    return SPARX_E_ARG;
  }
  *out = d;
  return SPARX_OK;
}

// A prepared launch: members laid out in one union, CSR already on device.
struct UnionJob;
struct Engine;
// The peel loop's state a served union's hook may change between launches.
struct PeelCtx {
  Union U;                        // host copy (working rows, counts)
  const uint32_t* cur_off;        // working rows in use
  const unsigned long long* cur_row;
  unsigned long long csr_slots;   // entries in the working rows
  uint64_t m;                     // edges in the union
  uint64_t Ws;                    // slots in the union
  uint32_t N, G;
  uint64_t waves_run = 0;         // waves the union's loop has run so far
  bool resume = false;            // the hook added members or some are still running
};
// Served unions: called at every stop of the peel loop (a member finished,
// requests wait to join, a compaction, the end); delivers finished members
// and may append new ones.
struct ServeHook {
  virtual ~ServeHook() = default;
  virtual int at_stop(Engine& E, UnionJob& J, PeelCtx& ctx, uint32_t reason, cudaStream_t s) = 0;
  const volatile uint32_t* admit_dev = nullptr;  // device view of the lane's admission word
};

struct UnionJob {
  uint64_t N = 0, W = 0;
  ServeHook* hook = nullptr;     // served union (members join and leave between graph launches)
  bool prep_only = false;        // stop after the support pass (members about to join a served union)
  const uint32_t* smap = nullptr;  // multigraphs: caller slot -> deduplicated slot (device)
  uint64_t budget = 0;             // device bytes the launch may hold (batched and served unions); 0: no bound
  bool hook_hash = false;          // served union that takes no joins: row hash tables allowed
  uint64_t prep_m = 0, prep_Ws = 0;  // prep_only: edges and slots prepared
  std::vector<Member> members;  // vb, n, sb, w set; eb, m filled by the pipeline
  Layout L{};
  uint32_t* off = nullptr;
  const uint32_t* nbr = nullptr;
  void* out = nullptr;          // device truss output (u8 or u32 per slot)
  bool support_only = false;
  uint32_t* support_out = nullptr;  // device u32 per slot (support_only)
  bool clustering = false;          // support_only, then local coefficients (f64 per vertex) into out
  bool kcore = false;               // k-core decomposition: core per vertex into out
  bool multi = false;               // parallel edges found: rows were deduplicated
  uint64_t slot_self_loops = 0;     // self-loop slots of the caller's CSR
  uint32_t kc_levels = 0, kc_waves = 0, kc_max = 0;
  double cc_possible = 0, cc_local = 0;
  unsigned long long cc_slots = 0;
  // results
  std::vector<MemberState> states;
  std::vector<unsigned long long> mem_tri;
  std::vector<uint32_t> mem_maxsup;
  unsigned long long self_loops = 0, tri = 0;
  uint32_t kmax = 0;
  uint32_t err = 0;
  float ms_orient = 0, ms_support = 0, ms_peel = 0, ms_finalize = 0;
  uint32_t launches = 0;
  unsigned long long support_elements = 0;
  uint32_t hubs = 0;  // hub maps built
  Tuning tuning;      // the knobs this launch used
  Control ctl{};
};

template <class T>
T* at(Engine& E, size_t off) { return reinterpret_cast<T*>(E.ws + off); }

PeelArrays peel_arrays(const Union& U) {
  PeelArrays a{};
  a.ocol = U.ocol;
  a.osrc = U.osrc;
  a.es = U.es;
  a.act0 = U.act[0];
  a.act1 = U.act[1];
  a.q0 = U.q[0];
  a.q1 = U.q[1];
  a.qd0 = U.qd[0];
  a.qd1 = U.qd[1];
  a.hub_slot = U.hub_slot;
  a.hub_map = U.hub_map;
  a.hub_base = U.hub_base;
  a.mu = nullptr;
  a.hpool = U.hpool;
  a.off0 = U.off0;
  a.qh0 = U.qh[0];
  a.qh1 = U.qh[1];
  a.n = U.n;
  a.merge_ratio = Tuning{}.merge_ratio;
  a.hash_min = U.hash_min;
  a.pad = 0;
  return a;
}

#ifndef SPARX_WAVES_PER_ITERATION
#define SPARX_WAVES_PER_ITERATION 4
#endif
constexpr int kWavesPerIteration = SPARX_WAVES_PER_ITERATION;

int build_peel_graph(Engine& E, const UnionJob& J, const PeelArrays& arr) {
  const Layout& L = J.L;
  std::vector<size_t> key = {(size_t)E.ws, L.uni, L.mem, L.st, L.ctl, L.wpref, L.cnt, (size_t)J.members.size(),
                             (size_t)E.wave_blocks, (size_t)E.wave_blocks_multi};
  // the arrays are baked into the captured kernels' parameters
  static_assert(sizeof(PeelArrays) % sizeof(size_t) == 0, "PeelArrays is keyed word by word");
  const size_t* words = reinterpret_cast<const size_t*>(&arr);
  key.insert(key.end(), words, words + sizeof(PeelArrays) / sizeof(size_t));
  if (E.peel.exec && E.peel.key == key) return SPARX_OK;
  if (E.peel.exec) {
    cudaGraphExecDestroy(E.peel.exec);
    cudaGraphDestroy(E.peel.graph);
    E.peel = PeelGraph{};
  }
  cudaGraph_t g;
  CU(cudaGraphCreate(&g, 0));
  cudaGraphConditionalHandle h;
  CU(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  CU(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  WaveArgs wa;
  wa.Up = at<Union>(E, L.uni);
  wa.arr = arr;
  wa.mem = at<Member>(E, L.mem);
  wa.st = at<MemberState>(E, L.st);
  wa.ctl = at<Control>(E, L.ctl);
  wa.wpref = at<unsigned long long>(E, L.wpref);
  wa.err = &at<Counters>(E, L.cnt)->err;
  wa.handle = h;
  wa.use_handle = 1;
  CU(cudaStreamBeginCaptureToGraph(E.capture, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
  // several waves per loop iteration: a wave that finds the loop stopped does
  // nothing, and the condition is read once per iteration
  for (int i = 0; i < kWavesPerIteration; ++i) {
    if (arr.mu) k_wave<true><<<E.wave_blocks_multi, 256, 0, E.capture>>>(wa);
    else k_wave<false><<<E.wave_blocks, 256, 0, E.capture>>>(wa);
  }
  cudaGraph_t captured;
  CU(cudaStreamEndCapture(E.capture, &captured));
  cudaGraphExec_t ex;
  CU(cudaGraphInstantiate(&ex, g, 0));
  E.peel.exec = ex;
  E.peel.graph = g;
  E.peel.key = key;
  return SPARX_OK;
}

// Stable LSD radix sort of u64 keys (and a u32 payload when pa is given) over
// the 8-bit digits at `shifts` (mtx_kernels.cuh); returns the buffers holding
// the sorted keys and payload.
struct SortedBufs {
  unsigned long long* keys;
  uint32_t* pay;
};
SortedBufs radix_sort(int sm_count, unsigned long long* ka, unsigned long long* kb, uint32_t* pa, uint32_t* pb,
                      unsigned long long count, const std::vector<int>& shifts, uint32_t* hist, uint32_t* hstart,
                      uint32_t* tiles, uint32_t* grand, cudaStream_t s) {
  const uint32_t blocks =
      (uint32_t)std::max<unsigned long long>(1, std::min<unsigned long long>(sm_count * 4ull, (count + 4095) / 4096));
  if (count > 1) {
    for (int sh : shifts) {
      k_radix_hist<<<blocks, kRadixThreads, 0, s>>>(ka, count, sh, hist);
      exclusive_scan<uint32_t>(LoadU32{hist}, 256ull * blocks, hstart, tiles, grand, s);
      if (pa)
        k_radix_scatter<true><<<blocks, kRadixThreads, 0, s>>>(ka, kb, count, sh, hstart, pa, pb);
      else
        k_radix_scatter<false><<<blocks, kRadixThreads, 0, s>>>(ka, kb, count, sh, hstart, nullptr, nullptr);
      std::swap(ka, kb);
      std::swap(pa, pb);
    }
  }
  return {ka, pa};
}

// Rebuild a graph's (or a union's) CSR on vertex ids in (floor(log2 degree),
// id) order within each member's id range (relabel_kernels.cuh): J.off / J.nbr
// become the new rows, J.smap the caller slot -> new slot map the finalize
// reads through.  `big` / `big_count`:
// the rows longer than kWarpRow (listed by the orientation pass).  Everything
// lives in the second workspace.
static_assert(kRelabelWarpRow == kWarpRow, "the relabel's block rows are the orientation's big-row list");
int relabel_graph(Engine& E, UnionJob& J, uint32_t N, uint64_t W, const uint32_t* big, const uint32_t* big_count,
                  cudaStream_t s) {
  const uint32_t blocks_max = (uint32_t)E.sm_count * 4;
  const uint64_t scan_items = std::max<uint64_t>(256ull * blocks_max + 1, N + 1ull);
  size_t p = 0;
  auto take = [&](size_t bytes) {
    size_t r = p;
    p = align_up(p + std::max<size_t>(bytes, 1));
    return r;
  };
  const size_t o_off = take(4ull * (N + 1)), o_nbr = take(4 * W), o_rmap = take(4 * W), o_va = take(8ull * N),
               o_vb = take(8ull * N), o_newid = take(4ull * N), o_deg = take(4ull * N), o_bucket = take(N),
               o_hist = take(4ull * 256 * blocks_max), o_hstart = take(4ull * (256 * blocks_max + 1)),
               o_tiles = take(4 * (scan_items / kScanTile + 4)), o_grand = take(4),
               o_mvb = take(4ull * J.members.size());
  int rc = ensure_ws2(E, p);
  if (rc) return rc;
  char* b = E.ws2;
  uint32_t* off_r = (uint32_t*)(b + o_off);
  uint32_t* nbr_r = (uint32_t*)(b + o_nbr);
  uint32_t* rmap = (uint32_t*)(b + o_rmap);
  uint32_t* newid = (uint32_t*)(b + o_newid);
  uint32_t* deg_r = (uint32_t*)(b + o_deg);
  uint8_t* bucket = (uint8_t*)(b + o_bucket);
  uint32_t* tiles = (uint32_t*)(b + o_tiles);
  uint32_t* grand = (uint32_t*)(b + o_grand);
  // vertices: (member, bucket, id) order; radix passes over the member and
  // bucket bits (one pass for a single graph)
  const uint32_t G = (uint32_t)J.members.size();
  std::vector<uint32_t> mvb(G);
  for (uint32_t g = 0; g < G; ++g) mvb[g] = J.members[g].vb;
  uint32_t* member_vb = (uint32_t*)(b + o_mvb);
  CU(cudaMemcpyAsync(member_vb, mvb.data(), 4ull * G, cudaMemcpyHostToDevice, s));  // pageable: staged
  const int kbits = 5 + (G > 1 ? 32 - __builtin_clz(G - 1) : 0);
  std::vector<int> vshifts;
  for (int bit = 0; bit < kbits; bit += 8) vshifts.push_back(32 + bit);
  k_vertex_keys<<<grid_for(N, 256, E.sm_count * 16), 256, 0, s>>>(J.off, N, member_vb, G,
                                                                   (unsigned long long*)(b + o_va), bucket);
  const SortedBufs vs = radix_sort(E.sm_count, (unsigned long long*)(b + o_va), (unsigned long long*)(b + o_vb),
                                   nullptr, nullptr, N, vshifts, (uint32_t*)(b + o_hist), (uint32_t*)(b + o_hstart),
                                   tiles, grand, s);
  k_vertex_order<<<grid_for(N, 256, E.sm_count * 16), 256, 0, s>>>(vs.keys, J.off, N, newid, deg_r);
  exclusive_scan<uint32_t>(LoadU32{deg_r}, N, off_r, tiles, grand, s);
  // rows: each moved to its new place and stably partitioned by bucket
  k_relabel_rows<<<grid_for(32ull * N, 256, E.sm_count * 16), 256, 0, s>>>(J.off, J.nbr, N, newid, bucket, off_r,
                                                                          nbr_r, rmap);
  k_relabel_rows_big<<<E.sm_count * 4, 256, 0, s>>>(J.off, J.nbr, big, big_count, newid, bucket, off_r, nbr_r,
                                                     rmap);
  J.launches += 10;
  J.off = off_r;
  J.nbr = nbr_r;
  J.smap = rmap;
  return SPARX_OK;
}

// Orientation, support, peel and finalize over a prepared union.
int run_union(Engine& E, UnionJob& J, const Opts& O, cudaStream_t s) {
  const Layout& L = J.L;
  const uint32_t G = (uint32_t)J.members.size();
  const uint32_t N = (uint32_t)J.N;
  const uint64_t W = J.W;
  Counters* cnt = at<Counters>(E, L.cnt);
  uint32_t* err = &cnt->err;
  unsigned long long* row0 = at<unsigned long long>(E, L.row0);
  uint32_t* dplus = at<uint32_t>(E, L.dplus);
  uint32_t* opos = at<uint32_t>(E, L.opos);
  uint32_t* ocol = at<uint32_t>(E, L.ocol);
  uint32_t* osrc = at<uint32_t>(E, L.osrc);
  int2* es = at<int2>(E, L.es);
  Member* dmem = at<Member>(E, L.mem);
  const int vgrid = grid_for(N, 256, E.sm_count * 32);  // row kernels: 32 vertices per warp

  CU(cudaEventRecord(E.tev[1], s));
  {
    // offsets / ids validated by the upload must be sound before any kernel
    // dereferences them
    uint32_t* herr = (uint32_t*)E.pinned_small;
    CU(cudaMemcpyAsync(herr, err, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (*herr) { J.err = *herr; return status_from_flags(*herr); }
  }
  // -- orientation (Kernel B) --
  const bool hubs_possible = L.hub_cap > 0 && !J.support_only;
  uint32_t* hub_hist = at<uint32_t>(E, L.hub_hist);  // degree signature (tuning key) and hub choice
  unsigned long long* hub_hist_slots = reinterpret_cast<unsigned long long*>(hub_hist + 34);
  uint32_t* big = at<uint32_t>(E, L.big);
  // multigraphs: deduplicated rows, copies per slot, caller slot -> slot and
  // multiplicity per edge id (in the second workspace), filled by pass 0
  uint64_t Ws = W;                      // slots of the rows the pipeline runs on
  uint32_t* mult2 = nullptr;
  uint32_t* smap = nullptr;
  uint32_t* mu = nullptr;
  Counters hc;
  uint32_t m32 = 0;
  uint32_t hist[34] = {};
  unsigned long long hist_slots[34] = {};
  for (int pass = 0;; ++pass) {
    CU(cudaMemsetAsync(hub_hist, 0, 4 * 34 + 8 * 34, s));
    k_hub_hist<<<grid_for(N, 256, E.sm_count * 4), 256, 0, s>>>(J.off, N, hub_hist, hub_hist_slots);
    J.launches += 1;
    // rows orientation and compaction give a block each (listed by original degree)
    CU(cudaMemsetAsync(&cnt->big_count, 0, 4, s));
    k_big_rows<<<grid_for(N, 256, E.sm_count * 8), 256, 0, s>>>(J.off, N, big, &cnt->big_count);
    k_orient_count<<<vgrid, 256, 0, s>>>(J.off, J.nbr, N, dplus, &cnt->self_loops, err, &cnt->max_dplus, big,
                                         &cnt->big_count);
    J.launches += 1;
    exclusive_scan<uint32_t>(LoadU32{dplus}, N, opos, at<uint32_t>(E, L.tiles), (uint32_t*)&cnt->grand, s);
    J.launches += 4;
    CU(cudaMemcpyAsync(dmem, J.members.data(), sizeof(Member) * G, cudaMemcpyHostToDevice, s));
    k_member_edges<<<grid_for(G, 256, 1024), 256, 0, s>>>(dmem, G, opos);
    J.launches += 1;
    CU(cudaMemcpyAsync(J.members.data(), dmem, sizeof(Member) * G, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(&hc, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(&m32, opos + N, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(hist, hub_hist, 4 * 34, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(hist_slots, hub_hist_slots, 8 * 34, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (pass == 0) J.slot_self_loops = hc.self_loops;
    // (batched unions: the packer counted the relabelled copy in their budget)
    if (pass == 0 && hc.err == 0 && N > 1 && W > 0 && !J.support_only && !J.prep_only && !J.hook &&
        resolve_tuning(tune_key(hist, hist_slots, W)).relabel) {
      // a sound simple graph: orient its degree-ordered copy instead (when the
      // device has no room for the copy, the caller's ids are used as they are)
      int rc = relabel_graph(E, J, N, W, big, &cnt->big_count, s);
      if (rc == SPARX_E_OOM) break;
      if (rc) return rc;
      smap = const_cast<uint32_t*>(J.smap);
      // the next pass counts them again
      CU(cudaMemsetAsync(&cnt->self_loops, 0, 8, s));
      CU(cudaMemsetAsync(&cnt->max_dplus, 0, 4, s));
      continue;
    }
    if (pass > 0 || hc.err != kErrMulti) break;
    // parallel edges and no other defect: reduce every row to its distinct
    // neighbours (copies per slot, caller slot -> slot), then orient again
    J.multi = true;
    const uint64_t Mx = std::max<uint64_t>(W / 2, 1);
    const size_t o_off = 0, o_nbr = align_up(4 * (N + 1)), o_mult = o_nbr + align_up(4 * W),
                 o_smap = o_mult + align_up(4 * W), o_mu = o_smap + align_up(4 * W), total = o_mu + align_up(4 * Mx);
    int rc = ensure_ws2(E, total);
    if (rc) return rc;
    uint32_t* off2 = (uint32_t*)(E.ws2 + o_off);
    uint32_t* nbr2 = (uint32_t*)(E.ws2 + o_nbr);
    mult2 = (uint32_t*)(E.ws2 + o_mult);
    smap = (uint32_t*)(E.ws2 + o_smap);
    mu = (uint32_t*)(E.ws2 + o_mu);
    const int wgrid = grid_for(32ull * N, 256, E.sm_count * 16);  // a warp per row
    k_dedupe_count<<<wgrid, 256, 0, s>>>(J.off, J.nbr, N, dplus);
    exclusive_scan<uint32_t>(LoadU32{dplus}, N, off2, at<uint32_t>(E, L.tiles), (uint32_t*)&cnt->grand, s);
    CU(cudaMemsetAsync(mult2, 0, 4 * std::max<uint64_t>(W, 1), s));
    CU(cudaMemsetAsync(err, 0, 4, s));
    CU(cudaMemsetAsync(&cnt->self_loops, 0, 8, s));
    CU(cudaMemsetAsync(&cnt->max_dplus, 0, 4, s));
    k_dedupe_fill<<<wgrid, 256, 0, s>>>(J.off, J.nbr, N, off2, nbr2, mult2, smap, err);
    J.launches += 6;
    uint32_t ws32 = 0;
    CU(cudaMemcpyAsync(&ws32, off2 + N, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    Ws = ws32;
    J.off = off2;
    J.nbr = nbr2;
    J.smap = smap;
  }
  J.self_loops = hc.self_loops;
  if (hc.err) { J.err = hc.err; return status_from_flags(hc.err); }
  const uint64_t m = m32;
  if (2 * m + hc.self_loops != Ws) { J.err = kErrAsym; return SPARX_E_INVALID_CSR; }
  for (const Member& M : J.members)
    if (M.m > kEidMask) { set_error("a graph has >= 2^28 edges"); return SPARX_E_TOO_LARGE; }
  {
    uint32_t* owner = at<uint32_t>(E, L.q0);  // in-slot owners; the q buffers are idle until the peel
    k_orient_fill<<<vgrid, 256, 0, s>>>(J.off, J.nbr, N, opos, ocol, osrc, row0, owner, big, &cnt->big_count);
    k_orient_reverse<<<grid_for(Ws, 256, E.sm_count * 16), 256, 0, s>>>(J.nbr, owner, Ws, opos, ocol, row0, err);
    if (J.multi) {
      // multiplicity per edge id from its out-slot; the in-slot must agree
      k_mult_out<<<grid_for(Ws, 256, E.sm_count * 16), 256, 0, s>>>(row0, owner, mult2, Ws, mu);
      k_mult_check<<<grid_for(Ws, 256, E.sm_count * 16), 256, 0, s>>>(row0, owner, mult2, Ws, mu, err);
      J.launches += 2;
      uint32_t* herr = (uint32_t*)E.pinned_small;
      CU(cudaMemcpyAsync(herr, err, 4, cudaMemcpyDeviceToHost, s));
      CU(cudaStreamSynchronize(s));
      if (*herr) { J.err = *herr; return status_from_flags(*herr); }
    }
  }
  J.launches += 2;
  // hub maps: the smallest power-of-two degree bound (>= kHubMinDegree) whose
  // vertices fit the reserved maps; hist[b] counts degrees in [2^(b-1), 2^b)
  const Tuning T = resolve_tuning(tune_key(hist, hist_slots, Ws));
  J.tuning = T;
  uint32_t hubs = 0, hub_min_deg = 0;
  if (hubs_possible && T.hub_min_degree) {
    uint64_t above = 0;
    const uint64_t floor_deg = std::max<uint32_t>(T.hub_min_degree, kHubFloor);
    for (int b = 32; b >= 1; --b) {
      const uint64_t lo = 1ull << (b - 1);
      if (lo < floor_deg || above + hist[b] > L.hub_cap) break;
      above += hist[b];
      hub_min_deg = (uint32_t)lo;
    }
    hubs = (uint32_t)above;
  }
  const uint32_t* d_hub_slot = nullptr;
  const uint32_t* d_hub_map = nullptr;
  const uint32_t* d_hub_base = nullptr;
  if (hubs) {
    uint32_t* hslot = at<uint32_t>(E, L.hub_slot);
    uint32_t* hvert = at<uint32_t>(E, L.hub_vertex);
    uint32_t* hbase = at<uint32_t>(E, L.hub_base);
    uint32_t* hmap = at<uint32_t>(E, L.hub_map);
    uint64_t max_n = 0;
    for (const Member& M : J.members) max_n = std::max<uint64_t>(max_n, M.n);
    CU(cudaMemsetAsync(&cnt->hub_count, 0, 4, s));
    k_hub_assign<<<grid_for(N, 256, E.sm_count * 8), 256, 0, s>>>(J.off, N, hub_min_deg, hubs, hslot, hvert,
                                                                  &cnt->hub_count);
    k_hub_layout<<<1, 1024, 0, s>>>(hvert, hubs, dmem, G, L.hub_pool, hbase, hslot);
    CU(cudaMemsetAsync(hmap, 0xFF, 4ull * std::min<unsigned long long>(L.hub_pool, hubs * max_n), s));
    k_hub_fill<<<std::min<uint32_t>(hubs, E.sm_count * 8), 256, 0, s>>>(J.off, row0, hvert, hubs, hslot, hbase,
                                                                        hmap);
    J.launches += 3;
    d_hub_slot = hslot;
    d_hub_map = hmap;
    d_hub_base = hbase;
  }
  J.hubs = hubs;
  // row hash tables for the peel's per-lane search (tuned; in a served union
  // only when it takes no joins, since joining rows would have none) and
  // out-list hash tables for the support pass (tuned)
  unsigned long long* hpool = nullptr;
  unsigned long long* spool = nullptr;
  uint2* qh0 = nullptr;
  uint2* qh1 = nullptr;
  uint32_t hash_min = 0, sup_hash_min = 0;
  // Both are optional: when their workspace does not fit the launch's budget
  // or cannot be allocated, the launch runs without them (same results).
  {
    bool peel_hash = T.hash_min_degree && !J.support_only && !J.prep_only && (!J.hook || J.hook_hash) &&
                     Ws < (1ull << 30) && Ws;
    bool sup_hash = T.sup_hash_min && m > 0 && m < (1ull << 28);
    const uint64_t Mx = std::max<uint64_t>(W / 2, 1);
    size_t pool_b = peel_hash ? align_up(32ull * Ws) : 0, qh_b = peel_hash ? align_up(8ull * Mx) : 0;
    size_t spool_b = sup_hash ? align_up(32ull * m) : 0;
    // rows with tables past a warp's shared slice (more than kTableSmem / 2
    // entries) are listed for the block-per-row fill: at most W / 512 rows
    const size_t big_b = align_up(4ull * (W / (kTableSmem / 2) + 2));
    if ((peel_hash || sup_hash) &&
        ((J.budget && L.total + pool_b + 2 * qh_b + spool_b + big_b > J.budget) ||
         ensure_ws3(E, pool_b + 2 * qh_b + spool_b + big_b) != SPARX_OK)) {
      peel_hash = sup_hash = false;
      pool_b = qh_b = spool_b = 0;
    }
    uint32_t* big_list = (uint32_t*)(E.ws3 + pool_b + 2 * qh_b + spool_b);
    uint32_t* big_count = &cnt->table_big;
    if (peel_hash) {
      hpool = (unsigned long long*)E.ws3;
      qh0 = (uint2*)(E.ws3 + pool_b);
      qh1 = (uint2*)(E.ws3 + pool_b + qh_b);
      hash_min = T.hash_min_degree;
      CU(cudaMemsetAsync(big_count, 0, 4, s));
      k_table_fill<<<grid_for(N, kTableWarps * 32, E.sm_count * 16), kTableWarps * 32, 0, s>>>(
          J.off, N, hash_min, d_hub_slot, RowPairSource{row0}, hpool, big_list, big_count);
      k_table_fill_big<<<E.sm_count * 8, 256, 0, s>>>(J.off, big_list, big_count, RowPairSource{row0}, hpool);
      J.launches += 2;
    }
    if (sup_hash) {
      spool = (unsigned long long*)(E.ws3 + pool_b + 2 * qh_b);
      sup_hash_min = T.sup_hash_min;
      CU(cudaMemsetAsync(big_count, 0, 4, s));
      k_table_fill<<<grid_for(N, kTableWarps * 32, E.sm_count * 16), kTableWarps * 32, 0, s>>>(
          opos, N, sup_hash_min, nullptr, OutListSource{ocol}, spool, big_list, big_count);
      k_table_fill_big<<<E.sm_count * 8, 256, 0, s>>>(opos, big_list, big_count, OutListSource{ocol}, spool);
      J.launches += 2;
    }
  }
  CU(cudaEventRecord(E.tev[2], s));

  // -- support (Kernel C) --
  CU(cudaMemsetAsync(es, 0, 8 * std::max<uint64_t>(m, 1), s));
  {
    int rc = launch_support(E.sm_count, O.support_kernel ? O.support_kernel : T.support_kernel, N, m,
                            hc.max_dplus, opos, ocol, osrc, es, at<unsigned long long>(E, L.q0),
                            at<unsigned long long>(E, L.tiles), cnt, at<uint32_t>(E, L.act0), s, &J.launches,
                            &J.support_elements, mu, T.sample_min, spool, sup_hash_min);
    if (rc) return rc;
  }
  CU(cudaEventRecord(E.tev[3], s));

  if (J.prep_only) {
    J.prep_m = m;
    J.prep_Ws = Ws;
    CU(cudaStreamSynchronize(s));
    return J.multi ? SPARX_E_MULTIGRAPH : SPARX_OK;
  }
  if (J.support_only && J.clustering) {
    k_clustering<<<vgrid, 256, 0, s>>>(J.off, row0, es, N, O.support_mode == SPARX_SUPPORT_U8, (double*)J.out,
                                       &cnt->cc_possible, &cnt->cc_local, &cnt->cc_slots, mult2);
    J.launches += 1;
    CU(cudaEventRecord(E.tev[4], s));
    CU(cudaEventRecord(E.tev[5], s));
  } else if (J.support_only) {
    k_support_slots<<<grid_for(W, 256, E.sm_count * 16), 256, 0, s>>>(row0, es, W, J.support_out,
                                                                       O.support_mode == SPARX_SUPPORT_U8, smap);
    J.launches += 1;
    CU(cudaEventRecord(E.tev[4], s));
    CU(cudaEventRecord(E.tev[5], s));
  } else {
    // -- peel (Kernel D) --
    Union U{};
    U.off = J.off;
    U.row = row0;
    U.opos = opos;
    U.ocol = ocol;
    U.osrc = osrc;
    U.es = es;
    U.act[0] = at<uint32_t>(E, L.act0);
    U.act[1] = at<uint32_t>(E, L.act1);
    U.q[0] = at<unsigned long long>(E, L.q0);
    U.q[1] = at<unsigned long long>(E, L.q1);
    U.qd[0] = at<uint4>(E, L.qd0);
    U.qd[1] = at<uint4>(E, L.qd1);
    U.hub_slot = d_hub_slot;
    U.hub_map = d_hub_map;
    U.hub_base = d_hub_base;
    U.hpool = hpool;
    U.off0 = J.off;
    U.qh[0] = qh0;
    U.qh[1] = qh1;
    U.hash_min = hash_min;
    U.vinfo = nullptr;
    if (d_hub_slot || hash_min) {
      unsigned long long* vinfo = at<unsigned long long>(E, L.vinfo);
      k_vinfo<<<grid_for(N, 256, E.sm_count * 16), 256, 0, s>>>(N, d_hub_slot, d_hub_base, J.off, hash_min, vinfo);
      J.launches += 1;
      U.vinfo = vinfo;
    }
    U.n = N;
    U.m = (uint32_t)m;
    U.width = (uint32_t)W;
    U.G = G;
    CU(cudaMemcpyAsync(at<Union>(E, L.uni), &U, sizeof(Union), cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(at<unsigned long long>(E, L.mem_tri), 0, 8ull * G, s));
    CU(cudaMemsetAsync(at<uint32_t>(E, L.mem_maxsup), 0, 4ull * G, s));
    Control c0{};
    c0.G = G;
    c0.max_waves = 3ull * m + 64;  // each frontier wave processes >= 1 edge; <= 2 scans per level
    c0.timeout_ns = O.timeout_ms * 1000000ull;
    c0.csr_slots = Ws;
    c0.compact_min = kCompactMinSlots;
    c0.compact_pct = T.compact_pct;
    if (J.hook) {
      c0.notify_done = 1;
      c0.admit = J.hook->admit_dev;
    }
    // wave trace: when SPARX_TRACE_FILE names a file, the planner records
    // each wave's start time and work there (first 2^20 waves)
    const char* trace_path = std::getenv("SPARX_TRACE_FILE");
    if (trace_path && *trace_path) {
      if (!E.trace) CU(cudaMalloc(&E.trace, kTraceRecords * sizeof(ulonglong4)));
      c0.trace = E.trace;
      c0.trace_cap = kTraceRecords;
    }
    CU(cudaMemcpyAsync(at<Control>(E, L.ctl), &c0, sizeof(Control), cudaMemcpyHostToDevice, s));
    if (m > 0)
      k_peel_setup<<<grid_for(m, 256, E.sm_count * 8), 256, 0, s>>>(at<Union>(E, L.uni), dmem,
                                                                     O.support_mode == SPARX_SUPPORT_U8,
                                                                     at<unsigned long long>(E, L.mem_tri),
                                                                     at<uint32_t>(E, L.mem_maxsup), mu, err);
    k_peel_init<<<1, 1024, 0, s>>>(dmem, at<MemberState>(E, L.st), at<Control>(E, L.ctl),
                                   at<unsigned long long>(E, L.wpref), G);
    J.launches += m > 0 ? 2 : 1;
    CU(cudaEventRecord(E.tev[4], s));
    WaveArgs wa;
    wa.Up = at<Union>(E, L.uni);
    wa.arr = peel_arrays(U);
    wa.arr.mu = mu;
    wa.arr.merge_ratio = T.merge_ratio;
    if (J.hook) wa.arr.n = 0;  // unused by the kernels; a constant keeps the graph across joins
    wa.mem = dmem;
    wa.st = at<MemberState>(E, L.st);
    wa.ctl = at<Control>(E, L.ctl);
    wa.wpref = at<unsigned long long>(E, L.wpref);
    wa.err = err;
    wa.handle = cudaGraphConditionalHandle{};
    wa.use_handle = 0;
    Control* hctl = (Control*)E.pinned_small;
    const uint32_t* cur_off = J.off;
    const unsigned long long* cur_row = row0;
    int next_buf = 0;
    // counts a served union's joins change (the rest of the pipeline is done)
    uint32_t pN = N, pG = G;
    uint64_t pm = m, pWs = Ws;
    auto serve_stop = [&](uint32_t reason, bool* resume) -> int {
      PeelCtx ctx;
      ctx.U = U;
      ctx.U.off = cur_off;
      ctx.U.row = cur_row;
      ctx.cur_off = cur_off;
      ctx.cur_row = cur_row;
      ctx.csr_slots = hctl->csr_slots;
      ctx.m = pm;
      ctx.Ws = pWs;
      ctx.N = pN;
      ctx.G = pG;
      ctx.waves_run = hctl->waves_run;
      int rc = J.hook->at_stop(E, J, ctx, reason, s);
      if (rc) return rc;
      U = ctx.U;
      pm = ctx.m;
      pWs = ctx.Ws;
      pN = ctx.N;
      pG = ctx.G;
      *resume = ctx.resume;
      return SPARX_OK;
    };
    for (;;) {
      if (O.loop == SPARX_LOOP_GRAPH) {
        int rc = build_peel_graph(E, J, wa.arr);
        if (rc) return rc;
        CU(cudaGraphLaunch(E.peel.exec, s));
        CU(cudaMemcpyAsync(hctl, wa.ctl, sizeof(Control), cudaMemcpyDeviceToHost, s));
        CU(cudaStreamSynchronize(s));
      } else {
        for (;;) {
          for (int i = 0; i < 16; ++i) {
            if (mu) k_wave<true><<<E.wave_blocks_multi, 256, 0, s>>>(wa);
            else k_wave<false><<<E.wave_blocks, 256, 0, s>>>(wa);
          }
          J.launches += 16;
          CU(cudaMemcpyAsync(hctl, wa.ctl, sizeof(Control), cudaMemcpyDeviceToHost, s));
          CU(cudaStreamSynchronize(s));
          if (hctl->done) break;
        }
      }
      if (J.hook && hctl->exit_reason != kExitCompact && hctl->exit_reason != kExitError) {
        bool resume = false;
        const int r = serve_stop(hctl->exit_reason, &resume);
        if (r) return r;
        if (!resume) break;
        k_replan<<<1, 1024, 0, s>>>(dmem, at<MemberState>(E, L.st), wa.ctl, wa.wpref);
        J.launches += 1;
        continue;
      }
      if (hctl->exit_reason != kExitCompact) break;
      // drop processed edges from the working rows, then resume the loop
      uint32_t* off2 = at<uint32_t>(E, next_buf ? L.offB : L.offA);
      unsigned long long* row2 = at<unsigned long long>(E, next_buf ? L.rowB : L.rowA);
      uint32_t* alive = at<uint32_t>(E, L.alive);
      const int pvgrid = grid_for(pN, 256, E.sm_count * 32);
      k_compact_mark<<<grid_for((pm + 31) / 32 * 32ull, 256, E.sm_count * 16), 256, 0, s>>>(es, (uint32_t)pm,
                                                                                           wa.ctl, alive);
      k_compact_count<<<pvgrid, 256, 0, s>>>(cur_off, cur_row, pN, alive, dplus, J.off);
      k_compact_count_big<<<E.sm_count * 2, 1024, 0, s>>>(cur_off, cur_row, alive, dplus, big, &cnt->big_count);
      exclusive_scan<uint32_t>(LoadU32{dplus}, pN, off2, at<uint32_t>(E, L.tiles), (uint32_t*)&cnt->grand, s);
      k_compact_fill<<<pvgrid, 256, 0, s>>>(cur_off, cur_row, pN, alive, off2, row2, J.off);
      k_compact_fill_big<<<E.sm_count * 2, 1024, 0, s>>>(cur_off, cur_row, alive, off2, row2, big,
                                                         &cnt->big_count);
      k_compact_commit<<<1, 1, 0, s>>>(at<Union>(E, L.uni), off2, row2, off2 + pN, wa.ctl);
      const uint32_t per = std::max<uint32_t>(1, (uint32_t)(E.sm_count * 8) / std::max<uint32_t>(pG, 1));
      k_refresh_desc<<<pG * per, 256, 0, s>>>(wa.Up, dmem, wa.st, pG, per);
      J.launches += 8;
      cur_off = off2;
      cur_row = row2;
      U.off = off2;
      U.row = row2;
      next_buf ^= 1;
    }
    if (J.hook) {
      // every member went out through the hook
      CU(cudaEventRecord(E.tev[5], s));
      CU(cudaEventRecord(E.tev[6], s));
      CU(cudaMemcpyAsync(&hc, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, s));
      CU(cudaStreamSynchronize(s));
      J.err = hc.err;
      return status_from_flags(hc.err);
    }
    CU(cudaEventRecord(E.tev[5], s));
    // -- finalize (Kernel E) --
    const int fgrid = grid_for(W, 256, E.sm_count * 16);
    const int u8 = O.support_mode == SPARX_SUPPORT_U8;
    if (W > 0) {
      if (O.out_bits == 8)
        k_finalize<uint8_t><<<fgrid, 256, 0, s>>>(row0, es, W, (uint8_t*)J.out, u8, 1, &cnt->kmax, err, smap);
      else
        k_finalize<uint32_t><<<fgrid, 256, 0, s>>>(row0, es, W, (uint32_t*)J.out, u8, 0, &cnt->kmax, err, smap);
      J.launches += 1;
    }
  }
  CU(cudaEventRecord(E.tev[6], s));
  // read back
  J.states.resize(G);
  J.mem_tri.resize(G);
  J.mem_maxsup.resize(G);
  if (!J.support_only) {
    CU(cudaMemcpyAsync(J.states.data(), at<MemberState>(E, L.st), sizeof(MemberState) * G, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(J.mem_tri.data(), at<unsigned long long>(E, L.mem_tri), 8ull * G, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(J.mem_maxsup.data(), at<uint32_t>(E, L.mem_maxsup), 4ull * G, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(&J.ctl, at<Control>(E, L.ctl), sizeof(Control), cudaMemcpyDeviceToHost, s));
  }
  CU(cudaMemcpyAsync(&hc, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  J.tri = hc.tri;
  J.kmax = hc.kmax;
  J.cc_possible = hc.cc_possible;
  J.cc_local = hc.cc_local;
  J.cc_slots = hc.cc_slots;
  if (!J.support_only && J.ctl.trace) {
    const char* trace_path = std::getenv("SPARX_TRACE_FILE");
    const size_t nrec = (size_t)std::min<unsigned long long>(J.ctl.waves_run, J.ctl.trace_cap);
    std::vector<ulonglong4> rec(nrec);
    if (nrec) CU(cudaMemcpy(rec.data(), J.ctl.trace, nrec * sizeof(ulonglong4), cudaMemcpyDeviceToHost));
    if (FILE* f = std::fopen(trace_path, "w")) {
      std::fprintf(f, "wave,t_ns,work,frontier_elements,scan_elements\n");
      for (size_t i = 0; i < nrec; ++i)
        std::fprintf(f, "%zu,%llu,%llu,%llu,%llu\n", i + 1, rec[i].x, rec[i].y, rec[i].z, rec[i].w);
      std::fclose(f);
    }
  }
  // each WHILE-loop iteration is one wave kernel (its last block plans)
  if (!J.support_only && O.loop == SPARX_LOOP_GRAPH)
    J.launches += (uint32_t)std::max<unsigned long long>(J.ctl.waves_run, 1);
  J.err = hc.err;
  CU(cudaEventElapsedTime(&J.ms_orient, E.tev[1], E.tev[2]));
  CU(cudaEventElapsedTime(&J.ms_support, E.tev[2], E.tev[3]));
  CU(cudaEventElapsedTime(&J.ms_peel, E.tev[4], E.tev[5]));
  CU(cudaEventElapsedTime(&J.ms_finalize, E.tev[5], E.tev[6]));
  CU(cudaGetLastError());
  return status_from_flags(hc.err);
}

void fill_stats(const UnionJob& J, uint32_t g, sparx_pkt_stats* st) {
  if (!st) return;
  std::memset(st, 0, sizeof(*st));
  const Member& M = J.members[g];
  st->n = M.n;
  st->width = M.w;
  st->m = M.m;
  // a multigraph's width also counts parallel copies: its self-loop slots were
  // counted before the rows were deduplicated (for a lone graph; not split per
  // member in a batch)
  st->self_loops = !J.multi ? M.w - 2ull * M.m : J.members.size() == 1 ? J.slot_self_loops : 0;
  if (g < J.mem_tri.size()) st->triangles = J.mem_tri[g] / 3;
  if (g < J.mem_maxsup.size()) st->max_support = J.mem_maxsup[g];
  if (g < J.states.size() && !J.support_only) {  // support-only runs have no peel state
    st->levels = J.states[g].levels;
    st->waves = J.states[g].waves;
    st->k_max = M.w ? J.states[g].max_level + 2 : 0;
  }
  if (J.members.size() == 1 && J.support_only) st->triangles = J.tri;
  if (J.kcore) {
    st->m = 0;
    st->self_loops = 0;
    st->levels = J.kc_levels;
    st->waves = J.kc_waves;
    st->k_max = J.kc_max;
  }
  st->launches = J.launches;
  st->support_elements = J.support_elements;
  if (J.members.size() == 1) {
    st->peel_elements = J.ctl.el_proc;
    st->peel_hits = J.ctl.hits;
    st->peel_scanned = J.ctl.el_scan;
    st->peel_edges = J.ctl.edges_proc;
    st->compactions = J.ctl.compactions;
    st->hub_maps = J.hubs;
    st->merge_iters = J.ctl.merge_iters;
    st->lane_iters = J.ctl.lane_iters;
    st->merge_chunks = J.ctl.merge_chunks;
  }
  st->ms_orient = J.ms_orient;
  st->ms_support = J.ms_support;
  st->ms_peel = J.ms_peel;
  st->ms_finalize = J.ms_finalize;
}

int check_dims(uint64_t n_plus_1, uint64_t width) {
  if (n_plus_1 < 1) { set_error("n_plus_1 must be >= 1"); return SPARX_E_ARG; }
  if (n_plus_1 - 1 >= 0xFFFFFFFFull || width >= 0xFFFFFFFFull) {
    set_error("n or width does not fit 32 bits");
    return SPARX_E_TOO_LARGE;
  }
  return SPARX_OK;
}

// k-core workspace: the uploaded CSR, degree, live flag, core and two
// frontier queues per vertex (Layout fields reused by name).
Layout make_kcore_layout(uint64_t N, uint64_t W, size_t out_bytes) {
  Layout L{};
  size_t p = 0;
  auto take = [&](size_t bytes) {
    size_t r = p;
    p = align_up(p + std::max<size_t>(bytes, 1));
    return r;
  };
  L.off = take(4 * (N + 1));
  L.nbr = take(4 * W);
  L.dplus = take(4 * N);  // degree
  L.act0 = take(4 * N);   // live flag
  L.opos = take(4 * N);   // core
  L.q0 = take(4 * N);     // frontier
  L.q1 = take(4 * N);     // next frontier
  L.out = take(out_bytes);
  L.stage0 = take(kStageBytes);
  L.stage1 = take(kStageBytes);
  L.cnt = take(sizeof(Counters));
  L.tiles = take(256);    // the level loop's state (KcState)
  L.total = p;
  return L;
}

// Level loop of the k-core peel (liu_et_al.rs:295-420) on the device: a CUDA
// graph whose WHILE node runs k_kcore_wave four times per iteration (the last
// block of each wave plans the next and sets the condition), or host-launched
// waves with SPARX_LOOP_HOST.
int run_kcore(Engine& E, UnionJob& J, const Opts& O, cudaStream_t s) {
  const Layout& L = J.L;
  const uint32_t N = (uint32_t)J.N;
  Counters* cnt = at<Counters>(E, L.cnt);
  {
    uint32_t* herr = (uint32_t*)E.pinned_small;
    CU(cudaMemcpyAsync(herr, &cnt->err, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (*herr) { J.err = *herr; return status_from_flags(*herr); }
  }
  static_assert(sizeof(KcState) <= 256, "KcState fits its slot");
  uint32_t* deg = at<uint32_t>(E, L.dplus);
  uint32_t* alive = at<uint32_t>(E, L.act0);
  uint32_t* core = at<uint32_t>(E, L.opos);
  uint32_t* qa = at<uint32_t>(E, L.q0);
  uint32_t* qb = at<uint32_t>(E, L.q1);
  KcState* kst = at<KcState>(E, L.tiles);
  const int u8 = O.support_mode == SPARX_SUPPORT_U8;
  const int vgrid = grid_for(N, 256, E.sm_count * 16);
  CU(cudaMemsetAsync(kst, 0, sizeof(KcState), s));
  CU(cudaEventRecord(E.tev[1], s));
  k_kcore_init<<<vgrid, 256, 0, s>>>(J.off, N, u8, deg, alive, core, &kst->remaining);
  // every wave is a scan or a sub-level that peels >= 1 vertex; scans per level <= 2
  k_kcore_start<<<1, 1, 0, s>>>(kst, 3ull * N + 2 * J.W + 64, O.timeout_ms * 1000000ull);
  J.launches += 2;
  CU(cudaEventRecord(E.tev[4], s));
  const int wgrid = E.sm_count * 8;
  if (O.loop == SPARX_LOOP_GRAPH) {
    cudaGraph_t g;
    CU(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    CU(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    CU(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CU(cudaStreamBeginCaptureToGraph(E.capture, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    for (int i = 0; i < 4; ++i)
      k_kcore_wave<<<wgrid, 256, 0, E.capture>>>(J.off, J.nbr, N, deg, alive, core, qa, qb, kst, h, 1);
    cudaGraph_t captured;
    CU(cudaStreamEndCapture(E.capture, &captured));
    cudaGraphExec_t ex;
    cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
    if (ie != cudaSuccess) {
      cudaGraphDestroy(g);
      set_error(std::string("k-core graph: ") + cudaGetErrorString(ie));
      return SPARX_E_CUDA;
    }
    const cudaError_t le = cudaGraphLaunch(ex, s);
    const cudaError_t se = cudaStreamSynchronize(s);
    cudaGraphExecDestroy(ex);
    cudaGraphDestroy(g);
    if (le != cudaSuccess || se != cudaSuccess) {
      set_error(std::string("k-core loop: ") + cudaGetErrorString(le != cudaSuccess ? le : se));
      return SPARX_E_CUDA;
    }
  } else {
    KcState* h = (KcState*)E.pinned_small;
    for (;;) {
      for (int i = 0; i < 16; ++i)
        k_kcore_wave<<<wgrid, 256, 0, s>>>(J.off, J.nbr, N, deg, alive, core, qa, qb, kst,
                                           cudaGraphConditionalHandle{}, 0);
      J.launches += 16;
      CU(cudaMemcpyAsync(h, kst, sizeof(KcState), cudaMemcpyDeviceToHost, s));
      CU(cudaStreamSynchronize(s));
      if (h->phase == 2) break;
    }
  }
  CU(cudaEventRecord(E.tev[5], s));
  KcState hs;
  CU(cudaMemcpyAsync(&hs, kst, sizeof(KcState), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (O.loop == SPARX_LOOP_GRAPH) J.launches += (uint32_t)hs.waves_run;
  if (hs.err) {
    J.err = hs.err;
    set_error("k-core level loop stopped: " + std::string(hs.err & kErrTimeout ? "time budget" : "wave bound"));
    return status_from_flags(hs.err);
  }
  J.kc_levels = hs.levels;
  J.kc_waves = hs.subs;
  J.kc_max = hs.kmax;
  if (O.out_bits == 8 && J.kc_max > 255) {
    // the reference's u8 level counter overflows (liu_et_al.rs:335-343)
    set_error("a core number exceeds 255 with 8-bit output");
    J.err = kErrOverflowU8;
    return SPARX_E_OVERFLOW_U8;
  }
  if (N) {
    if (O.out_bits == 8) k_kcore_out<uint8_t><<<vgrid, 256, 0, s>>>(core, N, (uint8_t*)J.out);
    else k_kcore_out<uint32_t><<<vgrid, 256, 0, s>>>(core, N, (uint32_t*)J.out);
    J.launches += 1;
  }
  CU(cudaEventRecord(E.tev[6], s));
  CU(cudaEventRecord(E.tev[2], s));
  CU(cudaEventRecord(E.tev[3], s));
  CU(cudaStreamSynchronize(s));
  float ms = 0;
  CU(cudaEventElapsedTime(&ms, E.tev[4], E.tev[5]));
  J.ms_peel = ms;
  return SPARX_OK;
}

// Sums behind the clustering coefficients (out_host then holds one f64 local
// coefficient per vertex).
struct ClusterSums {
  double possible = 0, local = 0;
  unsigned long long slots = 0;
};

// Single graph from host memory (ids u64 or u32): truss per slot, support per
// slot (support_only) or local clustering coefficients (cc != nullptr).
int run_host(const uint64_t* offsets, uint64_t n_plus_1, const void* nbrs, int bits, uint64_t width,
             void* out_host, bool support_only, const sparx_pkt_opts* opts, sparx_pkt_stats* stats,
             ClusterSums* cc = nullptr, bool kcore = false) {
  g_last_error.clear();
  if (!offsets || (!nbrs && width) || (!out_host && width)) { set_error("null pointer"); return SPARX_E_ARG; }
  int rc = check_dims(n_plus_1, width);
  if (rc) return rc;
  Opts O;
  rc = read_opts(opts, &O);
  if (rc) return rc;
  Engine* Ep;
  rc = get_engine(O.device, &Ep);
  if (rc) return rc;
  Engine& E = *Ep;
  std::lock_guard<std::mutex> lk(E.mu);
  CU(cudaSetDevice(E.device));
  const uint64_t n = n_plus_1 - 1;
  UnionJob J;
  J.N = n;
  J.W = width;
  J.members.push_back(Member{0, (uint32_t)n, 0, (uint32_t)width, 0, 0});
  J.support_only = support_only || cc;
  J.clustering = cc != nullptr;
  J.kcore = kcore;
  support_only = J.support_only;
  const size_t out_bytes = kcore ? (O.out_bits / 8) * n
                           : J.clustering ? 8 * n : support_only ? 4 * width : (O.out_bits / 8) * width;
  J.L = kcore ? make_kcore_layout(n, width, out_bytes) : make_layout(n, width, 1, true, out_bytes);
  rc = ensure_ws(E, J.L.total);
  if (rc) return rc;
  cudaStream_t s = E.stream;
  J.off = at<uint32_t>(E, J.L.off);
  J.nbr = at<uint32_t>(E, J.L.nbr);
  if (support_only && !J.clustering) J.support_out = at<uint32_t>(E, J.L.out);
  else J.out = at<void>(E, J.L.out);
  char* stage[2] = {E.ws + J.L.stage0, E.ws + J.L.stage1};
  Counters* cnt = at<Counters>(E, J.L.cnt);
  auto t0 = std::chrono::steady_clock::now();
  CU(cudaMemsetAsync(cnt, 0, sizeof(Counters), s));
  CU(cudaEventRecord(E.tev[0], s));
  bool bad_host = false;
  {
    // offsets: stage -> narrow (one chunk suffices below 8M vertices; larger
    // offset arrays go through the same double-buffered loop)
    const uint64_t chunk = kStageBytes / 8;
    bad_host = offsets[0] != 0 || offsets[n] != width;
    for (uint64_t c = 0, a = 0; a < n_plus_1; ++c, a += chunk) {
      const int slot = (int)(c & 1);
      const uint64_t k = std::min<uint64_t>(chunk, n_plus_1 - a);
      if (a > 0 && offsets[a] < offsets[a - 1]) bad_host = true;
      CU(cudaEventSynchronize(E.pin_ev[slot]));
      parallel_copy(E.pinned[slot], offsets + a, k * 8);
      CU(cudaMemcpyAsync(stage[slot], E.pinned[slot], k * 8, cudaMemcpyHostToDevice, s));
      k_narrow_offsets<<<grid_for(k, 256, E.sm_count * 16), 256, 0, s>>>(
          (const unsigned long long*)stage[slot], J.off + a, (uint32_t)k, 0u, -1ll, -1ll, &cnt->err);
      CU(cudaEventRecord(E.pin_ev[slot], s));
    }
  }
  if (bad_host) { set_error("offsets: first must be 0, last must equal width, non-decreasing"); return SPARX_E_INVALID_CSR; }
  rc = upload_ids(E, nbrs, bits, width, (uint32_t*)J.nbr, n, 0, s, stage, &cnt->err);
  if (rc) return rc;
  // one narrowing kernel per offsets chunk (the ids are narrowed by the host)
  J.launches += (uint32_t)((n_plus_1 + kStageBytes / 8 - 1) / (kStageBytes / 8));
  rc = kcore ? run_kcore(E, J, O, s) : run_union(E, J, O, s);
  if (rc) {
    fill_stats(J, 0, stats);
    return rc;
  }
  CU(cudaEventRecord(E.tev[7], s));
  if (cc) {
    cc->possible = J.cc_possible;
    cc->local = J.cc_local;
    cc->slots = J.cc_slots;
  }
  rc = download(E, out_host, (support_only && !J.clustering) ? (void*)J.support_out : J.out, out_bytes, s);
  if (rc) return rc;
  CU(cudaStreamSynchronize(s));
  auto t1 = std::chrono::steady_clock::now();
  fill_stats(J, 0, stats);
  if (stats) {
    float up = 0;
    cudaEventElapsedTime(&up, E.tev[0], E.tev[1]);
    stats->ms_upload = up;
    stats->ms_total = std::chrono::duration<double, std::milli>(t1 - t0).count();
    stats->ms_download = stats->ms_total - (up + J.ms_orient + J.ms_support + J.ms_peel + J.ms_finalize);
  }
  return SPARX_OK;
}

// ---------------------------------------------------------------------------
// Batched decomposition: independent graphs packed into unions.

struct HostMember {
  const uint64_t* off = nullptr;
  uint64_t n = 0;
  const void* nbr = nullptr;
  int bits = 64;
  uint64_t w = 0;
  void* out = nullptr;
  uint64_t index = 0;
};

inline uint64_t host_id(const HostMember& h, uint64_t i) {
  return h.bits == 64 ? ((const uint64_t*)h.nbr)[i] : ((const uint32_t*)h.nbr)[i];
}

// Host checks that need no device: offsets run from 0 to width without
// decreasing, ids < n.  Row order, duplicates and symmetry are checked on the
// device during orientation.
int host_validate(const HostMember& h) {
  if (h.off[0] != 0 || h.off[h.n] != h.w) return SPARX_E_INVALID_CSR;
  for (uint64_t v = 0; v < h.n; ++v)
    if (h.off[v + 1] < h.off[v]) return SPARX_E_INVALID_CSR;
  bool bad = false;
  if (h.w > (1u << 20)) {
#pragma omp parallel for schedule(static) reduction(|| : bad)
    for (long long i = 0; i < (long long)h.w; ++i) bad = bad || host_id(h, (uint64_t)i) >= h.n;
  } else {
    for (uint64_t i = 0; i < h.w && !bad; ++i) bad = host_id(h, i) >= h.n;
  }
  return bad ? SPARX_E_INVALID_CSR : SPARX_OK;
}

// Stream a union's u32 offsets and ids to the device through the pinned
// staging buffers: host threads narrow and shift each member's arrays into a
// chunk, which is then copied straight to its final place in HBM.
int upload_union(Engine& E, const std::vector<HostMember>& hm, const std::vector<Member>& mem, uint64_t N,
                 uint64_t W, uint32_t* d_off, uint32_t* d_nbr, cudaStream_t s) {
  const uint64_t chunk = kStageBytes / 4;
  for (int pass = 0; pass < 2; ++pass) {
    const uint64_t total = pass == 0 ? N + 1 : W;
    uint32_t* dst = pass == 0 ? d_off : d_nbr;
    size_t g0 = 0;  // first member that can overlap the chunk
    for (uint64_t c = 0, a = 0; a < total; ++c, a += chunk) {
      const int slot = (int)(c & 1);
      const uint64_t b = std::min<uint64_t>(a + chunk, total);
      CU(cudaEventSynchronize(E.pin_ev[slot]));
      uint32_t* buf = (uint32_t*)E.pinned[slot];
      auto lo_of = [&](const Member& M) -> uint64_t { return pass == 0 ? M.vb : M.sb; };
      auto len_of = [&](const Member& M) -> uint64_t { return pass == 0 ? M.n : M.w; };
      while (g0 < mem.size() && lo_of(mem[g0]) + len_of(mem[g0]) <= a) ++g0;
      // fixed-size pieces of the chunk, whatever members they cross: a large
      // member is narrowed by all threads, not by one
      constexpr uint64_t kPiece = 1ull << 18;
      const long long pieces = (long long)((b - a + kPiece - 1) / kPiece);
#pragma omp parallel for schedule(dynamic, 1)
      for (long long pi = 0; pi < pieces; ++pi) {
        const uint64_t lo = a + (uint64_t)pi * kPiece, hi = std::min<uint64_t>(b, lo + kPiece);
        // first member whose range reaches past lo
        size_t g = g0, gh = mem.size();
        while (g < gh) {
          const size_t mid = (g + gh) / 2;
          if (lo_of(mem[mid]) + len_of(mem[mid]) <= lo) g = mid + 1; else gh = mid;
        }
        for (uint64_t x = lo; x < hi;) {
          while (g < mem.size() && lo_of(mem[g]) + len_of(mem[g]) <= x) ++g;
          if (g >= mem.size()) break;
          const Member& M = mem[g];
          const HostMember& H = hm[g];
          const uint64_t end = std::min<uint64_t>(hi, lo_of(M) + len_of(M));
          if (pass == 0) {
            for (; x < end; ++x) buf[x - a] = (uint32_t)(H.off[x - M.vb] + M.sb);
          } else if (H.bits == 64) {
            const uint64_t* src = (const uint64_t*)H.nbr;
            for (; x < end; ++x) buf[x - a] = (uint32_t)src[x - M.sb] + M.vb;
          } else {
            const uint32_t* src = (const uint32_t*)H.nbr;
            for (; x < end; ++x) buf[x - a] = src[x - M.sb] + M.vb;
          }
        }
      }
      if (pass == 0 && b == total) buf[total - 1 - a] = (uint32_t)W;  // the closing offset
      CU(cudaMemcpyAsync(dst + a, buf, (b - a) * 4, cudaMemcpyHostToDevice, s));
      CU(cudaEventRecord(E.pin_ev[slot], s));
    }
  }
  return SPARX_OK;
}

// The union's per-slot results to each member's host buffer: pinned chunks
// (double-buffered against the copies), split into fixed pieces that all
// threads copy out, whatever members they cross.
int download_union(Engine& E, const std::vector<HostMember>& hm, const std::vector<Member>& mem, const void* dev,
                   size_t esz, cudaStream_t s) {
  uint64_t W = 0;
  for (const Member& M : mem) W = std::max<uint64_t>(W, (uint64_t)M.sb + M.w);
  if (!W) return SPARX_OK;
  const uint64_t chunk = kStageBytes / esz;
  const uint64_t nchunks = (W + chunk - 1) / chunk;
  auto issue = [&](uint64_t c) -> int {
    const int slot = (int)(c & 1);
    const uint64_t a = c * chunk, k = std::min<uint64_t>(chunk, W - a);
    CU(cudaMemcpyAsync(E.pinned[slot], (const char*)dev + a * esz, k * esz, cudaMemcpyDeviceToHost, s));
    CU(cudaEventRecord(E.pin_ev[slot], s));
    return SPARX_OK;
  };
  CU(cudaEventSynchronize(E.pin_ev[0]));
  CU(cudaEventSynchronize(E.pin_ev[1]));
  int rc = issue(0);
  if (rc) return rc;
  for (uint64_t c = 0; c < nchunks; ++c) {
    const int slot = (int)(c & 1);
    if (c + 1 < nchunks && (rc = issue(c + 1))) return rc;
    CU(cudaEventSynchronize(E.pin_ev[slot]));
    const uint64_t a = c * chunk, b = std::min<uint64_t>(W, a + chunk);
    const char* buf = (const char*)E.pinned[slot];
    constexpr uint64_t kPiece = 1ull << 18;
    const long long pieces = (long long)((b - a + kPiece - 1) / kPiece);
#pragma omp parallel for schedule(dynamic, 1)
    for (long long pi = 0; pi < pieces; ++pi) {
      const uint64_t lo = a + (uint64_t)pi * kPiece, hi = std::min<uint64_t>(b, lo + kPiece);
      size_t g = 0, gh = mem.size();
      while (g < gh) {
        const size_t mid = (g + gh) / 2;
        if ((uint64_t)mem[mid].sb + mem[mid].w <= lo) g = mid + 1; else gh = mid;
      }
      for (uint64_t x = lo; x < hi && g < mem.size(); ++g) {
        const Member& M = mem[g];
        if ((uint64_t)M.sb + M.w <= x) continue;
        const uint64_t end = std::min<uint64_t>(hi, (uint64_t)M.sb + M.w);
        std::memcpy((char*)hm[g].out + (x - M.sb) * esz, buf + (x - a) * esz, (end - x) * esz);
        x = end;
      }
    }
  }
  return SPARX_OK;
}

// Decompose one union of validated members; on a device-detected input error
// the members are re-run one by one to attribute the status.
int run_batch_union(Engine& E, std::vector<HostMember>& hm, const Opts& O, int* status_out,
                    sparx_pkt_stats* stats_out, int* first_fail, uint64_t budget = 0) {
  const size_t G = hm.size();
  UnionJob J;
  J.budget = budget;
  uint64_t N = 0, Wt = 0, max_n = 0;
  for (const HostMember& h : hm) {
    J.members.push_back(Member{(uint32_t)N, (uint32_t)h.n, (uint32_t)Wt, (uint32_t)h.w, 0, 0});
    N += h.n;
    Wt += h.w;
    max_n = std::max<uint64_t>(max_n, h.n);
  }
  J.N = N;
  J.W = Wt;
  const size_t out_bytes = (O.out_bits / 8) * Wt;
  J.L = make_layout(N, Wt, (uint32_t)G, true, out_bytes, max_n);
  int rc = ensure_ws(E, J.L.total);
  auto fail_all = [&](int code) {
    for (size_t g = 0; g < G; ++g) {
      if (status_out) status_out[hm[g].index] = code;
      if (!*first_fail) *first_fail = code;
    }
  };
  if (rc) { fail_all(rc); return rc; }
  cudaStream_t s = E.stream;
  J.off = at<uint32_t>(E, J.L.off);
  J.nbr = at<uint32_t>(E, J.L.nbr);
  J.out = at<void>(E, J.L.out);
  Counters* cnt = at<Counters>(E, J.L.cnt);
  auto t0 = std::chrono::steady_clock::now();
  CU(cudaMemsetAsync(cnt, 0, sizeof(Counters), s));
  CU(cudaEventRecord(E.tev[0], s));
  rc = upload_union(E, hm, J.members, N, Wt, J.off, (uint32_t*)J.nbr, s);
  if (rc) { fail_all(rc); return rc; }
  J.launches += 0;
  rc = run_union(E, J, O, s);
  if (rc == SPARX_E_INVALID_CSR || rc == SPARX_E_MULTIGRAPH || rc == SPARX_E_OVERFLOW_U8 ||
      rc == SPARX_E_TOO_LARGE) {
    if (G == 1) {
      fill_stats(J, 0, stats_out ? stats_out + hm[0].index : nullptr);
      if (status_out) status_out[hm[0].index] = rc;
      if (!*first_fail) *first_fail = rc;
      return rc;
    }
    // attribute: one member at a time
    for (size_t g = 0; g < G; ++g) {
      std::vector<HostMember> one{hm[g]};
      run_batch_union(E, one, O, status_out, stats_out, first_fail, budget);
    }
    return SPARX_OK;
  }
  if (rc) { fail_all(rc); return rc; }
  const size_t esz = O.out_bits / 8;
  // download the union's truss numbers straight into the members' buffers
  rc = G == 1 ? download(E, hm[0].out, J.out, out_bytes, s) : download_union(E, hm, J.members, J.out, esz, s);
  if (rc) { fail_all(rc); return rc; }
  CU(cudaStreamSynchronize(s));
  auto t1 = std::chrono::steady_clock::now();
  const double total_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
  for (size_t g = 0; g < G; ++g) {
    if (status_out) status_out[hm[g].index] = SPARX_OK;
    if (stats_out) {
      fill_stats(J, (uint32_t)g, stats_out + hm[g].index);
      stats_out[hm[g].index].ms_total = total_ms;  // the union's wall time, shared by its members
    }
  }
  return SPARX_OK;
}

// workspace of the peel's row hash tables for W slots (run_union's pool, the
// two queue descriptor arrays and the list of rows built a block each), and
// of the relabelled copy of N vertices' rows (relabel_graph, bounded above)
size_t table_bytes(uint64_t W) {
  return align_up(32ull * W) + 2 * align_up(8ull * std::max<uint64_t>(W / 2, 1)) +
         align_up(4ull * (W / (kTableSmem / 2) + 2));
}
size_t relabel_bytes(uint64_t N, uint64_t W) { return 8 * W + 30 * N + (64ull << 20); }
#ifndef SPARX_BATCH_FOR_TABLES
#define SPARX_BATCH_FOR_TABLES 1  // size batched unions so the row hash tables fit
#endif
constexpr bool kBatchForTables = SPARX_BATCH_FOR_TABLES;

int run_batch(const sparx_graph_view* graphs, uint64_t count, uint64_t budget, const sparx_pkt_opts* opts,
              int* status_out, sparx_pkt_stats* stats_out) {
  g_last_error.clear();
  if (!graphs && count) { set_error("null graph list"); return SPARX_E_ARG; }
  Opts O;
  int rc = read_opts(opts, &O);
  if (rc) return rc;
  Engine* Ep;
  rc = get_engine(O.device, &Ep);
  if (rc) return rc;
  Engine& E = *Ep;
  std::lock_guard<std::mutex> lk(E.mu);
  CU(cudaSetDevice(E.device));
  if (!budget) budget = 150ull << 30;
  if (stats_out) std::memset(stats_out, 0, sizeof(sparx_pkt_stats) * count);
  int first_fail = SPARX_OK;
  // host validation, then greedy packing in input order
  std::vector<HostMember> valid;
  valid.reserve(count);
  for (uint64_t i = 0; i < count; ++i) {
    const sparx_graph_view& v = graphs[i];
    HostMember h;
    h.off = v.offsets;
    h.n = v.n_plus_1 ? v.n_plus_1 - 1 : 0;
    h.nbr = v.neighbours;
    h.bits = v.neighbour_bits == 32 ? 32 : 64;
    h.w = v.width;
    h.out = v.truss_out;
    h.index = i;
    int st = SPARX_OK;
    if (!v.offsets || v.n_plus_1 < 1 || (v.width && (!v.neighbours || !v.truss_out)) ||
        (v.neighbour_bits != 32 && v.neighbour_bits != 64))
      st = SPARX_E_ARG;
    else if ((st = check_dims(v.n_plus_1, v.width)) == SPARX_OK)
      st = host_validate(h);
    if (st == SPARX_OK && h.w / 2 > kEidMask) st = SPARX_E_TOO_LARGE;
    if (status_out) status_out[i] = st;
    if (st != SPARX_OK) {
      if (!first_fail) first_fail = st;
      continue;
    }
    valid.push_back(h);
  }
  size_t at_i = 0;
  while (at_i < valid.size()) {
    std::vector<HostMember> wave;
    uint64_t N = 0, Wt = 0, max_n = 0;
    while (at_i < valid.size()) {
      const HostMember& h = valid[at_i];
      const uint64_t N2 = N + h.n, W2 = Wt + h.w, mx2 = std::max<uint64_t>(max_n, h.n);
      const size_t bytes =
          make_layout(N2, W2, (uint32_t)wave.size() + 1, true, (O.out_bits / 8) * W2, mx2).total;
      const bool fits = N2 < 0xFFFFFFFFull && W2 < 0xFFFFFFFFull && bytes <= budget && wave.size() < 65536;
      // a union grows only while its row hash tables fit as well (below 2^30
      // slots, and within the budget with them): on the mix the tables take
      // more off the peel than the extra unions' waves cost.  A graph too large
      // for that still runs, alone, without them.
      const bool fits_tables =
          fits && (!kBatchForTables ||
                   (W2 < (1ull << 30) && bytes + table_bytes(W2) + relabel_bytes(N2, W2) <= budget));
      if (!fits_tables && !wave.empty()) break;
      if (!fits) {  // a single graph over the budget
        if (status_out) status_out[h.index] = SPARX_E_OOM;
        if (!first_fail) first_fail = SPARX_E_OOM;
        ++at_i;
        continue;
      }
      wave.push_back(h);
      N = N2;
      Wt = W2;
      max_n = mx2;
      ++at_i;
    }
    if (!wave.empty()) run_batch_union(E, wave, O, status_out, stats_out, &first_fail, budget);
  }
  return first_fail;
}

// ---------------------------------------------------------------------------
// Serving: continuous batching over execution lanes.  Each lane is a private
// engine (stream, workspace, staging, cached peel graph) running one served
// union at a time: an idle lane packs the queued requests that fit its share
// of the HBM budget into a union with room to spare; while its peel runs,
// requests that arrive are admitted into it at the next wave boundary (the
// lane's planner stops when the host sets the lane's admission word; the
// newcomers are prepared -- narrowed, oriented, supported -- on the lane's
// second engine and joined behind the running members), and each member's
// truss numbers go back as soon as its own peel ends, not when the union's
// does.  Lanes run on separate streams, so their work overlaps on the GPU.

constexpr int kServerLanes = 4;                // default; SPARX_SERVE_LANES (1..16) overrides
constexpr uint32_t kServeMaxMembers = 4096;   // members per served union, joined ones included
// a union holding a member with more slots than this takes no joins: every
// member advances one step per wave, and such a member's waves would set the
// pace of small newcomers (R-MAT-24's waves take milliseconds)
constexpr uint64_t kJoinMaxMemberSlots = 1ull << 26;
// nor does a union whose waves, measured between its last two stops, take
// longer than this on average (a large member sets every member's pace; a
// union of small graphs runs at the ~15-25 us floor of a wave)
constexpr double kJoinMaxWaveUs = 60.0;

struct ServerReq {
  uint64_t ticket = 0;
  HostMember h;
  int status = SPARX_OK;
  bool running = false, done = false, cancelled = false;
  bool fresh_only = false;  // joining failed on the device: run in a fresh (unserved) union
  sparx_pkt_stats st{};
  std::chrono::steady_clock::time_point t_submit, t_start, t_done;
};

void engine_release(Engine* E) {
  if (!E) return;
  cudaSetDevice(E->device);
  if (E->stream) cudaStreamSynchronize(E->stream);
  if (E->peel.exec) { cudaGraphExecDestroy(E->peel.exec); cudaGraphDestroy(E->peel.graph); }
  if (E->ws) cudaFree(E->ws);
  if (E->ws2) cudaFree(E->ws2);
  if (E->ws3) cudaFree(E->ws3);
  if (E->trace) cudaFree(E->trace);
  for (int i = 0; i < 2; ++i) {
    if (E->pinned[i]) cudaFreeHost(E->pinned[i]);
    if (E->pin_ev[i]) cudaEventDestroy(E->pin_ev[i]);
  }
  for (auto& e : E->tev) if (e) cudaEventDestroy(e);
  if (E->pinned_small) cudaFreeHost(E->pinned_small);
  if (E->stream) cudaStreamDestroy(E->stream);
  if (E->capture) cudaStreamDestroy(E->capture);
  delete E;
}

}  // namespace

struct sparx_server {
  int device = 0;
  Opts O;
  std::vector<uint64_t> lane_budget;  // lane 0: half the budget (large graphs), the others a sixth
  std::vector<Engine*> lanes;         // runs the lane's unions
  std::vector<Engine*> prep;          // prepares the requests that join the lane's running union
  uint32_t* admit_host = nullptr;     // one mapped word per lane: requests wait to join
  uint32_t* admit_dev = nullptr;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<ServerReq*> queue;
  std::unordered_map<uint64_t, ServerReq*> reqs;
  uint64_t next_ticket = 1;
  bool stop = false;
  int nlanes = kServerLanes;
  int idle = 0;  // lanes waiting for work (a newcomer goes to one of them rather than joining)
  std::atomic<uint64_t> unions{0}, joined{0};  // served unions started; requests that joined one running
};

namespace {

void server_finish(sparx_server* S, ServerReq* r, int status) {
  r->status = status;
  r->done = true;
  r->running = false;
  r->t_done = std::chrono::steady_clock::now();
  r->st.ms_total = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
  (void)S;
}

uint64_t prep_budget(uint64_t lane_budget) { return lane_budget / 5; }

bool layout_fits(uint64_t N, uint64_t W, uint32_t G, size_t esz, uint64_t max_n, uint64_t budget) {
  return N < 0xFFFFFFFFull && W < 0xFFFFFFFFull && make_layout(N, W, G, true, esz * W, max_n).total <= budget;
}

// The lane's hook: delivers members as they finish and joins waiting requests.
struct LaneHook : ServeHook {
  sparx_server* S = nullptr;
  int lane = 0;
  Engine* P = nullptr;              // prepares joining requests
  std::vector<ServerReq*> reqs;     // per member of the union
  std::vector<char> delivered;
  uint64_t N_cap = 0, W_cap = 0;    // the union's room
  uint64_t max_n0 = 0;              // largest initial member (the hub pool was sized for it)
  uint64_t max_member_w = 0;        // slots of the union's largest member
  // the union's wave pace, measured between stops (host work at a stop excluded)
  std::chrono::steady_clock::time_point t_mark{};
  uint64_t w_mark = 0;
  bool marked = false;
  double wave_us = 0;

  int deliver(Engine& E, UnionJob& J, uint32_t G, cudaStream_t s) {
    const Layout& L = J.L;
    std::vector<MemberState> st(G);
    std::vector<unsigned long long> tri(G);
    std::vector<uint32_t> mx(G);
    CU(cudaMemcpyAsync(st.data(), at<MemberState>(E, L.st), sizeof(MemberState) * G, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(tri.data(), at<unsigned long long>(E, L.mem_tri), 8ull * G, cudaMemcpyDeviceToHost, s));
    CU(cudaMemcpyAsync(mx.data(), at<uint32_t>(E, L.mem_maxsup), 4ull * G, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    const size_t esz = S->O.out_bits / 8;
    const int u8 = S->O.support_mode == SPARX_SUPPORT_U8;
    Counters* cnt = at<Counters>(E, L.cnt);
    const unsigned long long* row0 = at<unsigned long long>(E, L.row0);
    const int2* es = at<int2>(E, L.es);
    for (uint32_t g = 0; g < G; ++g) {
      if (delivered[g] || st[g].phase != kPhaseDone) continue;
      const Member& M = J.members[g];
      uint32_t* ferr = &cnt->fin_err;
      CU(cudaMemsetAsync(ferr, 0, 4, s));
      char* out = (char*)J.out + (size_t)M.sb * esz;
      if (M.w) {
        // a deduplicated (multigraph) union maps the member's caller slots through smap
        const int fg = grid_for(M.w, 256, E.sm_count * 16);
        const unsigned long long* r0 = J.smap ? row0 : row0 + M.sb;
        const uint32_t* sm = J.smap ? J.smap + M.sb : nullptr;
        if (esz == 1)
          k_finalize<uint8_t><<<fg, 256, 0, s>>>(r0, es, M.w, (uint8_t*)out, u8, 1, &cnt->kmax, ferr, sm);
        else
          k_finalize<uint32_t><<<fg, 256, 0, s>>>(r0, es, M.w, (uint32_t*)out, u8, 0, &cnt->kmax, ferr, sm);
      }
      uint32_t* hferr = (uint32_t*)E.pinned_small;
      CU(cudaMemcpyAsync(hferr, ferr, 4, cudaMemcpyDeviceToHost, s));
      CU(cudaStreamSynchronize(s));
      const int status = status_from_flags(*hferr);
      ServerReq* r = reqs[g];
      if (!status && M.w) {
        int rc = download(E, r->h.out, out, (size_t)M.w * esz, s);
        if (rc) return rc;
        CU(cudaStreamSynchronize(s));
      }
      sparx_pkt_stats ps{};
      ps.n = M.n;
      ps.width = M.w;
      ps.m = M.m;
      ps.self_loops = M.w - 2ull * M.m;
      ps.triangles = tri[g] / 3;
      ps.max_support = mx[g];
      ps.k_max = M.w ? st[g].max_level + 2 : 0;
      ps.levels = st[g].levels;
      ps.waves = st[g].waves;
      delivered[g] = 1;
      {
        std::lock_guard<std::mutex> lk(S->mu);
        r->st = ps;
        server_finish(S, r, status);
      }
      S->cv_done.notify_all();
    }
    return SPARX_OK;
  }

  // Join the queued requests that fit; returns the number joined.
  int admit(Engine& E, UnionJob& J, PeelCtx& ctx, cudaStream_t s, uint32_t* joined) {
    *joined = 0;
    S->admit_host[lane] = 0;
    if (J.multi) return SPARX_OK;  // a deduplicated union has no room for more rows: wait for a lane
    if (max_member_w > kJoinMaxMemberSlots) return SPARX_OK;
    if (wave_us > kJoinMaxWaveUs) return SPARX_OK;  // its waves would set a newcomer's pace
    std::vector<ServerReq*> take;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      if (S->idle > 0) return SPARX_OK;  // an idle lane starts them at once, at their own pace
      // the largest lane drains (takes no joins) while a request only it can hold is waiting
      uint64_t other = 0;
      for (size_t i = 0; i < S->lane_budget.size(); ++i)
        if ((int)i != lane) other = std::max<uint64_t>(other, S->lane_budget[i] - prep_budget(S->lane_budget[i]));
      const uint64_t mine = S->lane_budget[lane] - prep_budget(S->lane_budget[lane]);
      if (other > 0 && mine > other)
        for (const ServerReq* r : S->queue)
          if (!layout_fits(r->h.n, r->h.w, kServeMaxMembers, 4, r->h.n, other) &&
              layout_fits(r->h.n, r->h.w, kServeMaxMembers, 4, r->h.n, mine))
            return SPARX_OK;
      uint64_t N = ctx.N, W = ctx.Ws, pn = 0, pw = 0, pmax = 0;
      uint32_t G = ctx.G;
      for (auto it = S->queue.begin(); it != S->queue.end();) {
        ServerReq* r = *it;
        const uint64_t n2 = N + r->h.n, w2 = W + r->h.w;
        const bool fits = !r->fresh_only && G + 1 <= kServeMaxMembers && n2 <= N_cap && w2 <= W_cap &&
                          layout_fits(pn + r->h.n, pw + r->h.w, (uint32_t)take.size() + 1, 4,
                                      std::max<uint64_t>(pmax, r->h.n), prep_budget(S->lane_budget[lane]));
        if (!fits) { ++it; continue; }
        it = S->queue.erase(it);
        r->running = true;
        r->t_start = std::chrono::steady_clock::now();
        take.push_back(r);
        N = n2;
        W = w2;
        pn += r->h.n;
        pw += r->h.w;
        pmax = std::max<uint64_t>(pmax, r->h.n);
        ++G;
      }
    }
    if (take.empty()) return SPARX_OK;
    // host checks, then one prepared union of the valid newcomers
    std::vector<HostMember> hm;
    std::vector<ServerReq*> ok;
    for (ServerReq* r : take) {
      int st = host_validate(r->h);
      if (st == SPARX_OK && r->h.w / 2 > kEidMask) st = SPARX_E_TOO_LARGE;
      if (st) {
        std::lock_guard<std::mutex> lk(S->mu);
        server_finish(S, r, st);
        continue;
      }
      HostMember h = r->h;
      h.index = hm.size();
      hm.push_back(h);
      ok.push_back(r);
    }
    S->cv_done.notify_all();
    if (hm.empty()) return SPARX_OK;
    int rc = join_group(E, J, ctx, s, hm, ok, joined);
    if (rc == SPARX_E_CUDA) return rc;
    if (rc) {
      // one of them could not be prepared (an input defect, parallel edges, no
      // room): try them one by one, so the others still join
      std::vector<ServerReq*> back;
      for (size_t i = 0; i < hm.size(); ++i) {
        std::vector<HostMember> one{hm[i]};
        one[0].index = 0;
        std::vector<ServerReq*> r1{ok[i]};
        const int r = join_group(E, J, ctx, s, one, r1, joined);
        if (r == SPARX_E_CUDA) return r;
        if (r) back.push_back(ok[i]);
      }
      // the rest run in a fresh union, through the batch path that names the error
      std::lock_guard<std::mutex> lk(S->mu);
      for (auto it = back.rbegin(); it != back.rend(); ++it) {
        (*it)->running = false;
        (*it)->fresh_only = true;
        S->queue.push_front(*it);
      }
      S->cv_work.notify_all();
    }
    return SPARX_OK;
  }

  // Prepare a group of newcomers on the second engine and join them behind
  // the running members; nonzero: the group could not be prepared (nothing
  // joined), SPARX_E_CUDA: the device failed.
  int join_group(Engine& E, UnionJob& J, PeelCtx& ctx, cudaStream_t s, std::vector<HostMember>& hm,
                 std::vector<ServerReq*>& ok, uint32_t* joined) {
    UnionJob PJ;
    uint64_t Np = 0, Wp = 0, maxn = 0;
    for (const HostMember& h : hm) {
      PJ.members.push_back(Member{(uint32_t)Np, (uint32_t)h.n, (uint32_t)Wp, (uint32_t)h.w, 0, 0});
      Np += h.n;
      Wp += h.w;
      maxn = std::max<uint64_t>(maxn, h.n);
    }
    PJ.N = Np;
    PJ.W = Wp;
    PJ.prep_only = true;
    PJ.L = make_layout(Np, Wp, (uint32_t)hm.size(), true, 4 * Wp, maxn);
    PJ.L.hub_cap = 0;  // joining members get no hub maps
    int rc = ensure_ws(*P, PJ.L.total, false);
    int prc = rc;
    if (!rc) {
      cudaStream_t ps = P->stream;
      PJ.off = at<uint32_t>(*P, PJ.L.off);
      PJ.nbr = at<uint32_t>(*P, PJ.L.nbr);
      CU(cudaMemsetAsync(at<Counters>(*P, PJ.L.cnt), 0, sizeof(Counters), ps));
      prc = upload_union(*P, hm, PJ.members, Np, Wp, PJ.off, (uint32_t*)PJ.nbr, ps);
      if (!prc) prc = run_union(*P, PJ, S->O, ps);
    }
    if (prc) {
      cudaStreamSynchronize(P->stream);
      cudaGetLastError();
      return prc == SPARX_E_CUDA ? SPARX_E_CUDA : prc;
    }
    // join: the prepared arrays go behind the union's, ids shifted
    const Layout& L = J.L;
    const uint32_t N0 = ctx.N, G0 = ctx.G;
    const uint64_t W0 = ctx.Ws, m0 = ctx.m, mp = PJ.prep_m;
    const int gridW = grid_for(std::max<uint64_t>(Wp, 1), 256, E.sm_count * 16);
    const int gridN = grid_for(Np + 1, 256, E.sm_count * 16);
    const int gridM = grid_for(std::max<uint64_t>(mp, 1), 256, E.sm_count * 16);
    uint32_t* off = J.off;
    unsigned long long* row0 = at<unsigned long long>(E, L.row0);
    k_shift_u32<<<gridN, 256, 0, s>>>(off + N0, at<uint32_t>(*P, PJ.L.off), Np + 1, (uint32_t)W0);
    if (Wp) k_shift_pairs<<<gridW, 256, 0, s>>>(row0 + W0, at<unsigned long long>(*P, PJ.L.row0), Wp, N0,
                                                (uint32_t)m0);
    if (ctx.cur_row != row0) {  // compacted working rows: the new rows go behind their live entries
      k_shift_u32<<<gridN, 256, 0, s>>>((uint32_t*)ctx.cur_off + N0, at<uint32_t>(*P, PJ.L.off), Np + 1,
                                        (uint32_t)ctx.csr_slots);
      if (Wp)
        k_shift_pairs<<<gridW, 256, 0, s>>>((unsigned long long*)ctx.cur_row + ctx.csr_slots,
                                            at<unsigned long long>(*P, PJ.L.row0), Wp, N0, (uint32_t)m0);
    }
    k_shift_u32<<<gridN, 256, 0, s>>>(at<uint32_t>(E, L.opos) + N0, at<uint32_t>(*P, PJ.L.opos), Np + 1,
                                      (uint32_t)m0);
    if (mp) {
      k_shift_u32<<<gridM, 256, 0, s>>>(at<uint32_t>(E, L.ocol) + m0, at<uint32_t>(*P, PJ.L.ocol), mp, N0);
      k_shift_u32<<<gridM, 256, 0, s>>>(at<uint32_t>(E, L.osrc) + m0, at<uint32_t>(*P, PJ.L.osrc), mp, N0);
      CU(cudaMemcpyAsync(at<int2>(E, L.es) + m0, at<int2>(*P, PJ.L.es), 8 * mp, cudaMemcpyDeviceToDevice, s));
    }
    if (ctx.U.hub_slot && Np) CU(cudaMemsetAsync(at<uint32_t>(E, L.hub_slot) + N0, 0xFF, 4 * Np, s));
    // joining rows offer neither hub maps nor tables
    if (ctx.U.vinfo && Np) CU(cudaMemsetAsync(at<unsigned long long>(E, L.vinfo) + N0, 0, 8 * Np, s));
    Counters* cnt = at<Counters>(E, L.cnt);
    if (Np) k_big_rows_range<<<grid_for(Np, 256, E.sm_count * 8), 256, 0, s>>>(off, N0, N0 + (uint32_t)Np,
                                                                                 at<uint32_t>(E, L.big),
                                                                                 &cnt->big_count);
    std::vector<Member> nm;
    for (const Member& M : PJ.members)
      nm.push_back(Member{M.vb + N0, M.n, M.sb + (uint32_t)W0, M.w, M.eb + (uint32_t)m0, M.m});
    Member* dmem = at<Member>(E, L.mem);
    CU(cudaMemcpyAsync(dmem + G0, nm.data(), sizeof(Member) * nm.size(), cudaMemcpyHostToDevice, s));
    CU(cudaMemsetAsync(at<unsigned long long>(E, L.mem_tri) + G0, 0, 8 * nm.size(), s));
    CU(cudaMemsetAsync(at<uint32_t>(E, L.mem_maxsup) + G0, 0, 4 * nm.size(), s));
    const uint32_t G1 = G0 + (uint32_t)nm.size();
    k_member_init<<<1, 256, 0, s>>>(dmem, at<MemberState>(E, L.st), G0, G1);
    ctx.U.n = N0 + (uint32_t)Np;
    ctx.U.m = (uint32_t)(m0 + mp);
    ctx.U.width = (uint32_t)(W0 + Wp);
    ctx.U.G = G1;
    CU(cudaMemcpyAsync(at<Union>(E, L.uni), &ctx.U, sizeof(Union), cudaMemcpyHostToDevice, s));
    if (mp)
      k_peel_setup<<<grid_for(mp, 256, E.sm_count * 8), 256, 0, s>>>(
          at<Union>(E, L.uni), dmem, S->O.support_mode == SPARX_SUPPORT_U8, at<unsigned long long>(E, L.mem_tri),
          at<uint32_t>(E, L.mem_maxsup), nullptr, &cnt->err, (uint32_t)m0);
    k_ctl_join<<<1, 1, 0, s>>>(at<Control>(E, L.ctl), G1, 3ull * mp + 64, Wp);
    CU(cudaStreamSynchronize(s));
    for (const Member& M : nm) {
      J.members.push_back(M);
      (void)M;
    }
    for (ServerReq* r : ok) {
      reqs.push_back(r);
      max_member_w = std::max<uint64_t>(max_member_w, r->h.w);
    }
    delivered.resize(reqs.size(), 0);
    ctx.N = N0 + (uint32_t)Np;
    ctx.G = G1;
    ctx.m = m0 + mp;
    ctx.Ws = W0 + Wp;
    ctx.csr_slots += Wp;
    *joined += (uint32_t)nm.size();
    S->joined += nm.size();
    return SPARX_OK;
  }

  int at_stop(Engine& E, UnionJob& J, PeelCtx& ctx, uint32_t reason, cudaStream_t s) override {
    if (marked && ctx.waves_run >= w_mark + 16)
      wave_us = std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t_mark).count() /
                (double)(ctx.waves_run - w_mark);
    int rc = deliver(E, J, ctx.G, s);
    if (rc) return rc;
    uint32_t joined = 0;
    bool stopping;
    {
      std::lock_guard<std::mutex> lk(S->mu);
      stopping = S->stop;
    }
    if (!stopping && reason != kExitDone) {
      rc = admit(E, J, ctx, s, &joined);
      if (rc) return rc;
    }
    bool live = false;
    for (size_t g = 0; g < delivered.size(); ++g) live |= !delivered[g];
    ctx.resume = live;
    t_mark = std::chrono::steady_clock::now();
    w_mark = ctx.waves_run;
    marked = true;
    return SPARX_OK;
  }
};

// Requests that could not join (an input defect or a multigraph): the batch
// path, which attributes a device error to the member that caused it.
void run_fresh(sparx_server* S, Engine& E, std::vector<ServerReq*>& batch) {
  std::vector<HostMember> hm;
  std::vector<size_t> which;
  std::vector<int> status(batch.size(), SPARX_OK);
  for (size_t i = 0; i < batch.size(); ++i) {
    HostMember h = batch[i]->h;
    status[i] = host_validate(h);
    if (status[i] == SPARX_OK && h.w / 2 > kEidMask) status[i] = SPARX_E_TOO_LARGE;
    if (status[i] == SPARX_OK) {
      h.index = hm.size();
      hm.push_back(h);
      which.push_back(i);
    }
  }
  std::vector<int> st2(hm.size(), SPARX_OK);
  std::vector<sparx_pkt_stats> stats(hm.size());
  int first_fail = SPARX_OK;
  if (!hm.empty()) run_batch_union(E, hm, S->O, st2.data(), stats.data(), &first_fail);
  {
    std::lock_guard<std::mutex> lk(S->mu);
    for (size_t k = 0; k < which.size(); ++k) {
      status[which[k]] = st2[k];
      batch[which[k]]->st = stats[k];
    }
    for (size_t i = 0; i < batch.size(); ++i) server_finish(S, batch[i], status[i]);
  }
  S->cv_done.notify_all();
}

void server_worker(sparx_server* S, int lane) {
  Engine& E = *S->lanes[lane];
  cudaSetDevice(S->device);
  const size_t esz = S->O.out_bits / 8;
  const uint64_t budget = S->lane_budget[lane];
  const uint64_t main_budget = budget - prep_budget(budget);
  for (;;) {
    std::vector<ServerReq*> batch;
    bool fresh = false;
    {
      std::unique_lock<std::mutex> lk(S->mu);
      S->idle += 1;
      S->cv_work.wait(lk, [&] { return S->stop || !S->queue.empty(); });
      S->idle -= 1;
      if (S->queue.empty()) {
        if (S->stop) return;
        continue;
      }
      // FIFO; a request too large for this lane is left for a larger one
      uint64_t N = 0, W = 0, mx = 0;
      for (auto it = S->queue.begin(); it != S->queue.end() && batch.size() < kServeMaxMembers;) {
        ServerReq* r = *it;
        if (!batch.empty() && r->fresh_only != fresh) { ++it; continue; }
        const uint64_t N2 = N + r->h.n, W2 = W + r->h.w, mx2 = std::max<uint64_t>(mx, r->h.n);
        if (!layout_fits(N2, W2, kServeMaxMembers, esz, mx2, main_budget)) {
          bool fits_any = false;
          for (uint64_t b : S->lane_budget)
            fits_any |= layout_fits(r->h.n, r->h.w, kServeMaxMembers, esz, r->h.n, b - prep_budget(b));
          if (!fits_any) {  // no lane can ever hold it
            it = S->queue.erase(it);
            server_finish(S, r, SPARX_E_OOM);
            S->cv_done.notify_all();
            continue;
          }
          ++it;
          continue;
        }
        if (batch.empty()) fresh = r->fresh_only;
        it = S->queue.erase(it);
        r->running = true;
        r->t_start = std::chrono::steady_clock::now();
        batch.push_back(r);
        N = N2;
        W = W2;
        mx = mx2;
      }
      if (batch.empty()) {
        // nothing fits this lane now: wait for a change
        S->cv_work.wait_for(lk, std::chrono::milliseconds(20));
        continue;
      }
    }
    if (fresh) {
      run_fresh(S, E, batch);
      continue;
    }
    // a served union: the batch, with room for requests that join while it runs
    std::vector<HostMember> hm;
    LaneHook hook;
    hook.S = S;
    hook.lane = lane;
    hook.P = S->prep[lane];
    hook.admit_dev = S->admit_dev + lane;
    for (ServerReq* r : batch) {
      int st = host_validate(r->h);
      if (st == SPARX_OK && r->h.w / 2 > kEidMask) st = SPARX_E_TOO_LARGE;
      if (st) {
        std::lock_guard<std::mutex> lk(S->mu);
        server_finish(S, r, st);
        continue;
      }
      HostMember h = r->h;
      h.index = hm.size();
      hm.push_back(h);
      hook.reqs.push_back(r);
    }
    S->cv_done.notify_all();
    if (hm.empty()) continue;
    UnionJob J;
    uint64_t N = 0, W = 0, mx = 0;
    for (const HostMember& h : hm) {
      J.members.push_back(Member{(uint32_t)N, (uint32_t)h.n, (uint32_t)W, (uint32_t)h.w, 0, 0});
      N += h.n;
      W += h.w;
      mx = std::max<uint64_t>(mx, h.n);
    }
    for (const HostMember& h : hm) hook.max_member_w = std::max<uint64_t>(hook.max_member_w, h.w);
    // a union holding a member past kJoinMaxMemberSlots never takes joins: it
    // gets no room for them, and its rows are final, so the row hash tables
    // (built once, before the peel) are safe for it within the lane's budget
    const bool no_joins = hook.max_member_w > kJoinMaxMemberSlots;
    // room: the largest extra (slots e, vertices e / 2) the lane's budget holds
    uint64_t extra = 0;
    for (uint64_t step = 1ull << 40; step && !no_joins; step >>= 1) {
      const uint64_t e2 = extra + step;
      if (W + e2 < (1ull << 31) && layout_fits(N + e2 / 2, W + e2, kServeMaxMembers, esz, mx, main_budget))
        extra = e2;
    }
    hook.N_cap = N + extra / 2;
    hook.W_cap = W + extra;
    hook.max_n0 = mx;
    hook.delivered.assign(hook.reqs.size(), 0);
    J.N = N;
    J.W = W;
    J.hook = &hook;
    J.hook_hash = no_joins;
    J.budget = main_budget;
    S->unions += 1;
    J.L = make_layout(hook.N_cap, hook.W_cap, kServeMaxMembers, true, esz * hook.W_cap, mx);
    int rc = ensure_ws(E, J.L.total, false);
    if (!rc) {
      cudaStream_t s = E.stream;
      J.off = at<uint32_t>(E, J.L.off);
      J.nbr = at<uint32_t>(E, J.L.nbr);
      J.out = at<void>(E, J.L.out);
      cudaMemsetAsync(at<Counters>(E, J.L.cnt), 0, sizeof(Counters), s);
      cudaEventRecord(E.tev[0], s);
      rc = upload_union(E, hm, J.members, N, W, J.off, (uint32_t*)J.nbr, s);
      if (!rc) rc = run_union(E, J, S->O, s);
    }
    if (E.ws3) {
      // the hash tables of a union without join room leave with it, so the
      // lane holds no more than its share while its next union runs
      cudaStreamSynchronize(E.stream);
      cudaFree(E.ws3);
      E.ws3 = nullptr;
      E.ws3_cap = 0;
    }
    if (rc) {
      // members not delivered: run them again through the batch path (which
      // names the member an input defect belongs to)
      std::vector<ServerReq*> rest;
      for (size_t g = 0; g < hook.reqs.size(); ++g)
        if (!hook.delivered[g]) rest.push_back(hook.reqs[g]);
      cudaStreamSynchronize(E.stream);
      cudaGetLastError();
      if (!rest.empty()) run_fresh(S, E, rest);
    }
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->admit_host[lane] = 0;
    }
  }
}

int server_result(ServerReq* r, int* status, sparx_pkt_stats* stats) {
  if (status) *status = r->status;
  if (stats) *stats = r->st;
  return SPARX_OK;
}

}  // namespace

namespace {

// ---------------------------------------------------------------------------
// MatrixMarket -> CSR (GraphCache::from_mtx_file, parser_mtx/mod.rs:34-162):
// the header and size line are read on the host (parser_mtx/producers.rs:
// 139-176: "%%MatrixMarket matrix coordinate pattern|integer
// symmetric|skew-symmetric|general", comment lines skipped, nrows == ncols),
// the body on the device (mtx_kernels.cuh).

bool ieq(const std::string& a, const char* b) {
  if (a.size() != std::strlen(b)) return false;
  for (size_t i = 0; i < a.size(); ++i)
    if (std::tolower((unsigned char)a[i]) != b[i]) return false;
  return true;
}

std::vector<std::string> split_ws(const std::string& line) {
  std::vector<std::string> t;
  size_t i = 0;
  auto ws = [](char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == 0x0B || c == 0x0C; };
  while (i < line.size()) {
    while (i < line.size() && ws(line[i])) ++i;
    size_t j = i;
    while (j < line.size() && !ws(line[j])) ++j;
    if (j > i) t.push_back(line.substr(i, j - i));
    i = j;
  }
  return t;
}

bool parse_usize(const std::string& t, uint64_t* out) {
  size_t i = 0;
  if (i < t.size() && t[i] == '+') ++i;
  if (i >= t.size()) return false;
  uint64_t v = 0;
  for (; i < t.size(); ++i) {
    const unsigned c = (unsigned char)t[i] - '0';
    if (c > 9 || v > (~0ull - c) / 10) return false;
    v = v * 10 + c;
  }
  *out = v;
  return true;
}

struct MtxHeader {
  uint64_t n = 0, nnz = 0, body = 0, header_lines = 0;
  bool symmetric = true;
};

int mtx_header(const char* text, uint64_t len, MtxHeader* h) {
  uint64_t p = 0, lines = 0;
  auto next_line = [&](std::string* out) -> bool {
    if (p >= len) return false;
    uint64_t e = p;
    while (e < len && text[e] != '\n') ++e;
    out->assign(text + p, e - p);
    p = e < len ? e + 1 : e;
    ++lines;
    return true;
  };
  std::string line;
  if (!next_line(&line) || line.compare(0, 14, "%%MatrixMarket") != 0) {
    set_error("invalid MatrixMarket header");
    return SPARX_E_PARSE;
  }
  const auto tok = split_ws(line);
  if (tok.size() < 5) { set_error("malformed MatrixMarket header"); return SPARX_E_PARSE; }
  if (!ieq(tok[1], "matrix") || !ieq(tok[2], "coordinate") || !(ieq(tok[3], "pattern") || ieq(tok[3], "integer")) ||
      !(ieq(tok[4], "symmetric") || ieq(tok[4], "skew-symmetric") || ieq(tok[4], "general"))) {
    set_error("only 'matrix coordinate pattern/integer symmetric|skew-symmetric|general' is supported");
    return SPARX_E_PARSE;
  }
  h->symmetric = !ieq(tok[4], "general");
  for (;;) {
    if (!next_line(&line)) { set_error("unexpected end of text before the size line"); return SPARX_E_PARSE; }
    const auto t = split_ws(line);
    if (t.empty() || t[0][0] == '%') continue;
    uint64_t nr = 0, nc = 0, nnz = 0;
    if (t.size() < 3 || !parse_usize(t[0], &nr) || !parse_usize(t[1], &nc) || !parse_usize(t[2], &nnz)) {
      set_error("malformed size line");
      return SPARX_E_PARSE;
    }
    if (nr != nc) { set_error("only square matrices are supported (nrows != ncols)"); return SPARX_E_PARSE; }
    h->n = nr;
    h->nnz = nnz;
    break;
  }
  h->body = p;
  h->header_lines = lines;
  return SPARX_OK;
}

int mtx_to_csr(const char* text, uint64_t len, uint64_t* offsets_out, uint64_t offsets_cap,
               uint64_t* neighbours_out, uint64_t neighbours_cap, uint64_t* n_out, uint64_t* width_out,
               const sparx_pkt_opts* opts) {
  g_last_error.clear();
  if (!text || !n_out || !width_out) { set_error("null pointer"); return SPARX_E_ARG; }
  MtxHeader H;
  int rc = mtx_header(text, len, &H);
  if (rc) return rc;
  if (H.n >= 0xFFFFFFFFull) { set_error("more than 2^32 - 2 vertices"); return SPARX_E_TOO_LARGE; }
  Opts O;
  rc = read_opts(opts, &O);
  if (rc) return rc;
  Engine* Ep;
  rc = get_engine(O.device, &Ep);
  if (rc) return rc;
  Engine& E = *Ep;
  std::lock_guard<std::mutex> lk(E.mu);
  CU(cudaSetDevice(E.device));
  cudaStream_t s = E.stream;
  const uint64_t blen = len - H.body;
  const uint64_t chunks = (blen + 15) / 16;
  // lines of the body (a line starts at byte 0 and after every '\n' but the last byte)
  unsigned long long lines = 0;
  if (blen) {
    const char* bp = text + H.body;
    long long nl = 0;
#pragma omp parallel for reduction(+ : nl) schedule(static)
    for (long long i = 0; i < (long long)blen - 1; ++i) nl += bp[i] == '\n';
    lines = 1 + (unsigned long long)nl;
  }
  // one workspace: body, line starts and counts, keys (two per line at most,
  // ping-pong), radix histograms, degrees, offsets and neighbours
  size_t p = 0;
  auto take = [&](size_t bytes) { size_t r = p; p = align_up(p + std::max<size_t>(bytes, 1)); return r; };
  const uint64_t edges_max = 2 * lines;
  const uint32_t rblocks = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(E.sm_count * 4ull,
                                                                              (edges_max + 4095) / 4096));
  const uint64_t scan_items = std::max<uint64_t>({chunks, lines, H.n, 256ull * rblocks, 1});
  const size_t o_body = take(blen), o_cpref = take(8 * (chunks + 1)),
               o_tiles = take(8 * ((scan_items + kScanTile - 1) / kScanTile + 2)), o_cnt = take(64),
               o_starts = take(8 * lines), o_count = take(4 * lines), o_at = take(8 * (lines + 1)),
               o_ka = take(8 * edges_max), o_kb = take(8 * edges_max), o_hist = take(4ull * 256 * rblocks),
               o_start = take(4ull * 256 * rblocks + 4), o_deg = take(4 * (H.n + 1)), o_off = take(8 * (H.n + 1)),
               o_nbr = take(8 * edges_max);
  rc = ensure_ws(E, p);
  if (rc) return rc;
  unsigned char* body = at<unsigned char>(E, o_body);
  unsigned long long* cpref = at<unsigned long long>(E, o_cpref);
  unsigned long long* tiles = at<unsigned long long>(E, o_tiles);
  unsigned long long* dcnt = at<unsigned long long>(E, o_cnt);  // [0] scan total, [1] first bad line
  uint32_t* derr = (uint32_t*)(dcnt + 2);
  // body -> device through the pinned staging buffers
  for (uint64_t c = 0, a = 0; a < blen; ++c, a += kStageBytes) {
    const int slot = (int)(c & 1);
    const uint64_t k = std::min<uint64_t>(kStageBytes, blen - a);
    CU(cudaEventSynchronize(E.pin_ev[slot]));
    parallel_copy(E.pinned[slot], text + H.body + a, k);
    CU(cudaMemcpyAsync(body + a, E.pinned[slot], k, cudaMemcpyHostToDevice, s));
    CU(cudaEventRecord(E.pin_ev[slot], s));
  }
  CU(cudaMemsetAsync(dcnt, 0, 64, s));
  CU(cudaMemsetAsync(dcnt + 1, 0xFF, 8, s));
  if (chunks) {
    unsigned long long dl = 0;
    exclusive_scan<unsigned long long>(MtxLineCount{body, blen}, chunks, cpref, tiles, dcnt, s);
    CU(cudaMemcpyAsync(&dl, cpref + chunks, 8, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (dl != lines) { set_error("line count mismatch"); return SPARX_E_CUDA; }
  }
  unsigned long long* starts = at<unsigned long long>(E, o_starts);
  uint32_t* count = at<uint32_t>(E, o_count);
  unsigned long long* atp = at<unsigned long long>(E, o_at);
  const int pgrid = grid_for(lines, 256, E.sm_count * 16);
  if (lines) {
    k_mtx_fill_lines<<<grid_for(chunks, 256, E.sm_count * 16), 256, 0, s>>>(body, blen, cpref, starts);
    k_mtx_parse<false><<<pgrid, 256, 0, s>>>(body, blen, starts, lines, H.n, H.symmetric, count, nullptr, nullptr,
                                             derr, dcnt + 1);
  }
  uint32_t herr = 0;
  unsigned long long bad = 0, edges = 0;
  CU(cudaMemcpyAsync(&herr, derr, 4, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(&bad, dcnt + 1, 8, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (herr) {
    const char* what = (herr & kMtxBadNumber) ? "an index that is not an unsigned integer"
                       : (herr & kMtxZeroIndex) ? "an index of 0 (MatrixMarket indices are 1-based)"
                                                : "an index beyond the size line";
    set_error(std::string("line ") + std::to_string(H.header_lines + bad + 1) + ": " + what);
    return SPARX_E_PARSE;
  }
  if (lines) {
    exclusive_scan<unsigned long long>(LoadCount{count}, lines, atp, tiles, dcnt, s);
    CU(cudaMemcpyAsync(&edges, atp + lines, 8, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
  }
  if (edges >= 0xFFFFFFFFull) { set_error("more than 2^32 - 2 entries after mirroring"); return SPARX_E_TOO_LARGE; }
  *n_out = H.n;
  *width_out = edges;
  if (!offsets_out || !neighbours_out) return SPARX_OK;  // sizes only
  if (offsets_cap < H.n + 1 || neighbours_cap < edges) {
    set_error("output buffers too small (need n + 1 offsets and width neighbours)");
    return SPARX_E_ARG;
  }
  unsigned long long* ka = at<unsigned long long>(E, o_ka);
  unsigned long long* kb = at<unsigned long long>(E, o_kb);
  uint32_t* hist = at<uint32_t>(E, o_hist);
  uint32_t* hstart = at<uint32_t>(E, o_start);
  uint32_t* deg = at<uint32_t>(E, o_deg);
  unsigned long long* doff = at<unsigned long long>(E, o_off);
  unsigned long long* dnbr = at<unsigned long long>(E, o_nbr);
  if (lines)
    k_mtx_parse<true><<<pgrid, 256, 0, s>>>(body, blen, starts, lines, H.n, H.symmetric, nullptr, atp, ka, derr,
                                            dcnt + 1);
  // sort by (row, column): the low 32 bits (columns), then the high (rows),
  // only the bits that vertex ids < n use
  const int bits = H.n > 1 ? 64 - __builtin_clzll(H.n - 1) : 1;
  std::vector<int> shifts;
  for (int b = 0; b < bits; b += 8) shifts.push_back(b);
  for (int b = 0; b < bits; b += 8) shifts.push_back(32 + b);
  const uint32_t blocks = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(rblocks, (edges + 4095) / 4096));
  unsigned long long *src = ka, *dst = kb;
  if (edges > 1) {
    for (int sh : shifts) {
      k_radix_hist<<<blocks, kRadixThreads, 0, s>>>(src, edges, sh, hist);
      exclusive_scan<uint32_t>(LoadU32{hist}, 256ull * blocks, hstart, (uint32_t*)tiles, (uint32_t*)dcnt, s);
      k_radix_scatter<false><<<blocks, kRadixThreads, 0, s>>>(src, dst, edges, sh, hstart, nullptr, nullptr);
      std::swap(src, dst);
    }
  }
  CU(cudaMemsetAsync(deg, 0, 4 * (H.n + 1), s));
  if (edges) k_mtx_rows<<<grid_for(edges, 256, E.sm_count * 16), 256, 0, s>>>(src, edges, deg);
  exclusive_scan<unsigned long long>(LoadCount{deg}, H.n, doff, tiles, dcnt, s);
  if (edges) k_mtx_columns<<<grid_for(edges, 256, E.sm_count * 16), 256, 0, s>>>(src, edges, dnbr);
  if (H.n == 0) CU(cudaMemsetAsync(doff, 0, 8, s));
  rc = download(E, offsets_out, doff, 8 * (H.n + 1), s);
  if (rc) return rc;
  rc = download(E, neighbours_out, dnbr, 8 * edges, s);
  if (rc) return rc;
  CU(cudaStreamSynchronize(s));
  CU(cudaGetLastError());
  return SPARX_OK;
}

}  // namespace

extern "C" int sparx_mtx_to_csr(const char* text, uint64_t len, uint64_t* offsets_out, uint64_t offsets_cap,
                                uint64_t* neighbours_out, uint64_t neighbours_cap, uint64_t* n_out,
                                uint64_t* width_out, const sparx_pkt_opts* opts) {
  return mtx_to_csr(text, len, offsets_out, offsets_cap, neighbours_out, neighbours_cap, n_out, width_out, opts);
}

extern "C" {

int sparx_pkt_run_batch(const sparx_graph_view* graphs, uint64_t count, uint64_t hbm_budget_bytes,
                        const sparx_pkt_opts* opts, int* status_out, sparx_pkt_stats* stats_out) {
  return run_batch(graphs, count, hbm_budget_bytes, opts, status_out, stats_out);
}

int sparx_server_create(sparx_server** out, uint64_t hbm_budget_bytes, const sparx_pkt_opts* opts) {
  g_last_error.clear();
  if (!out) { set_error("null server pointer"); return SPARX_E_ARG; }
  Opts O;
  int rc = read_opts(opts, &O);
  if (rc) return rc;
  int device = O.device;
  if (device < 0) CU(cudaGetDevice(&device));
  CU(cudaSetDevice(device));
  if (!hbm_budget_bytes) hbm_budget_bytes = 150ull << 30;
  size_t free_b = 0, total_b = 0;
  CU(cudaMemGetInfo(&free_b, &total_b));
  const uint64_t usable = free_b > (2ull << 30) ? free_b - (2ull << 30) : free_b / 2;
  const uint64_t budget = std::min<uint64_t>(hbm_budget_bytes, usable);
  auto* S = new sparx_server();
  S->device = device;
  S->O = O;
  if (const char* env = std::getenv("SPARX_SERVE_LANES")) {
    const int k = std::atoi(env);
    if (k >= 1 && k <= 16) S->nlanes = k;
  }
  const int nl = S->nlanes;
  // lane 0 takes half the budget (a large graph fits there, with room for
  // requests that join it); the other lanes share the rest
  for (int i = 0; i < nl; ++i)
    S->lane_budget.push_back(nl == 1 ? budget : i == 0 ? budget / 2 : budget / 2 / (nl - 1));
  auto fail = [&](int code) {
    for (Engine* L : S->lanes) engine_release(L);
    for (Engine* L : S->prep) engine_release(L);
    if (S->admit_host) cudaFreeHost(S->admit_host);
    delete S;
    return code;
  };
  cudaError_t e = cudaHostAlloc(&S->admit_host, 4 * nl, cudaHostAllocMapped);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); S->admit_host = nullptr; return fail(SPARX_E_CUDA); }
  std::memset(S->admit_host, 0, 4 * nl);
  e = cudaHostGetDevicePointer((void**)&S->admit_dev, S->admit_host, 0);
  if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return fail(SPARX_E_CUDA); }
  for (int i = 0; i < 2 * nl; ++i) {
    Engine* E = new Engine();
    rc = engine_init(*E, device);
    if (rc) {
      engine_release(E);
      return fail(rc);
    }
    (i < nl ? S->lanes : S->prep).push_back(E);
  }
  for (int i = 0; i < nl; ++i) S->workers.emplace_back(server_worker, S, i);
  *out = S;
  return SPARX_OK;
}

int sparx_server_submit(sparx_server* S, const sparx_graph_view* v, uint64_t* ticket) {
  g_last_error.clear();
  if (!S || !v || !ticket) { set_error("null argument"); return SPARX_E_ARG; }
  if (!v->offsets || v->n_plus_1 < 1 || (v->width && (!v->neighbours || !v->truss_out)) ||
      (v->neighbour_bits != 32 && v->neighbour_bits != 64)) {
    set_error("bad graph view");
    return SPARX_E_ARG;
  }
  int rc = check_dims(v->n_plus_1, v->width);
  if (rc) return rc;
  auto* r = new ServerReq();
  r->h.off = v->offsets;
  r->h.n = v->n_plus_1 - 1;
  r->h.nbr = v->neighbours;
  r->h.bits = v->neighbour_bits == 32 ? 32 : 64;
  r->h.w = v->width;
  r->h.out = v->truss_out;
  r->t_submit = std::chrono::steady_clock::now();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) { delete r; set_error("server is shutting down"); return SPARX_E_ARG; }
    r->ticket = S->next_ticket++;
    S->reqs[r->ticket] = r;
    S->queue.push_back(r);
    // running unions stop at their next wave to see whether it can join
    for (int i = 0; i < S->nlanes; ++i) ((volatile uint32_t*)S->admit_host)[i] = 1;
  }
  S->cv_work.notify_one();
  *ticket = r->ticket;
  return SPARX_OK;
}

int sparx_server_poll(sparx_server* S, uint64_t ticket, int* done, int* status, sparx_pkt_stats* stats) {
  if (!S || !done) return SPARX_E_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return SPARX_E_NOT_FOUND;
  *done = it->second->done ? 1 : 0;
  if (it->second->done) server_result(it->second, status, stats);
  return SPARX_OK;
}

int sparx_server_wait(sparx_server* S, uint64_t ticket, uint64_t timeout_ms, int* status, sparx_pkt_stats* stats) {
  if (!S) return SPARX_E_ARG;
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return SPARX_E_NOT_FOUND;
  ServerReq* r = it->second;
  auto pred = [&] { return r->done; };
  if (timeout_ms) {
    if (!S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) return SPARX_E_TIMEOUT;
  } else {
    S->cv_done.wait(lk, pred);
  }
  return server_result(r, status, stats);
}

int sparx_server_cancel(sparx_server* S, uint64_t ticket) {
  if (!S) return SPARX_E_ARG;
  std::lock_guard<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return SPARX_E_NOT_FOUND;
  ServerReq* r = it->second;
  if (r->running || r->done) { set_error("request already admitted"); return SPARX_E_ARG; }
  for (auto q = S->queue.begin(); q != S->queue.end(); ++q)
    if (*q == r) { S->queue.erase(q); break; }
  r->cancelled = true;
  server_finish(S, r, SPARX_E_CANCELLED);
  S->cv_done.notify_all();
  return SPARX_OK;
}

int sparx_server_info(sparx_server* S, uint64_t* unions, uint64_t* joined) {
  if (!S) return SPARX_E_ARG;
  if (unions) *unions = S->unions.load();
  if (joined) *joined = S->joined.load();
  return SPARX_OK;
}

int sparx_server_destroy(sparx_server* S) {
  if (!S) return SPARX_E_ARG;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  for (auto& t : S->workers) t.join();
  for (Engine* E : S->lanes) engine_release(E);
  for (Engine* E : S->prep) engine_release(E);
  if (S->admit_host) cudaFreeHost(S->admit_host);
  for (auto& kv : S->reqs) delete kv.second;
  delete S;
  return SPARX_OK;
}


// ---- tuning and the autotuner ------------------------------------------------

int sparx_tuning_default(sparx_tuning* t) {
  if (!t) return SPARX_E_ARG;
  const Tuning d;
  t->struct_size = sizeof(sparx_tuning);
  t->merge_ratio = d.merge_ratio;
  t->hub_min_degree = d.hub_min_degree;
  t->sample_min = d.sample_min;
  t->support_kernel = d.support_kernel;
  t->compact_pct = d.compact_pct;
  t->hash_min_degree = d.hash_min_degree;
  t->sup_hash_min = d.sup_hash_min;
  t->relabel = d.relabel;
  return SPARX_OK;
}

int sparx_tuning_signature(const uint64_t* offsets, uint64_t n_plus_1, uint32_t key[3]) {
  if (!offsets || !key || n_plus_1 < 1) return SPARX_E_ARG;
  uint32_t cnt[34] = {};
  unsigned long long slots[34] = {};
  for (uint64_t u = 0; u + 1 < n_plus_1; ++u) {
    const uint64_t d = offsets[u + 1] - offsets[u];
    if (!d || d > 0xFFFFFFFFull) continue;
    const int b = 32 - __builtin_clz((uint32_t)d);
    cnt[b]++;
    slots[b] += d;
  }
  const TuneKey k = tune_key(cnt, slots, offsets[n_plus_1 - 1] - offsets[0]);
  key[0] = k.log_w;
  key[1] = k.log_dmax;
  key[2] = k.skew8;
  return SPARX_OK;
}

namespace {
Tuning from_c(const sparx_tuning* t) {
  return Tuning{t->merge_ratio, t->hub_min_degree, t->sample_min, t->support_kernel, t->compact_pct,
                t->hash_min_degree, t->sup_hash_min, t->relabel};
}
void to_c(const Tuning& t, sparx_tuning* o) {
  o->struct_size = sizeof(sparx_tuning);
  o->merge_ratio = t.merge_ratio;
  o->hub_min_degree = t.hub_min_degree;
  o->sample_min = t.sample_min;
  o->support_kernel = t.support_kernel;
  o->compact_pct = t.compact_pct;
  o->hash_min_degree = t.hash_min_degree;
  o->sup_hash_min = t.sup_hash_min;
  o->relabel = t.relabel;
}
}  // namespace

int sparx_tuning_lookup(const uint32_t key[3], sparx_tuning* out, int* found) {
  if (!key || !out) return SPARX_E_ARG;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  const TuneKey k{key[0], key[1], key[2]};
  auto it = g_tune.find(k);
  if (found) *found = it != g_tune.end();
  to_c(it != g_tune.end() ? it->second : default_tuning(k), out);
  return SPARX_OK;
}

int sparx_tuning_store(const uint32_t key[3], const sparx_tuning* t) {
  if (!key || !t || (t->struct_size && t->struct_size < sizeof(sparx_tuning))) return SPARX_E_ARG;
  const Tuning v = from_c(t);
  if (!valid_tuning(v)) { g_last_error = "tuning value out of range"; return SPARX_E_ARG; }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[TuneKey{key[0], key[1], key[2]}] = v;
  return SPARX_OK;
}

int sparx_tuning_clear(void) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune.clear();
  g_tune_loaded = true;  // an explicit clear also drops what SPARX_TUNE_FILE would add
  return SPARX_OK;
}

int sparx_tuning_last(sparx_tuning* used, uint32_t key[3]) {
  if (used) to_c(g_tune_last, used);
  if (key) {
    key[0] = g_tune_last_key.log_w;
    key[1] = g_tune_last_key.log_dmax;
    key[2] = g_tune_last_key.skew8;
  }
  return SPARX_OK;
}

int sparx_tuning_save(const char* path) {
  if (!path) return SPARX_E_ARG;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  return tune_save_locked(path);
}

int sparx_tuning_load(const char* path) {
  if (!path) return SPARX_E_ARG;
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_loaded = true;
  return tune_load_locked(path);
}

}  // extern "C"

namespace {

// Coordinate descent over the knobs, one group at a time from the defaults:
// the support form and sampling threshold by the support pass's device time,
// then the hub-map floor (orientation + peel, since the maps are built with
// the orientation), the merge ratio and the compaction fill by the peel's.
// `run(t, &ms_support, &ms_rest)` decomposes the sample once with knobs t.
// The best knobs are stored under the sample's key (and written to the file
// SPARX_TUNE_FILE names, if any).
template <class RunF>
int autotune_core(RunF run, uint32_t repeats, Tuning* best_out, TuneKey* key_out) {
  repeats = std::max<uint32_t>(1, std::min<uint32_t>(repeats, 15));
  auto measure = [&](const Tuning& t, double* sup, double* rest) -> int {
    std::vector<double> a, b;
    g_tune_force = &t;
    int rc = SPARX_OK;
    for (uint32_t r = 0; r < repeats && !rc; ++r) {
      double x = 0, y = 0;
      rc = run(&x, &y);
      a.push_back(x);
      b.push_back(y);
    }
    g_tune_force = nullptr;
    if (rc) return rc;
    std::sort(a.begin(), a.end());
    std::sort(b.begin(), b.end());
    *sup = a[a.size() / 2];
    *rest = b[b.size() / 2];
    return SPARX_OK;
  };
  Tuning cur;
  double sup = 0, rest = 0;
  int rc = measure(cur, &sup, &rest);  // also warms the engine for this size and finds the key
  if (rc) return rc;
  const TuneKey key = g_tune_last_key;
  cur = default_tuning(key);  // descent starts from the key's defaults
  rc = measure(cur, &sup, &rest);
  if (rc) return rc;
  auto try_group = [&](std::vector<Tuning> cands, bool support_time) -> int {
    double best = support_time ? sup : rest;
    for (const Tuning& c : cands) {
      double x = 0, y = 0;
      const int r = measure(c, &x, &y);
      if (r) return r;
      const double v = support_time ? x : y;
      if (v < best * 0.98) {  // a 2% margin keeps noise from flipping a knob
        best = v;
        cur = c;
        sup = x;
        rest = y;
      }
    }
    return SPARX_OK;
  };
  std::vector<Tuning> c1;
  for (uint32_t smp : {32u, 128u, 256u}) { Tuning t = cur; t.sample_min = smp; c1.push_back(t); }
  { Tuning t = cur; t.support_kernel = cur.support_kernel == 1 ? 2 : 1; c1.push_back(t); }
  for (uint32_t sh : {16u, 64u}) { Tuning t = cur; t.sup_hash_min = sh; c1.push_back(t); }
  if ((rc = try_group(c1, true))) return rc;
  std::vector<Tuning> c2;
  for (uint32_t h : {0u, 512u, 4096u}) { Tuning t = cur; t.hub_min_degree = h; c2.push_back(t); }
  if ((rc = try_group(c2, false))) return rc;
  std::vector<Tuning> c3;
  for (uint32_t mr : {4u, 16u}) { Tuning t = cur; t.merge_ratio = mr; c3.push_back(t); }
  if ((rc = try_group(c3, false))) return rc;
  std::vector<Tuning> c4;
  for (uint32_t cp : {75u, 95u}) { Tuning t = cur; t.compact_pct = cp; c4.push_back(t); }
  if ((rc = try_group(c4, false))) return rc;
  {
    // the relabelling changes the support pass and the peel (and costs a pass
    // in the orientation): judged on the whole decomposition
    Tuning t = cur;
    t.relabel = cur.relabel ? 0 : 1;
    double x = 0, y = 0;
    if ((rc = measure(t, &x, &y))) return rc;
    if (x + y < (sup + rest) * 0.98) {
      cur = t;
      sup = x;
      rest = y;
    }
  }
  std::vector<Tuning> c5;
  for (uint32_t hm : {0u, 32u, 512u}) { Tuning t = cur; t.hash_min_degree = hm; c5.push_back(t); }
  if ((rc = try_group(c5, false))) return rc;
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tune[key] = cur;
    const char* path = std::getenv("SPARX_TUNE_FILE");
    if (path && *path) tune_save_locked(path);
  }
  *best_out = cur;
  *key_out = key;
  return SPARX_OK;
}

void key_to_c(const TuneKey& k, uint32_t key[3]) {
  if (!key) return;
  key[0] = k.log_w;
  key[1] = k.log_dmax;
  key[2] = k.skew8;
}

}  // namespace

extern "C" {

int sparx_autotune(const uint64_t* offsets, uint64_t n_plus_1, const uint64_t* neighbours, uint64_t width,
                   const sparx_pkt_opts* opts, uint32_t repeats, sparx_tuning* best, uint32_t key[3]) {
  g_last_error.clear();
  if (!offsets || !neighbours || !best) { set_error("null pointer"); return SPARX_E_ARG; }
  sparx_pkt_opts o;
  if (opts) o = *opts; else sparx_pkt_default_opts(&o);
  o.struct_size = sizeof(o);
  o.out_bits = 32;
  o.support_kernel = 0;  // the tuning picks the support form
  std::vector<uint32_t> out(std::max<uint64_t>(width, 1));
  auto run = [&](double* sup, double* rest) -> int {
    sparx_pkt_stats st;
    const int rc = run_host(offsets, n_plus_1, neighbours, 64, width, out.data(), false, &o, &st);
    *sup = st.ms_support;
    *rest = st.ms_orient + st.ms_peel;
    return rc;
  };
  Tuning t;
  TuneKey k;
  const int rc = autotune_core(run, repeats, &t, &k);
  if (rc) return rc;
  to_c(t, best);
  key_to_c(k, key);
  return SPARX_OK;
}

int sparx_autotune_batch(const sparx_graph_view* graphs, uint64_t count, uint64_t hbm_budget_bytes,
                         const sparx_pkt_opts* opts, uint32_t repeats, sparx_tuning* best, uint32_t key[3]) {
  g_last_error.clear();
  if (!graphs || !count || !best) { set_error("null or empty graph list"); return SPARX_E_ARG; }
  sparx_pkt_opts o;
  if (opts) o = *opts; else sparx_pkt_default_opts(&o);
  o.struct_size = sizeof(o);
  o.support_kernel = 0;
  std::vector<sparx_pkt_stats> st(count);
  std::vector<int> status(count);
  auto run = [&](double* sup, double* rest) -> int {
    const int rc = run_batch(graphs, count, hbm_budget_bytes, &o, status.data(), st.data());
    // the first union's phases (members of a union share them)
    *sup = st[0].ms_support;
    *rest = st[0].ms_orient + st[0].ms_peel;
    return rc;
  };
  Tuning t;
  TuneKey k;
  const int rc = autotune_core(run, repeats, &t, &k);
  if (rc) return rc;
  to_c(t, best);
  key_to_c(k, key);
  return SPARX_OK;
}

int sparx_pkt_default_opts(sparx_pkt_opts* o) {
  if (!o) return SPARX_E_ARG;
  std::memset(o, 0, sizeof(*o));
  o->struct_size = sizeof(sparx_pkt_opts);
  o->support_mode = SPARX_SUPPORT_WIDE;
  o->out_bits = 8;
  o->device = -1;
  o->loop = SPARX_LOOP_GRAPH;
  o->support_kernel = 0;
  o->timeout_ms = kDefaultTimeoutMs;
  return SPARX_OK;
}

const char* sparx_strerror(int s) {
  switch (s) {
    case SPARX_OK: return "ok";
    case SPARX_E_INVALID_CSR: return "invalid CSR (unsorted row, asymmetric, id >= n or bad offsets)";
    case SPARX_E_MULTIGRAPH: return "parallel edges are not supported";
    case SPARX_E_OVERFLOW_U8: return "truss number exceeds 255 with 8-bit output";
    case SPARX_E_OOM: return "out of device memory / HBM budget";
    case SPARX_E_TIMEOUT: return "device peel exceeded its time budget";
    case SPARX_E_CUDA: return "CUDA error";
    case SPARX_E_TOO_LARGE: return "graph too large (width >= 2^32 or m >= 2^28)";
    case SPARX_E_ARG: return "bad argument";
    case SPARX_E_NOT_FOUND: return "unknown ticket";
    case SPARX_E_CANCELLED: return "request cancelled";
    case SPARX_E_PARSE: return "malformed MatrixMarket text";
    default: return "unknown status";
  }
}

const char* sparx_last_error(void) { return g_last_error.c_str(); }

int sparx_pkt_run(const uint64_t* offsets, uint64_t n_plus_1, const uint64_t* neighbours, uint64_t width,
                  void* truss_out, const sparx_pkt_opts* opts, sparx_pkt_stats* stats) {
  return run_host(offsets, n_plus_1, neighbours, 64, width, truss_out, false, opts, stats);
}

int sparx_pkt_run_u32(const uint64_t* offsets, uint64_t n_plus_1, const uint32_t* neighbours, uint64_t width,
                      void* truss_out, const sparx_pkt_opts* opts, sparx_pkt_stats* stats) {
  return run_host(offsets, n_plus_1, neighbours, 32, width, truss_out, false, opts, stats);
}

int sparx_triangles_run(const uint64_t* offsets, uint64_t n_plus_1, const uint64_t* neighbours, uint64_t width,
                        uint32_t* support_out, const sparx_pkt_opts* opts, sparx_pkt_stats* stats) {
  return run_host(offsets, n_plus_1, neighbours, 64, width, support_out, true, opts, stats);
}

int sparx_kcore_run(const uint64_t* offsets, uint64_t n_plus_1, const uint64_t* neighbours, uint64_t width,
                    void* core_out, const sparx_pkt_opts* opts, sparx_pkt_stats* stats) {
  if (n_plus_1 > 1 && !core_out) {
    g_last_error = "null pointer";
    return SPARX_E_ARG;
  }
  return run_host(offsets, n_plus_1, neighbours, 64, width, core_out, false, opts, stats, nullptr, true);
}

int sparx_clustering_run(const uint64_t* offsets, uint64_t n_plus_1, const uint64_t* neighbours, uint64_t width,
                         double* local_out, double* transitivity, double* average, const sparx_pkt_opts* opts,
                         sparx_pkt_stats* stats) {
  if (n_plus_1 > 1 && !local_out) {
    g_last_error = "null pointer";
    return SPARX_E_ARG;
  }
  ClusterSums cc;
  const int rc = run_host(offsets, n_plus_1, neighbours, 64, width, local_out, true, opts, stats, &cc);
  if (rc) return rc;
  // clustering_coefficient.rs:178-181: (total slot support / 3) / 2 / total
  // possible pairs, and the mean local coefficient (IEEE semantics for 0/0)
  if (transitivity) *transitivity = (double)(cc.slots / 3) / 2.0 / cc.possible;
  if (average) *average = cc.local / (double)(n_plus_1 - 1);
  return SPARX_OK;
}

int sparx_pkt_run_device(const uint64_t* d_offsets, uint64_t n_plus_1, const uint32_t* d_neighbours, uint64_t width,
                         void* d_truss_out, const sparx_pkt_opts* opts, sparx_pkt_stats* stats, void* cuda_stream) {
  g_last_error.clear();
  if (!d_offsets || (!d_neighbours && width) || (!d_truss_out && width)) { set_error("null pointer"); return SPARX_E_ARG; }
  int rc = check_dims(n_plus_1, width);
  if (rc) return rc;
  Opts O;
  rc = read_opts(opts, &O);
  if (rc) return rc;
  Engine* Ep;
  rc = get_engine(O.device, &Ep);
  if (rc) return rc;
  Engine& E = *Ep;
  std::lock_guard<std::mutex> lk(E.mu);
  CU(cudaSetDevice(E.device));
  const uint64_t n = n_plus_1 - 1;
  UnionJob J;
  J.N = n;
  J.W = width;
  J.members.push_back(Member{0, (uint32_t)n, 0, (uint32_t)width, 0, 0});
  J.L = make_layout(n, width, 1, false, 0);
  rc = ensure_ws(E, J.L.total);
  if (rc) return rc;
  cudaStream_t s = cuda_stream ? (cudaStream_t)cuda_stream : E.stream;
  J.off = at<uint32_t>(E, J.L.off);
  J.nbr = d_neighbours;
  J.out = d_truss_out;
  Counters* cnt = at<Counters>(E, J.L.cnt);
  auto t0 = std::chrono::steady_clock::now();
  CU(cudaMemsetAsync(cnt, 0, sizeof(Counters), s));
  CU(cudaEventRecord(E.tev[0], s));
  k_narrow_offsets<<<grid_for(n_plus_1, 256, E.sm_count * 16), 256, 0, s>>>(
      (const unsigned long long*)d_offsets, J.off, (uint32_t)n_plus_1, 0u, 0ll, (long long)width, &cnt->err);
  if (width)
    k_range_ids<<<grid_for(width, 256, E.sm_count * 16), 256, 0, s>>>(d_neighbours, nullptr, width, (uint32_t)n, 0u,
                                                                       &cnt->err);
  J.launches += width ? 2 : 1;
  rc = run_union(E, J, O, s);
  fill_stats(J, 0, stats);
  if (rc) return rc;
  auto t1 = std::chrono::steady_clock::now();
  if (stats) {
    float up = 0;
    cudaEventElapsedTime(&up, E.tev[0], E.tev[1]);
    stats->ms_upload = up;
    stats->ms_total = std::chrono::duration<double, std::milli>(t1 - t0).count();
  }
  return SPARX_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free entry point (no counterpart in the reference).
//
// Some callers cannot allocate device memory at the moment they need a
// decomposition: services that reserve all device memory up front through
// their own pool and treat any allocation outside it as a fault, and
// latency-critical request paths that must neither wait for nor fail on
// cudaMalloc.  For them this variant of the single-graph pipeline keeps every
// scratch array in one fixed, file-scope device array instead of the engine's
// workspace.  It allocates nothing (device or pinned host memory, streams or
// events): the caller passes device inputs and the device output, and a
// stream.  The call is host-synchronous: it reads scalars back and waits for
// the stream several times, so `cuda_stream` must not be a stream that is
// being captured.
namespace {

constexpr size_t kNoAllocScratchBytes = 64ull << 20;  // per device; bounds the graph size below

// Lives in every GPU that loads this library, until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;

// Device address of the scratch array on `device` (which must be current).
// In host code the symbol is only a host-side stand-in, so the address is
// looked up with cudaGetSymbolAddress.  The first call on a device also loads
// the module there; later calls are cheap, and looking the address up on every
// call (rather than caching it) keeps it right after a context is torn down
// and recreated.
int noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= kMaxDevices) {
    set_error("device ordinal out of range");
    return SPARX_E_ARG;
  }
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) {
    set_error(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    return SPARX_E_CUDA;
  }
  *out = (unsigned char*)p;
  return SPARX_OK;
}

// Waits for the stream when a call leaves early after its first launch, so the
// shared array is idle when the call returns (kernels already queued would
// otherwise keep writing to it while the caller's next call starts).
struct DrainOnExit {
  cudaStream_t s;
  bool armed = false;
  ~DrainOnExit() {
    if (armed) {
      cudaStreamSynchronize(s);
      cudaGetLastError();
    }
  }
};

// The same arrays as the engine's workspace, minus staging and output.
Layout make_noalloc_layout(uint64_t N, uint64_t W) {
  Layout L{};
  size_t p = 0;
  auto take = [&](size_t bytes) {
    size_t r = p;
    p = align_up(p + std::max<size_t>(bytes, 1));
    return r;
  };
  const uint64_t M = std::max<uint64_t>(W / 2, 1);
  L.off = take(4 * (N + 1));
  L.row0 = take(8 * W);
  L.dplus = take(4 * N);
  L.opos = take(4 * (N + 1));
  L.ocol = take(4 * M);
  L.osrc = take(4 * M);
  L.es = take(8 * M);
  L.act0 = take(4 * M);
  L.act1 = take(4 * M);
  L.q0 = take(16 * M + 16);
  L.q1 = L.q0 + 8 * M;
  L.qd0 = take(16 * M);
  L.qd1 = take(16 * M);
  L.big = take(4 * (W / kWarpRow + 1));
  const uint64_t tiles = (std::max<uint64_t>(N + 1, M + 1) + kScanTile - 1) / kScanTile + 2;
  L.tiles = take(8 * tiles);
  L.ctl = take(sizeof(Control));
  L.mem = take(sizeof(Member));
  L.st = take(sizeof(MemberState));
  L.wpref = take(16);
  L.cnt = take(sizeof(Counters));
  L.mem_tri = take(8);
  L.mem_maxsup = take(4);
  L.uni = take(sizeof(Union));
  L.total = p;
  return L;
}

int run_noalloc(const uint64_t* d_offsets, uint64_t n_plus_1, const uint32_t* d_nbr, uint64_t width,
                uint32_t* d_out, int device, cudaStream_t s) {
  g_last_error.clear();
  if (!d_offsets || (width && (!d_nbr || !d_out))) { set_error("null pointer"); return SPARX_E_ARG; }
  int rc = check_dims(n_plus_1, width);
  if (rc) return rc;
  if (device < 0) CU(cudaGetDevice(&device));
  CU(cudaSetDevice(device));
  unsigned char* base = nullptr;
  rc = noalloc_scratch(device, &base);
  if (rc) return rc;
  const uint64_t n = n_plus_1 - 1;
  const Layout L = make_noalloc_layout(n, width);
  if (L.total > kNoAllocScratchBytes) {
    set_error("graph needs " + std::to_string(L.total) + " bytes of scratch; the allocation-free entry point has " +
              std::to_string(kNoAllocScratchBytes) + " (about 1.4 M CSR slots); use sparx_pkt_run_device");
    return SPARX_E_TOO_LARGE;
  }
  auto P = [&](size_t off) { return base + off; };
  uint32_t* off = (uint32_t*)P(L.off);
  unsigned long long* row0 = (unsigned long long*)P(L.row0);
  uint32_t* dplus = (uint32_t*)P(L.dplus);
  uint32_t* opos = (uint32_t*)P(L.opos);
  uint32_t* ocol = (uint32_t*)P(L.ocol);
  uint32_t* osrc = (uint32_t*)P(L.osrc);
  int2* es = (int2*)P(L.es);
  Counters* cnt = (Counters*)P(L.cnt);
  uint32_t* err = &cnt->err;
  int sm = 148, per_sm = 1;
  CU(cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, device));
  CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wave<false>, 256, 0));
  const int wave_blocks = std::max(1, per_sm) * sm;
  const uint32_t N = (uint32_t)n;

  DrainOnExit drain{s};
  drain.armed = true;
  // the array keeps the previous call's contents: reset what must start at zero
  CU(cudaMemsetAsync(cnt, 0, sizeof(Counters), s));
  k_narrow_offsets<<<grid_for(n_plus_1, 256, sm * 16), 256, 0, s>>>((const unsigned long long*)d_offsets, off,
                                                                    (uint32_t)n_plus_1, 0u, 0ll, (long long)width, err);
  if (width) k_range_ids<<<grid_for(width, 256, sm * 16), 256, 0, s>>>(d_nbr, nullptr, width, N, 0u, err);
  Counters hc;
  CU(cudaMemcpyAsync(&hc, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (hc.err) {
    set_error("invalid CSR input (offsets or neighbour ids)");
    return status_from_flags(hc.err);
  }

  const int vgrid = grid_for(N, 256, sm * 32);  // row kernels: 32 vertices per warp
  uint32_t* big = (uint32_t*)P(L.big);  // big_count was cleared with the counters above
  k_big_rows<<<grid_for(N, 256, sm * 8), 256, 0, s>>>(off, N, big, &cnt->big_count);
  k_orient_count<<<vgrid, 256, 0, s>>>(off, d_nbr, N, dplus, &cnt->self_loops, err, &cnt->max_dplus, big,
                                       &cnt->big_count);
  exclusive_scan<uint32_t>(LoadU32{dplus}, N, opos, (uint32_t*)P(L.tiles), (uint32_t*)&cnt->grand, s);
  uint32_t m32 = 0;
  CU(cudaMemcpyAsync(&m32, opos + N, 4, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(&hc, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  if (hc.err) {
    set_error("invalid CSR input (row order, duplicates or ids)");
    return status_from_flags(hc.err);
  }
  const uint64_t m = m32;
  if (2 * m + hc.self_loops != width) {
    set_error("CSR is not symmetric");
    return SPARX_E_INVALID_CSR;
  }
  if (m > kEidMask) {
    set_error("a graph has >= 2^28 edges");
    return SPARX_E_TOO_LARGE;
  }
  k_orient_fill<<<vgrid, 256, 0, s>>>(off, d_nbr, N, opos, ocol, osrc, row0, (uint32_t*)P(L.q0), big,
                                      &cnt->big_count);
  k_orient_reverse<<<grid_for(width, 256, sm * 16), 256, 0, s>>>(d_nbr, (uint32_t*)P(L.q0), width, opos, ocol,
                                                                row0, err);

  CU(cudaMemsetAsync(es, 0, 8 * std::max<uint64_t>(m, 1), s));
  {
    uint32_t launches = 0;
    unsigned long long elements = 0;
    rc = launch_support(sm, 0, N, m, hc.max_dplus, opos, ocol, osrc, es, (unsigned long long*)P(L.q0),
                        (unsigned long long*)P(L.tiles), cnt, (uint32_t*)P(L.act0), s, &launches, &elements);
    if (rc) return rc;
  }

  Union U{};  // no hub maps in the fixed scratch
  U.off = off;
  U.row = row0;
  U.opos = opos;
  U.ocol = ocol;
  U.osrc = osrc;
  U.es = es;
  U.act[0] = (uint32_t*)P(L.act0);
  U.act[1] = (uint32_t*)P(L.act1);
  U.q[0] = (unsigned long long*)P(L.q0);
  U.q[1] = (unsigned long long*)P(L.q1);
  U.qd[0] = (uint4*)P(L.qd0);
  U.qd[1] = (uint4*)P(L.qd1);
  U.n = N;
  U.m = (uint32_t)m;
  U.width = (uint32_t)width;
  U.G = 1;
  const Member M0{0, N, 0, (uint32_t)width, 0, (uint32_t)m};
  Control c0{};
  c0.G = 1;
  c0.max_waves = 3ull * m + 64;
  c0.timeout_ns = kDefaultTimeoutMs * 1000000ull;
  c0.csr_slots = width;
  c0.compact_min = ~0ull;  // no compaction buffers in the fixed scratch
  c0.compact_pct = Tuning{}.compact_pct;
  Union* dU = (Union*)P(L.uni);
  Member* dM = (Member*)P(L.mem);
  Control* dC = (Control*)P(L.ctl);
  MemberState* dS = (MemberState*)P(L.st);
  unsigned long long* wpref = (unsigned long long*)P(L.wpref);
  // pageable sources: the copies are staged before these calls return
  CU(cudaMemcpyAsync(dU, &U, sizeof(Union), cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(dM, &M0, sizeof(Member), cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(dC, &c0, sizeof(Control), cudaMemcpyHostToDevice, s));
  CU(cudaMemsetAsync(P(L.mem_tri), 0, 8, s));
  CU(cudaMemsetAsync(P(L.mem_maxsup), 0, 4, s));
  if (m > 0)
    k_peel_setup<<<grid_for(m, 256, sm * 8), 256, 0, s>>>(dU, dM, 0, (unsigned long long*)P(L.mem_tri),
                                                           (uint32_t*)P(L.mem_maxsup), nullptr, err);
  k_peel_init<<<1, 1024, 0, s>>>(dM, dS, dC, wpref, 1);
  WaveArgs wa;
  wa.Up = dU;
  wa.arr = peel_arrays(U);
  wa.mem = dM;
  wa.st = dS;
  wa.ctl = dC;
  wa.wpref = wpref;
  wa.err = err;
  wa.handle = cudaGraphConditionalHandle{};
  wa.use_handle = 0;
  for (;;) {
    for (int i = 0; i < 16; ++i) k_wave<false><<<wave_blocks, 256, 0, s>>>(wa);
    uint32_t done = 0;
    CU(cudaMemcpyAsync(&done, &dC->done, 4, cudaMemcpyDeviceToHost, s));
    CU(cudaStreamSynchronize(s));
    if (done) break;
  }
  if (width)
    k_finalize<uint32_t><<<grid_for(width, 256, sm * 16), 256, 0, s>>>(row0, es, width, d_out, 0, 0, &cnt->kmax, err,
                                                                       nullptr);
  CU(cudaMemcpyAsync(&hc, cnt, sizeof(Counters), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  drain.armed = false;
  CU(cudaGetLastError());
  if (hc.err) set_error("device peel reported an error");
  return status_from_flags(hc.err);
}

}  // namespace

extern "C" int sparx_pkt_run_device_noalloc(const uint64_t* d_offsets, uint64_t n_plus_1,
                                            const uint32_t* d_neighbours, uint64_t width, uint32_t* d_truss_out,
                                            int device, void* cuda_stream) {
  return run_noalloc(d_offsets, n_plus_1, d_neighbours, width, d_truss_out, device, (cudaStream_t)cuda_stream);
}
