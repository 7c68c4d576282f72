// Synthetic graph generators for the PKT k-truss workloads.
//
// Every generator writes the CSR layout that the reference's graph store
// memory-maps (graph/mod.rs:482-489, built by parser_mtx/mod.rs:34-162 and
// sorted per row by impl_sort.rs:10-51): offsets u64[n+1], neighbour ids
// sorted ascending inside each row, both directions of every undirected edge
// present.  Unlike the reference's MTX parser these generators also drop
// self-loops and duplicate edges, so the output is a simple graph.
//
// Randomness is counter based: draw k of stream s under seed S is
// splitmix64_mix(key(S, s) + (k + 1) * golden_gamma), i.e. element k of the
// splitmix64 sequence seeded with key(S, s).  Any draw can be computed
// independently, so the output does not depend on the number of threads.
//
// Workloads:
//   ER      n vertices, m distinct unordered pairs u != v, drawn without
//           replacement: candidates are drawn in order and the first m
//           distinct ones are kept.
//   R-MAT   2^scale vertices, edge_factor * 2^scale generated pairs, quadrant
//           probabilities a, b, c, d = 1 - a - b - c, no noise, vertex ids
//           passed through a seeded Fisher-Yates permutation.
//   de Bruijn  distinct k-mers (2 bits per base) of a seeded uniform ACGT
//           sequence plus mutated copies of random segments of it; an edge
//           joins k-mers a, b whenever suffix_{k-1}(a) == prefix_{k-1}(b).
//   mix     member i of a batch: ER or R-MAT (fair coin), n log-uniform in
//           [n_lo, n_hi], average degree uniform in [d_lo, d_hi].
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>
#include <omp.h>

namespace {

constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ull;

inline uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Stream key: distinct streams of one seed never share a splitmix sequence.
inline uint64_t stream_key(uint64_t seed, uint64_t stream) {
  return mix64(seed * kGamma + mix64(stream + 0x632BE59BD9B4E019ull));
}

inline uint64_t draw(uint64_t key, uint64_t k) { return mix64(key + (k + 1) * kGamma); }

// floor(r32 * n / 2^32): maps a 32-bit draw into [0, n) without division.
inline uint32_t bounded32(uint64_t r, uint32_t n) {
  return (uint32_t)(((r >> 32) * (uint64_t)n) >> 32);
}
inline uint64_t bounded64(uint64_t r, uint64_t n) {
  return (uint64_t)(((unsigned __int128)r * n) >> 64);
}

struct Graph {
  uint64_t n = 0;
  std::vector<uint64_t> off;  // n + 1
  std::vector<uint32_t> nbr;  // width
  // mix member description (zero for the other generators)
  uint32_t kind = 0;          // 0 = ER, 1 = R-MAT, 2 = de Bruijn
  double avg_degree = 0.0;
};

// LSD radix sort of 64-bit keys on the low `bits` bits, 11 bits per pass.
void radix_sort_u64(std::vector<uint64_t>& keys, int bits) {
  const size_t N = keys.size();
  if (N < 2) return;
  std::vector<uint64_t> tmp(N);
  const int R = 11, B = 1 << R;
  int nthreads = omp_get_max_threads();
  std::vector<size_t> hist((size_t)nthreads * B);
  uint64_t* src = keys.data();
  uint64_t* dst = tmp.data();
  int passes = (bits + R - 1) / R;
  for (int p = 0; p < passes; ++p) {
    int shift = p * R;
    std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(nthreads)
    {
      int t = omp_get_thread_num();
      size_t lo = N * t / nthreads, hi = N * (t + 1) / nthreads;
      size_t* h = &hist[(size_t)t * B];
      for (size_t i = lo; i < hi; ++i) h[(src[i] >> shift) & (B - 1)]++;
#pragma omp barrier
#pragma omp single
      {
        size_t sum = 0;
        for (int d = 0; d < B; ++d)
          for (int tt = 0; tt < nthreads; ++tt) {
            size_t c = hist[(size_t)tt * B + d];
            hist[(size_t)tt * B + d] = sum;
            sum += c;
          }
      }
      for (size_t i = lo; i < hi; ++i) dst[h[(src[i] >> shift) & (B - 1)]++] = src[i];
    }
    std::swap(src, dst);
  }
  if (src != keys.data()) std::memcpy(keys.data(), src, N * sizeof(uint64_t));
}

int bits_for(uint64_t n) {
  int b = 1;
  while (b < 64 && (1ull << b) < n) ++b;
  return b;
}

// Directed keys (src << 32 | dst), both directions present -> sorted,
// deduplicated symmetric CSR.  Self-loops must already be gone.
void keys_to_csr(std::vector<uint64_t>& keys, uint64_t n, Graph& g) {
  radix_sort_u64(keys, 32 + bits_for(n));
  size_t w = 0;
  for (size_t i = 0; i < keys.size(); ++i)
    if (i == 0 || keys[i] != keys[i - 1]) keys[w++] = keys[i];
  keys.resize(w);
  g.n = n;
  g.off.assign(n + 1, 0);
  g.nbr.resize(w);
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < w; ++i) g.nbr[i] = (uint32_t)keys[i];
  // row starts: first key of each source
  std::vector<uint64_t>& off = g.off;
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < w; ++i) {
    uint64_t s = keys[i] >> 32;
    if (i == 0 || (keys[i - 1] >> 32) != s) {
      uint64_t prev = (i == 0) ? 0 : (keys[i - 1] >> 32) + 1;
      for (uint64_t v = prev; v <= s; ++v) off[v] = i;
    }
  }
  uint64_t last = w ? (keys[w - 1] >> 32) + 1 : 0;
  for (uint64_t v = last; v <= n; ++v) off[v] = w;
}

void emit_pair(std::vector<uint64_t>& keys, size_t at, uint32_t u, uint32_t v) {
  keys[2 * at] = ((uint64_t)u << 32) | v;
  keys[2 * at + 1] = ((uint64_t)v << 32) | u;
}

Graph* gen_er(uint64_t n, uint64_t m, uint64_t seed) {
  Graph* g = new Graph();
  g->kind = 0;
  uint64_t max_pairs = n < 2 ? 0 : n * (n - 1) / 2;
  if (m > max_pairs) m = max_pairs;
  uint64_t key = stream_key(seed, 1);
  // candidate c -> (pair key, c); keep the first m distinct pairs in draw order
  uint64_t K = m + m / 8 + 1024;
  std::vector<std::pair<uint64_t, uint64_t>> cand;
  std::vector<uint64_t> chosen;
  for (;;) {
    cand.assign(K, {UINT64_MAX, UINT64_MAX});
#pragma omp parallel for schedule(static)
    for (uint64_t c = 0; c < K; ++c) {
      uint64_t a = bounded64(draw(key, 2 * c), n), b = bounded64(draw(key, 2 * c + 1), n);
      if (a == b) continue;
      uint64_t lo = a < b ? a : b, hi = a < b ? b : a;
      cand[c] = {(lo << 32) | hi, c};
    }
    std::sort(cand.begin(), cand.end());
    std::vector<std::pair<uint64_t, uint64_t>> firsts;  // (draw index, pair)
    firsts.reserve(K);
    for (size_t i = 0; i < cand.size(); ++i) {
      if (cand[i].first == UINT64_MAX) break;
      if (i == 0 || cand[i].first != cand[i - 1].first) firsts.push_back({cand[i].second, cand[i].first});
    }
    if (firsts.size() >= m || K > 64 * (m + 1024)) {
      std::sort(firsts.begin(), firsts.end());
      size_t take = std::min<size_t>(m, firsts.size());
      chosen.resize(take);
      for (size_t i = 0; i < take; ++i) chosen[i] = firsts[i].second;
      break;
    }
    K *= 2;
  }
  std::vector<uint64_t> keys(2 * chosen.size());
#pragma omp parallel for schedule(static)
  for (size_t i = 0; i < chosen.size(); ++i)
    emit_pair(keys, i, (uint32_t)(chosen[i] >> 32), (uint32_t)chosen[i]);
  keys_to_csr(keys, n, *g);
  g->avg_degree = n ? (double)g->nbr.size() / n : 0.0;
  return g;
}

// Seeded Fisher-Yates permutation of [0, n).
std::vector<uint32_t> permutation(uint64_t n, uint64_t key) {
  std::vector<uint32_t> p(n);
  for (uint64_t i = 0; i < n; ++i) p[i] = (uint32_t)i;
  for (uint64_t i = n; i > 1; --i) {
    uint64_t j = bounded64(draw(key, i - 1), i);
    std::swap(p[i - 1], p[j]);
  }
  return p;
}

// R-MAT over 2^scale ids; when n_out < 2^scale ids are scaled down to [0, n_out)
// (floor(id * n_out / 2^scale)) before the permutation, which keeps the skew.
Graph* gen_rmat(uint32_t scale, uint64_t n_out, uint64_t n_pairs, double a, double b, double c,
                uint64_t seed, int permute) {
  Graph* g = new Graph();
  g->kind = 1;
  const uint64_t N = 1ull << scale;
  if (n_out == 0 || n_out > N) n_out = N;
  const uint64_t ta = (uint64_t)std::floor(a * 4294967296.0);
  const uint64_t tab = (uint64_t)std::floor((a + b) * 4294967296.0);
  const uint64_t tabc = (uint64_t)std::floor((a + b + c) * 4294967296.0);
  uint64_t key = stream_key(seed, 2);
  std::vector<uint32_t> perm;
  if (permute) perm = permutation(n_out, stream_key(seed, 3));
  std::vector<uint64_t> keys(2 * n_pairs);
  std::atomic<uint64_t> kept{0};
#pragma omp parallel
  {
    std::vector<uint64_t> local;
    local.reserve(4096);
#pragma omp for schedule(static)
    for (uint64_t k = 0; k < n_pairs; ++k) {
      uint64_t u = 0, v = 0;
      for (uint32_t lvl = 0; lvl < scale; ++lvl) {
        uint64_t r = draw(key, k * scale + lvl) >> 32;
        uint64_t bu, bv;
        if (r < ta) { bu = 0; bv = 0; }
        else if (r < tab) { bu = 0; bv = 1; }
        else if (r < tabc) { bu = 1; bv = 0; }
        else { bu = 1; bv = 1; }
        u = (u << 1) | bu;
        v = (v << 1) | bv;
      }
      if (n_out != N) {
        u = (u * n_out) >> scale;
        v = (v * n_out) >> scale;
      }
      if (permute) { u = perm[u]; v = perm[v]; }
      if (u == v) continue;
      local.push_back((u << 32) | v);
      if (local.size() == 4096) {
        uint64_t at = kept.fetch_add(local.size());
        for (size_t i = 0; i < local.size(); ++i)
          emit_pair(keys, at + i, (uint32_t)(local[i] >> 32), (uint32_t)local[i]);
        local.clear();
      }
    }
    uint64_t at = kept.fetch_add(local.size());
    for (size_t i = 0; i < local.size(); ++i)
      emit_pair(keys, at + i, (uint32_t)(local[i] >> 32), (uint32_t)local[i]);
  }
  keys.resize(2 * kept.load());
  keys_to_csr(keys, n_out, *g);
  g->avg_degree = n_out ? (double)g->nbr.size() / n_out : 0.0;
  return g;
}

Graph* gen_debruijn(uint64_t seq_len, uint32_t k, uint32_t copies, uint32_t seg_len, double mut_rate,
                    uint64_t seed) {
  Graph* g = new Graph();
  g->kind = 2;
  if (k < 2 || k > 31 || seq_len < k) { g->off.assign(1, 0); return g; }
  const uint64_t mask = (k == 32) ? ~0ull : ((1ull << (2 * k)) - 1);
  uint64_t kseq = stream_key(seed, 4), kseg = stream_key(seed, 5), kmut = stream_key(seed, 6);
  std::vector<uint8_t> seq(seq_len);
#pragma omp parallel for schedule(static)
  for (uint64_t i = 0; i < seq_len; ++i) seq[i] = (uint8_t)(draw(kseq, i) >> 62);
  if (seg_len > seq_len) seg_len = (uint32_t)seq_len;
  const uint64_t tmut = (uint64_t)std::floor(mut_rate * 4294967296.0);
  uint64_t nk_main = seq_len - k + 1;
  uint64_t nk_copy = seg_len >= k ? seg_len - k + 1 : 0;
  std::vector<uint64_t> kmers(nk_main + (uint64_t)copies * nk_copy);
  // main sequence k-mers
#pragma omp parallel for schedule(static)
  for (uint64_t i = 0; i < nk_main; ++i) {
    uint64_t x = 0;
    for (uint32_t j = 0; j < k; ++j) x = (x << 2) | seq[i + j];
    kmers[i] = x;
  }
  // mutated copies of random segments
#pragma omp parallel for schedule(dynamic, 4)
  for (uint32_t cidx = 0; cidx < copies; ++cidx) {
    uint64_t start = bounded64(draw(kseg, cidx), seq_len - seg_len + 1);
    std::vector<uint8_t> s(seq.begin() + start, seq.begin() + start + seg_len);
    for (uint32_t p = 0; p < seg_len; ++p) {
      uint64_t r = draw(kmut, (uint64_t)cidx * seg_len + p);
      if ((r >> 32) < tmut) s[p] = (uint8_t)((s[p] + 1 + ((r & 0xffffffffull) % 3)) & 3);
    }
    uint64_t base = nk_main + (uint64_t)cidx * nk_copy;
    for (uint64_t i = 0; i < nk_copy; ++i) {
      uint64_t x = 0;
      for (uint32_t j = 0; j < k; ++j) x = (x << 2) | s[i + j];
      kmers[base + i] = x;
    }
  }
  radix_sort_u64(kmers, 2 * k);
  kmers.erase(std::unique(kmers.begin(), kmers.end()), kmers.end());
  const uint64_t n = kmers.size();
  // successor edges: a -> ((a << 2) | x) & mask when present
  std::vector<std::vector<uint64_t>> parts(omp_get_max_threads());
#pragma omp parallel
  {
    std::vector<uint64_t>& loc = parts[omp_get_thread_num()];
#pragma omp for schedule(static)
    for (uint64_t i = 0; i < n; ++i) {
      uint64_t a = kmers[i];
      for (uint64_t x = 0; x < 4; ++x) {
        uint64_t b = ((a << 2) | x) & mask;
        if (b == a) continue;
        auto it = std::lower_bound(kmers.begin(), kmers.end(), b);
        if (it != kmers.end() && *it == b) {
          uint64_t j = (uint64_t)(it - kmers.begin());
          loc.push_back((i << 32) | j);
          loc.push_back((j << 32) | i);
        }
      }
    }
  }
  size_t tot = 0;
  for (auto& p : parts) tot += p.size();
  std::vector<uint64_t> keys;
  keys.reserve(tot);
  for (auto& p : parts) { keys.insert(keys.end(), p.begin(), p.end()); std::vector<uint64_t>().swap(p); }
  keys_to_csr(keys, n, *g);
  g->avg_degree = n ? (double)g->nbr.size() / n : 0.0;
  return g;
}

}  // namespace

extern "C" {

typedef struct sgx_mix_member {
  uint32_t kind;        // 0 = ER, 1 = R-MAT
  uint32_t scale;       // R-MAT scale (ceil(log2 n)), 0 for ER
  uint64_t n;           // vertices
  uint64_t pairs;       // ER: distinct pairs; R-MAT: generated pairs
  double avg_degree;    // requested average degree
  uint64_t seed;
} sgx_mix_member;

void* sgx_gen_er(uint64_t n, uint64_t m, uint64_t seed) {
  if (n >= (1ull << 32)) return nullptr;
  try { return gen_er(n, m, seed); } catch (...) { return nullptr; }
}

void* sgx_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed,
                   int permute) {
  if (scale == 0 || scale > 31) return nullptr;
  try {
    return gen_rmat(scale, 1ull << scale, (uint64_t)edge_factor << scale, a, b, c, seed, permute);
  } catch (...) { return nullptr; }
}

void* sgx_gen_debruijn(uint64_t seq_len, uint32_t k, uint32_t copies, uint32_t seg_len,
                       double mut_rate, uint64_t seed) {
  try { return gen_debruijn(seq_len, k, copies, seg_len, mut_rate, seed); } catch (...) { return nullptr; }
}

// Describe member `index` of a batch mix (seed = base_seed + index).
int sgx_mix_describe(uint64_t index, uint64_t base_seed, double n_lo, double n_hi, double d_lo,
                     double d_hi, sgx_mix_member* out) {
  if (!out || n_lo < 2 || n_hi < n_lo) return -1;
  uint64_t seed = base_seed + index;
  uint64_t key = stream_key(seed, 7);
  double u1 = (double)(draw(key, 1) >> 11) * (1.0 / 9007199254740992.0);
  double u2 = (double)(draw(key, 2) >> 11) * (1.0 / 9007199254740992.0);
  uint64_t n = (uint64_t)std::floor(std::exp(std::log(n_lo) + u1 * (std::log(n_hi) - std::log(n_lo))));
  if (n < 2) n = 2;
  double d = d_lo + u2 * (d_hi - d_lo);
  out->kind = (uint32_t)(draw(key, 0) >> 63);
  out->n = n;
  out->avg_degree = d;
  out->seed = seed;
  uint64_t pairs = (uint64_t)std::llround((double)n * d / 2.0);
  if (out->kind == 0) {
    uint64_t mx = n * (n - 1) / 2;
    out->pairs = pairs > mx ? mx : pairs;
    out->scale = 0;
  } else {
    out->pairs = pairs;
    out->scale = (uint32_t)bits_for(n);
  }
  return 0;
}

void* sgx_gen_mix_member(const sgx_mix_member* d, double a, double b, double c) {
  if (!d) return nullptr;
  try {
    Graph* g = (d->kind == 0) ? gen_er(d->n, d->pairs, d->seed)
                              : gen_rmat(d->scale, d->n, d->pairs, a, b, c, d->seed, 1);
    g->avg_degree = d->avg_degree;
    return g;
  } catch (...) { return nullptr; }
}

void sgx_graph_dims(const void* h, uint64_t* n, uint64_t* width) {
  const Graph* g = (const Graph*)h;
  if (n) *n = g->n;
  if (width) *width = g->nbr.size();
}

// Copy into caller buffers: offsets u64[n+1]; neighbours as u64 (bits=64) or u32 (bits=32).
int sgx_graph_copy(const void* h, uint64_t* offsets, void* nbrs, int bits) {
  const Graph* g = (const Graph*)h;
  if (offsets) std::memcpy(offsets, g->off.data(), (g->n + 1) * sizeof(uint64_t));
  if (!nbrs) return 0;
  if (bits == 32) {
    std::memcpy(nbrs, g->nbr.data(), g->nbr.size() * sizeof(uint32_t));
  } else if (bits == 64) {
    uint64_t* o = (uint64_t*)nbrs;
    const size_t w = g->nbr.size();
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < w; ++i) o[i] = g->nbr[i];
  } else {
    return -1;
  }
  return 0;
}

void sgx_graph_free(void* h) { delete (Graph*)h; }

int sgx_set_threads(int t) {
  if (t > 0) omp_set_num_threads(t);
  return omp_get_max_threads();
}

}  // extern "C"
