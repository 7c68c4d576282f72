// ORACLE — test infrastructure only.  Nothing in the product path links,
// loads or calls this file: only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py use it, as the checker.
//
// CPU restatement of the reference's PKT k-truss path (alexfaisca/sparkx,
// Rust).  The reference cannot be built in this environment (no cargo/rustc,
// no crates registry), so this is a restatement of its algorithm, function
// by function:
//
//   orc_edge_index   graph/impl_csc.rs:87-263   edge_over (eo) + edge_reciprocal (er)
//   orc_triangles    k_truss/triangles.rs:144-243  per-slot triangle support
//   orc_pkt          k_truss/pkt.rs:216-563     PKT level / sub-level peel
//   orc_burkhardt    k_truss/burkhardt_et_al.rs:186-380  sequential stack peel
//   orc_verify       k_truss/mod.rs:30-216      verifier, with its bounds corrected
//   orc_fast_truss   (no counterpart) an independent exact peel used to check
//                    the large workloads, where the reference's hash-map-per-
//                    frontier-edge processing would take hours.
//
// Parity is unpinned by the reference itself: it ships no truss or support
// golden vectors (its PKT/Burkhardt tests read GGCAT datasets that are not
// in the repository, and its verifier rejects every non-empty graph, see
// orc_verify).  The restatements are pinned instead by hand-derived known
// answers and by agreement with a brute-force definition in tests/.
//
// Two support widths, as in the reference discussion:
//   wide (mode 0): u32 counters, the mathematically defined truss.
//   u8   (mode 1): the reference's AtomicU8 counters (triangles.rs:6,20),
//                  i.e. support modulo 256, then the same peel; truss = s + 2
//                  wrapping in u8, and a level counter overflow is an error
//                  (pkt.rs:508-516).
//
// Two defects of pkt.rs are NOT reproduced (the truss decomposition is unique,
// so a correct peel has exactly one answer):
//   D1 pkt.rs:492 clears in_curr[e_idx] with e_idx a frontier position, not
//      the edge id; here the edge's own flag is cleared.
//   D2 pkt.rs:489-495 marks processed[] before the barrier at :497 while
//      other threads may still be processing the sub-level; here the marks
//      are written between two barriers.
//   D3 shared_slice.rs:665-682 push_slice refuses a push that exactly fills
//      the queue (write_idx + len < max), so a frontier holding every slot
//      (e.g. a lone triangle) is dropped; here the queues hold width + 1.
// D5, in the multi-edge reciprocal index, is described at edge_index.
// A fourth defect, in the clustering coefficient built on the supports (D4:
// clustering_coefficient.rs:130-135 zeroes the supports before reading them),
// is restated in oracle.py's `clustering`, which computes the intended
// coefficients by default and the reference's zero output on request.
//
// Input: symmetric CSR (offsets u64[n+1], neighbour ids u32, rows sorted
// non-decreasing).  Self-loop slots are allowed and get truss 2, as in the
// reference (triangles.rs:194, impl_csc.rs:148-153).  Parallel edges (equal
// neighbour ids side by side in a row, as GGCAT's orientation labels give
// them) follow the reference's OneOrMany paths: every copy is its own slot
// with its own reciprocal (impl_csc.rs:154-215), a vertex maps to all of its
// copies (triangles.rs:172-191, pkt.rs:373-395, burkhardt_et_al.rs:288-312),
// and a triangle is one choice of a copy of each of its three pairs.
#include <algorithm>
#include <atomic>
#include <barrier>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <functional>
#include <thread>
#include <unordered_map>
#include <vector>

#include <omp.h>

namespace {

enum {
  ORC_OK = 0,
  ORC_E_INVALID = 1,
  ORC_E_MULTIGRAPH = 2,
  ORC_E_OVERFLOW = 3,
  ORC_E_QUEUE = 4,
};

struct Csr {
  uint64_t n;
  const uint64_t* off;
  const uint32_t* nbr;
  uint64_t width() const { return off[n]; }
};

// Rows sorted non-decreasing, ids < n; *multi tells whether any row repeats
// a neighbour (a multigraph).
int validate(const Csr& g, bool* multi = nullptr) {
  if (g.off[0] != 0) return ORC_E_INVALID;
  bool dup = false;
  for (uint64_t u = 0; u < g.n; ++u) {
    if (g.off[u + 1] < g.off[u]) return ORC_E_INVALID;
    for (uint64_t i = g.off[u]; i < g.off[u + 1]; ++i) {
      if (g.nbr[i] >= g.n) return ORC_E_INVALID;
      if (i > g.off[u]) {
        if (g.nbr[i] == g.nbr[i - 1]) dup = true;
        if (g.nbr[i] < g.nbr[i - 1]) return ORC_E_INVALID;
      }
    }
  }
  if (multi) *multi = dup;
  return ORC_OK;
}

void run_threads(int T, const std::function<void(int)>& fn) {
  std::vector<std::thread> th;
  for (int t = 1; t < T; ++t) th.emplace_back(fn, t);
  fn(0);
  for (auto& x : th) x.join();
}

// Vertex -> slots lookup used where the reference keeps a
// HashMap<usize, OneOrMany<usize>> per vertex (triangles.rs:171-191,
// pkt.rs:373-395, burkhardt_et_al.rs:288-312): put() is called for a row's
// slots in order, so the copies of one neighbour are consecutive slots and the
// OneOrMany list is the range [first, first + count).
//   HashSlots   std::unordered_map, for the timed CPU baseline.
//   DenseSlots  a vertex-indexed array reset after each use; same answers.
struct HashSlots {
  std::unordered_map<uint64_t, std::pair<uint64_t, uint64_t>> m;
  explicit HashSlots(uint64_t) {}
  void put(uint64_t w, uint64_t slot) {
    auto it = m.try_emplace(w, slot, 0).first;
    ++it->second.second;
  }
  bool get(uint64_t w, uint64_t* first, uint64_t* count) const {
    auto it = m.find(w);
    if (it == m.end()) return false;
    *first = it->second.first;
    *count = it->second.second;
    return true;
  }
  void clear() { m.clear(); }
};

struct DenseSlots {
  std::vector<uint64_t> slot;  // first slot + 1, 0 = absent
  std::vector<uint32_t> count;
  std::vector<uint64_t> used;
  explicit DenseSlots(uint64_t n) : slot(n, 0), count(n, 0) {}
  void put(uint64_t w, uint64_t s) {
    if (!slot[w]) { used.push_back(w); slot[w] = s + 1; }
    ++count[w];
  }
  bool get(uint64_t w, uint64_t* first, uint64_t* cnt) const {
    if (!slot[w]) return false;
    *first = slot[w] - 1;
    *cnt = count[w];
    return true;
  }
  void clear() {
    for (uint64_t w : used) { slot[w] = 0; count[w] = 0; }
    used.clear();
  }
};

// graph/impl_csc.rs:87-263.  Pass 1 (:124-139): eo[u] = first slot of u whose
// neighbour id is > u, else off[u+1].  Pass 2 (:143-241): for each slot u->v
// with v <= u: a self-loop is its own reciprocal (:148-153); the first copy of
// u->v binary-searches u in v's upper part (:217-235; the search may land on
// any copy of u there); a second copy takes the slot just after, else just
// before, the previous copy's reciprocal (:154-180); a later copy walks
// forwards, then backwards, from the first copy's reciprocal to the first
// copy of u not yet taken (:181-215).  Both directions are linked.
//
// Defect D5, not reproduced: the reference bounds neither those walks and
// probes (only by the array's ends) nor its binary search (inclusive upper
// bound off[v+1]) to v's row, so when v's copies of u end its row and row
// v + 1 starts with u, a copy is paired with a slot of vertex v + 1 and a slot
// of v stays unpaired (er is then not a pairing and the reference's supports
// go to the wrong slots).  Here every probe stays inside [eo[v], off[v+1]).
int edge_index(const Csr& g, uint64_t* eo, uint64_t* er, int T) {
  const uint64_t n = g.n;
  const uint64_t load = (n + T - 1) / T;
  std::atomic<int> status{ORC_OK};
  std::barrier sync(T);
  run_threads(T, [&](int tid) {
    uint64_t begin = std::min<uint64_t>(tid * load, n), end = std::min<uint64_t>(begin + load, n);
    for (uint64_t u = begin; u < end; ++u) {
      uint64_t stop = g.off[u + 1], at = stop;
      for (uint64_t i = g.off[u]; i < stop; ++i)
        if (g.nbr[i] > u) { at = i; break; }
      eo[u] = at;
    }
    sync.arrive_and_wait();
    // prev: the previous slot's (v, reciprocal) pairs, One = a single entry
    std::vector<std::pair<uint64_t, uint64_t>> prev;
    for (uint64_t u = begin; u < end; ++u) {
      prev.assign(1, {n, 0});
      for (uint64_t s = g.off[u]; s < eo[u]; ++s) {
        const uint64_t v = g.nbr[s];
        if (v == u) {
          er[s] = s;
          prev.assign(1, {v, s});
          continue;
        }
        const uint64_t vb = eo[v], ve = g.off[v + 1];  // v's upper part (D5: probes stay inside)
        if (prev[0].first == v) {
          uint64_t rec = UINT64_MAX;
          if (prev.size() == 1) {
            const uint64_t po = prev[0].second;
            if (po + 1 < ve && g.nbr[po + 1] == u) rec = po + 1;
            else if (po > vb && g.nbr[po - 1] == u) rec = po - 1;
          } else {
            auto taken = [&](uint64_t r) {
              for (auto& pr : prev) if (pr.second == r) return true;
              return false;
            };
            uint64_t r = prev[0].second;
            while (r + 1 < ve && g.nbr[r + 1] == u) {
              ++r;
              if (!taken(r)) { rec = r; break; }
            }
            if (rec == UINT64_MAX) {
              r = prev[0].second;
              while (r > vb && g.nbr[r - 1] == u) {
                --r;
                if (!taken(r)) { rec = r; break; }
              }
            }
          }
          if (rec == UINT64_MAX) { status = ORC_E_INVALID; return; }
          prev.push_back({v, rec});
          er[s] = rec;
          er[rec] = s;
          continue;
        }
        // the reference's probe order (floor + (ceil - floor) / 2 with ceil
        // starting at off[v+1], which picks the copy of u it lands on); a probe
        // at off[v+1] itself, outside the row, ends the search (D5)
        uint64_t lo = vb, hi = ve, rec = UINT64_MAX;
        while (lo <= hi) {
          const uint64_t mid = lo + (hi - lo) / 2;
          if (mid >= ve) break;
          const uint64_t d = g.nbr[mid];
          if (d == u) { rec = mid; break; }
          if (d > u) {
            if (mid == vb) break;
            hi = mid - 1;
          } else {
            lo = mid + 1;
          }
        }
        if (rec == UINT64_MAX) { status = ORC_E_INVALID; return; }
        er[s] = rec;
        er[rec] = s;
        prev.assign(1, {v, rec});
      }
    }
  });
  if (status != ORC_OK) return status;
  // every slot must have been linked: an upper slot whose lower twin is missing
  // means the CSR is not symmetric
  uint64_t lower = 0, upper = 0;
  for (uint64_t u = 0; u < n; ++u) {
    for (uint64_t s = g.off[u]; s < g.off[u + 1]; ++s) {
      if (g.nbr[s] == u) continue;
      if (g.nbr[s] < u) ++lower; else ++upper;
    }
  }
  if (lower != upper) return ORC_E_INVALID;
  // a copy paired twice leaves another unpaired: each upper slot must be the
  // reciprocal of the lower slot that names it
  for (uint64_t u = 0; u < n; ++u)
    for (uint64_t s = g.off[u]; s < g.off[u + 1]; ++s)
      if (er[er[s]] != s) return ORC_E_INVALID;
  return ORC_OK;
}

// k_truss/triangles.rs:144-243.  Threads own vertex ranges (:159-168).  For
// each u: map the upper neighbours w > u to their slots (:172-191, all copies);
// for each lower slot u->v (v < u, v != u; :192-195) walk v's upper part
// backwards while w > u (:197-200); each copy u->w of a hit is the triangle
// v < u < w, credited on all six directed slots (:201-222).  Counters are u32;
// u8 mode keeps the low byte, which is what the reference's wrapping AtomicU8
// adds leave.
template <class Slots>
void triangles(const Csr& g, const uint64_t* eo, const uint64_t* er, int T, int u8mode,
               uint32_t* sup) {
  const uint64_t n = g.n, W = g.width();
  std::vector<std::atomic<uint32_t>> s(W);
  for (uint64_t i = 0; i < W; ++i) s[i].store(0, std::memory_order_relaxed);
  const uint64_t load = (n + T - 1) / T;
  run_threads(T, [&](int tid) {
    uint64_t begin = std::min<uint64_t>(tid * load, n), end = std::min<uint64_t>(begin + load, n);
    Slots map(n);
    for (uint64_t u = begin; u < end; ++u) {
      for (uint64_t j = eo[u]; j < g.off[u + 1]; ++j) map.put(g.nbr[j], j);
      for (uint64_t uv = g.off[u]; uv < eo[u]; ++uv) {
        uint64_t v = g.nbr[uv];
        if (v == u) continue;
        for (uint64_t vw = g.off[v + 1]; vw-- > eo[v];) {
          uint64_t w = g.nbr[vw];
          if (w <= u) break;
          uint64_t first, copies;
          if (!map.get(w, &first, &copies)) continue;
          for (uint64_t uw = first; uw < first + copies; ++uw) {
            const uint64_t slots[6] = {uv, vw, uw, er[uv], er[vw], er[uw]};
            for (uint64_t x : slots) s[x].fetch_add(1, std::memory_order_relaxed);
          }
        }
      }
      map.clear();
    }
  });
  for (uint64_t i = 0; i < W; ++i) {
    uint32_t v = s[i].load(std::memory_order_relaxed);
    sup[i] = u8mode ? (v & 0xFFu) : v;
  }
}

// Frontier queue with the semantics of shared_slice.rs:647-775 (push_slice
// appends a whole buffer at an atomically reserved index, pop hands out
// entries from the front, clear resets).  Capacity is width + 1 (defect D3).
struct Queue {
  std::vector<uint64_t> buf;
  std::atomic<uint64_t> read{0}, write{0}, len{0};
  explicit Queue(uint64_t cap) : buf(cap) {}
  bool push_slice(const uint64_t* p, uint64_t k) {
    uint64_t at = write.fetch_add(k);
    if (at + k < buf.size()) {
      std::memcpy(&buf[at], p, k * sizeof(uint64_t));
      len.fetch_add(k);
      return true;
    }
    write.fetch_sub(k);
    return false;
  }
  bool pop(uint64_t* out) {
    uint64_t x = read.load();
    while (x < len.load()) {
      if (read.compare_exchange_weak(x, x + 1)) { *out = buf[x]; return true; }
    }
    return false;
  }
  uint64_t size() const { return len.load(); }
  void clear() { read = 0; write = 0; len = 0; }
};

struct PktStats {
  uint64_t levels, sublevels, max_level;
};

// k_truss/pkt.rs:216-563, threads T (pkt.rs:223-224; edge ranges :289-290).
template <class Slots>
int pkt(const Csr& g, const uint64_t* er, const uint32_t* sup0, int T, int u8mode, uint32_t* truss,
        PktStats* st) {
  const uint64_t W = g.width();
  const uint64_t buff_size = 4096;  // pkt.rs:267
  std::vector<std::atomic<uint32_t>> s(W);
  for (uint64_t i = 0; i < W; ++i) s[i].store(sup0[i], std::memory_order_relaxed);
  std::vector<uint8_t> processed(W, 0), flags_a(W, 0), flags_b(W, 0);
  Queue qa(W + 1), qb(W + 1);
  Queue* curr = &qa;
  Queue* next = &qb;
  uint8_t* in_curr = flags_a.data();
  uint8_t* in_next = flags_b.data();
  std::atomic<uint64_t> duds{0};
  std::atomic<int> status{ORC_OK};
  std::atomic<uint64_t> levels{0}, sublevels{0}, max_level{0};
  std::barrier sync(T);
  const uint64_t load = (W + T - 1) / T;

  run_threads(T, [&](int tid) {
    uint64_t begin = std::min<uint64_t>(tid * load, W), end = std::min<uint64_t>(begin + load, W);
    std::vector<uint64_t> buff(buff_size);
    uint64_t nb = 0;
    auto flush = [&](Queue* q) {
      if (nb && !q->push_slice(buff.data(), nb)) status = ORC_E_QUEUE;
      nb = 0;
    };
    auto add = [&](Queue* q, uint64_t e) {
      buff[nb++] = e;
      if (nb == buff_size) flush(q);
    };
    // zero-support slots are done at level 0 (:298-306)
    uint64_t local_duds = 0;
    for (uint64_t e = begin; e < end; ++e)
      if (s[e].load(std::memory_order_relaxed) == 0) { processed[e] = 1; ++local_duds; }
    duds += local_duds;
    sync.arrive_and_wait();
    uint64_t todo = W - duds.load();
    uint64_t l = 1;  // the reference's `l: u8`; u8 mode errors on overflow
    Slots map(g.n);
    while (todo > 0 && status == ORC_OK) {
      // level scan (:325-339)
      for (uint64_t e = begin; e < end; ++e) {
        if (s[e].load(std::memory_order_relaxed) == l) {
          in_curr[e] = 1;
          add(curr, e);
        }
      }
      flush(curr);
      sync.arrive_and_wait();
      if (tid == 0 && curr->size() > 0) { levels++; max_level = l; }
      while (curr->size() > 0) {
        todo -= curr->size();
        const uint64_t len = curr->size();
        const uint64_t* to_process = curr->buf.data();
        if (tid == 0) sublevels++;
        sync.arrive_and_wait();
        uint64_t uv;
        while (curr->pop(&uv)) {  // ProcessSubLevel (:366-484)
          uint64_t u = g.nbr[er[uv]], v = g.nbr[uv];
          for (uint64_t uw = g.off[u]; uw < g.off[u + 1]; ++uw) {
            uint64_t w = g.nbr[uw];
            if (w != u && w != v) map.put(w, uw);
          }
          auto dec = [&](uint64_t x) {
            uint32_t prev = s[x].fetch_sub(1, std::memory_order_relaxed);
            if (prev == l + 1) { in_next[x] = 1; add(next, x); }
            if (prev <= l) s[x].store((uint32_t)l, std::memory_order_relaxed);
          };
          for (uint64_t vw = g.off[v]; vw < g.off[v + 1]; ++vw) {
            uint64_t w = g.nbr[vw], first, copies;
            if (!map.get(w, &first, &copies)) continue;
            for (uint64_t uw = first; uw < first + copies; ++uw) {  // pkt.rs:404-409
              uint64_t wu = er[uw];
              if (processed[vw] || processed[wu]) continue;
              uint32_t s_vw = s[vw].load(std::memory_order_relaxed);
              uint32_t s_wu = s[wu].load(std::memory_order_relaxed);
              if (s_vw > l && s_wu > l) {
                dec(vw);
                dec(wu);
              } else if (s_vw > l && (uv < wu || !in_curr[wu])) {
                dec(vw);
              } else if (s_wu > l && (uv < vw || !in_curr[vw])) {
                dec(wu);
              }
            }
          }
          map.clear();
        }
        flush(next);
        sync.arrive_and_wait();  // D2: every thread has finished the sub-level
        const uint64_t share = (len + T - 1) / T;
        const uint64_t pb = std::min<uint64_t>(tid * share, len), pe = std::min<uint64_t>(pb + share, len);
        for (uint64_t i = pb; i < pe; ++i) {
          uint64_t e = to_process[i];
          processed[e] = 1;
          in_curr[e] = 0;  // D1: the edge's flag, not position i's
        }
        sync.arrive_and_wait();
        if (tid == 0) {
          curr->clear();
          std::swap(curr, next);
          std::swap(in_curr, in_next);
        }
        sync.arrive_and_wait();
      }
      ++l;
      if (u8mode && l > 255) status = ORC_E_OVERFLOW;  // :508-516
      sync.arrive_and_wait();
    }
  });
  if (status != ORC_OK) return status;
  for (uint64_t e = 0; e < W; ++e) {
    uint32_t v = s[e].load(std::memory_order_relaxed) + 2;  // :524-526
    truss[e] = u8mode ? (v & 0xFFu) : v;
  }
  if (st) { st->levels = levels; st->sublevels = sublevels; st->max_level = max_level; }
  return ORC_OK;
}

// k_truss/burkhardt_et_al.rs:186-380: sequential.  Level k scans the live
// slot list: count == k -> push (u, slot) (:246-254); count == 0 -> swap-
// remove from the live list with truss k + 1 (:255-277).  Popping a slot
// zeroes its count (:291) and charges each triangle whose two other slots are
// still non-zero (:321-356), pushing a slot whose count drops from k + 1.
// u8 mode runs k over 1..255 exclusive (:238) like the reference; wide mode
// runs until the live list is empty.
template <class Slots>
int burkhardt(const Csr& g, const uint64_t* er, const uint32_t* sup0, int u8mode, uint32_t* truss) {
  const uint64_t W = g.width();
  std::vector<uint32_t> tris(sup0, sup0 + W);
  std::vector<uint64_t> edges(W), edge_index(W);
  for (uint64_t i = 0; i < W; ++i) { truss[i] = 2; edges[i] = i; edge_index[i] = i; }
  std::vector<std::pair<uint64_t, uint64_t>> stack;
  stack.reserve(1024);
  uint64_t edge_count = W;
  Slots map(g.n);
  for (uint64_t k = 1; !u8mode || k < 255; ++k) {
    if (edge_count == 0) break;
    uint64_t idx = 0;
    while (idx < edge_count) {
      uint64_t e = edge_index[idx];
      uint32_t t = tris[e];
      if (t == k) {
        stack.push_back({g.nbr[er[e]], e});
        ++idx;
      } else if (t == 0) {
        --edge_count;
        uint64_t e_index = edge_index[edge_count];
        uint64_t r_index = edges[e];
        edge_index[edge_count] = edge_index[r_index];
        edge_index[r_index] = e_index;
        edges[e] = edge_count;
        edges[e_index] = r_index;
        truss[e] = u8mode ? (uint32_t)((k + 1) & 0xFF) : (uint32_t)(k + 1);
      } else {
        ++idx;
      }
    }
    while (!stack.empty()) {
      auto [u, off] = stack.back();
      stack.pop_back();
      tris[off] = 0;
      uint64_t v = g.nbr[off];
      for (uint64_t uw = g.off[u]; uw < g.off[u + 1]; ++uw) {
        uint64_t w = g.nbr[uw];
        if (w != u && w != v) map.put(w, uw);
      }
      for (uint64_t vw = g.off[v]; vw < g.off[v + 1]; ++vw) {
        uint64_t w = g.nbr[vw], first, copies;
        if (!map.get(w, &first, &copies)) continue;
        for (uint64_t uw = first; uw < first + copies; ++uw) {  // :321-356, every copy
          uint64_t wu = er[uw];
          if (tris[vw] != 0 && tris[wu] != 0) {
            uint32_t p = tris[wu]--;
            if (u8mode) tris[wu] &= 0xFF;
            if (p == k + 1) stack.push_back({w, wu});
            p = tris[vw]--;
            if (u8mode) tris[vw] &= 0xFF;
            if (p == k + 1) stack.push_back({v, vw});
          }
        }
      }
      map.clear();
    }
  }
  return ORC_OK;
}

// Sorted-list intersection of the rows of u and v, excluding u and v:
// f(i, ci, j, cj) for every common neighbour w, with [i, i + ci) its copies in
// u's row and [j, j + cj) in v's (ci = cj = 1 in a simple graph).  Rows of
// similar length are merged; otherwise each neighbour of the shorter row is
// binary-searched in the longer one (a hub row of 10^5 entries is not walked
// once per incident edge).
template <class F>
void for_common(const Csr& g, uint64_t u, uint64_t v, F&& f) {
  uint64_t i = g.off[u], ie = g.off[u + 1], j = g.off[v], je = g.off[v + 1];
  auto run = [&](uint64_t x, uint64_t end) {
    uint64_t y = x + 1;
    while (y < end && g.nbr[y] == g.nbr[x]) ++y;
    return y - x;
  };
  const uint64_t du = ie - i, dv = je - j;
  if (du * 16 < dv || dv * 16 < du) {
    const bool u_short = du <= dv;
    const uint64_t sb = u_short ? i : j, se = u_short ? ie : je;
    const uint64_t lb = u_short ? j : i, le = u_short ? je : ie;
    for (uint64_t x = sb; x < se;) {
      const uint32_t w = g.nbr[x];
      const uint64_t cx = run(x, se);
      if (w != u && w != v) {
        uint64_t lo = lb, hi = le;
        while (lo < hi) {
          const uint64_t mid = lo + (hi - lo) / 2;
          if (g.nbr[mid] < w) lo = mid + 1; else hi = mid;
        }
        if (lo < le && g.nbr[lo] == w) {
          const uint64_t cl = run(lo, le);
          if (u_short) f(x, cx, lo, cl); else f(lo, cl, x, cx);
        }
      }
      x += cx;
    }
    return;
  }
  while (i < ie && j < je) {
    uint32_t a = g.nbr[i], b = g.nbr[j];
    if (a < b) ++i;
    else if (b < a) ++j;
    else {
      const uint64_t ci = run(i, ie), cj = run(j, je);
      if (a != u && a != v) f(i, ci, j, cj);
      i += ci;
      j += cj;
    }
  }
}

// k_truss/mod.rs:30-216, corrected.  The reference checks, for each slot with
// stored truss k, support_{>=k} >= k (:176-184) and support_{>=k+1} < k+1
// (:188-197); with k = support level + 2 (pkt.rs:525) those bounds are off by
// two, so every graph with an edge fails (a 2-truss edge has 0 < 2).  Here:
// symmetric truss on both slots, the same truss on every copy of a parallel
// edge; support among edges with truss >= k is at least k - 2 (membership);
// support among edges with truss >= k + 1 is below k - 1 (local maximality).
// A common neighbour w counts once per choice of copies of u-w and v-w (the
// reference's triangle count in a multigraph).  Returns the smallest failing
// slot + 1, or 0.
// Vertices are handed out dynamically (hub rows would otherwise leave one
// thread with most of the work).
uint64_t verify(const Csr& g, const uint64_t* er, const uint32_t* truss, int T) {
  const uint64_t n = g.n;
  std::atomic<uint64_t> bad{UINT64_MAX};
  auto fail = [&](uint64_t s) {
    uint64_t cur = bad.load();
    while (s < cur && !bad.compare_exchange_weak(cur, s)) {}
  };
#pragma omp parallel for schedule(dynamic, 64) num_threads(T)
  for (uint64_t u = 0; u < n; ++u) {
    for (uint64_t s = g.off[u]; s < g.off[u + 1]; ++s) {
      uint64_t v = g.nbr[s];
      if (v == u) {
        if (truss[s] != 2) fail(s);
        continue;
      }
      if (v < u) continue;
      uint32_t k = truss[s];
      if (truss[er[s]] != k || k < 2) { fail(s); continue; }
      if (s > g.off[u] && g.nbr[s - 1] == v) {  // a later copy: same truss as the first
        if (truss[s - 1] != k) fail(s);
        continue;
      }
      uint64_t in_k = 0, in_k1 = 0;
      bool mixed = false;
      for_common(g, u, v, [&](uint64_t i, uint64_t ci, uint64_t j, uint64_t cj) {
        uint32_t a = truss[i], b = truss[j];
        for (uint64_t x = 1; x < ci; ++x) mixed |= truss[i + x] != a;
        for (uint64_t x = 1; x < cj; ++x) mixed |= truss[j + x] != b;
        if (a >= k && b >= k) in_k += ci * cj;
        if (a >= k + 1 && b >= k + 1) in_k1 += ci * cj;
      });
      if (mixed) { fail(s); continue; }
      if (in_k + 2 < k || in_k1 + 1 >= k) fail(s);
    }
  }
  const uint64_t b = bad.load();
  return b == UINT64_MAX ? 0 : b + 1;
}

// Independent exact truss decomposition (no reference counterpart), used for
// the workloads the restatements are too slow for.  Support per undirected
// edge by degree-oriented merge intersection; then a level-synchronous peel:
// every triangle of a peeled edge is resolved on edge ids -- a triangle
// charges its surviving edges once, when its first edge is peeled, and ties
// inside one frontier go to the smallest id.  Rows are rebuilt without
// peeled edges whenever the live edge count halves.
//
// Multigraphs: the rows are first reduced to distinct neighbours with a
// multiplicity mu per pair (all copies of a pair are interchangeable, so they
// share one truss number); a triangle of pairs (e, f, h) then stands for
// mu_e * mu_f * mu_h triangles of copies: a copy of e lies in mu_f * mu_h of
// them, and peeling e removes mu_e * mu_h from each copy of f.  This weighted
// peel shares no code with the copy-by-copy restatements above.
int fast_truss_core(const Csr& g, const uint32_t* mult, int T, int u8mode, uint32_t* truss_out,
                    uint64_t* tri_out, uint64_t* levels_out) {
  const uint64_t n = g.n, W = g.width();
  omp_set_num_threads(T);
  auto deg = [&](uint64_t x) { return g.off[x + 1] - g.off[x]; };
  auto before = [&](uint64_t a, uint64_t b) {
    uint64_t da = deg(a), db = deg(b);
    return da < db || (da == db && a < b);
  };
  // undirected edge ids: upper slots (u < v) in CSR order
  std::vector<uint64_t> upc(n + 1, 0);
#pragma omp parallel for schedule(static)
  for (uint64_t u = 0; u < n; ++u) {
    uint64_t c = 0;
    for (uint64_t s = g.off[u]; s < g.off[u + 1]; ++s) c += g.nbr[s] > u;
    upc[u + 1] = c;
  }
  for (uint64_t u = 0; u < n; ++u) upc[u + 1] += upc[u];
  const uint64_t m = upc[n];
  std::vector<uint64_t> eid(W, UINT64_MAX);
  std::vector<uint32_t> src(m), dst(m);
  std::vector<int64_t> mu(m, 1);
  std::atomic<int> bad{0};
#pragma omp parallel for schedule(static)
  for (uint64_t u = 0; u < n; ++u) {
    uint64_t p = upc[u];
    for (uint64_t s = g.off[u]; s < g.off[u + 1]; ++s)
      if (g.nbr[s] > u) {
        eid[s] = p; src[p] = (uint32_t)u; dst[p] = g.nbr[s];
        if (mult) mu[p] = mult[s];
        ++p;
      }
  }
#pragma omp parallel for schedule(dynamic, 1024)
  for (uint64_t u = 0; u < n; ++u)
    for (uint64_t s = g.off[u]; s < g.off[u + 1]; ++s) {
      uint64_t v = g.nbr[s];
      if (v >= u) continue;
      uint64_t lo = g.off[v], hi = g.off[v + 1];
      while (lo < hi) { uint64_t mid = (lo + hi) / 2; if (g.nbr[mid] < u) lo = mid + 1; else hi = mid; }
      if (lo == g.off[v + 1] || g.nbr[lo] != u) { bad = 1; continue; }
      eid[s] = eid[lo];
    }
  if (bad) return ORC_E_INVALID;
  // oriented out-lists (vertex ids ascending), with edge ids
  std::vector<uint64_t> opos(n + 1, 0);
#pragma omp parallel for schedule(static)
  for (uint64_t u = 0; u < n; ++u) {
    uint64_t c = 0;
    for (uint64_t s = g.off[u]; s < g.off[u + 1]; ++s)
      if (g.nbr[s] != u && before(u, g.nbr[s])) ++c;
    opos[u + 1] = c;
  }
  for (uint64_t u = 0; u < n; ++u) opos[u + 1] += opos[u];
  std::vector<uint32_t> ocol(m);
  std::vector<uint64_t> oeid(m);
#pragma omp parallel for schedule(static)
  for (uint64_t u = 0; u < n; ++u) {
    uint64_t p = opos[u];
    for (uint64_t s = g.off[u]; s < g.off[u + 1]; ++s)
      if (g.nbr[s] != u && before(u, g.nbr[s])) { ocol[p] = g.nbr[s]; oeid[p] = eid[s]; ++p; }
  }
  std::vector<std::atomic<int64_t>> as(m);
#pragma omp parallel for schedule(static)
  for (uint64_t e = 0; e < m; ++e) as[e].store(0, std::memory_order_relaxed);
  uint64_t tri = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : tri)
  for (uint64_t a = 0; a < n; ++a) {
    for (uint64_t p = opos[a]; p < opos[a + 1]; ++p) {
      uint64_t b = ocol[p];
      uint64_t i = opos[a], ie = opos[a + 1], j = opos[b], je = opos[b + 1];
      int64_t cnt = 0;
      const int64_t mp = mu[oeid[p]];
      while (i < ie && j < je) {
        if (ocol[i] < ocol[j]) ++i;
        else if (ocol[j] < ocol[i]) ++j;
        else {
          const int64_t mi = mu[oeid[i]], mj = mu[oeid[j]];
          cnt += mi * mj;
          as[oeid[i]].fetch_add(mp * mj, std::memory_order_relaxed);
          as[oeid[j]].fetch_add(mp * mi, std::memory_order_relaxed);
          ++i; ++j;
        }
      }
      if (cnt) as[oeid[p]].fetch_add(cnt, std::memory_order_relaxed);
      tri += (uint64_t)(cnt * mp);
    }
  }
  if (tri_out) *tri_out = tri;
  std::vector<int64_t> s(m);
#pragma omp parallel for schedule(static)
  for (uint64_t e = 0; e < m; ++e) {
    int64_t v = as[e].load(std::memory_order_relaxed);
    if (u8mode) v &= 0xFF;
    s[e] = v;
    as[e].store(v, std::memory_order_relaxed);
  }
  // live adjacency (rows of live edges: neighbour + edge id), rebuilt as edges die
  std::vector<uint8_t> state(m, 0);  // 0 live, 1 frontier, 2 done
  for (uint64_t e = 0; e < m; ++e) if (s[e] == 0) state[e] = 2;
  std::vector<uint64_t> loff(n + 1);
  std::vector<uint32_t> lnbr;
  std::vector<uint64_t> leid;
  uint64_t live_in_rows = 0;
  auto rebuild = [&]() {
    std::vector<uint64_t> cnt(n + 1, 0);
#pragma omp parallel for schedule(static)
    for (uint64_t u = 0; u < n; ++u) {
      uint64_t c = 0;
      for (uint64_t x = g.off[u]; x < g.off[u + 1]; ++x) c += eid[x] != UINT64_MAX && state[eid[x]] != 2;
      cnt[u + 1] = c;
    }
    for (uint64_t u = 0; u < n; ++u) cnt[u + 1] += cnt[u];
    loff = cnt;
    lnbr.assign(loff[n], 0);
    leid.assign(loff[n], 0);
#pragma omp parallel for schedule(static)
    for (uint64_t u = 0; u < n; ++u) {
      uint64_t p = loff[u];
      for (uint64_t x = g.off[u]; x < g.off[u + 1]; ++x)
        if (eid[x] != UINT64_MAX && state[eid[x]] != 2) { lnbr[p] = g.nbr[x]; leid[p] = eid[x]; ++p; }
    }
    live_in_rows = loff[n] / 2;
  };
  rebuild();
  std::vector<uint64_t> live, frontier, nextf;
  for (uint64_t e = 0; e < m; ++e) if (state[e] == 0) live.push_back(e);
  uint64_t levels = 0;
  int64_t l = 0;
  std::vector<std::vector<uint64_t>> pushed(T);
  while (!live.empty()) {
    if (live.size() * 2 < live_in_rows) rebuild();
    int64_t mn = INT64_MAX;
#pragma omp parallel for schedule(static) reduction(min : mn)
    for (uint64_t i = 0; i < live.size(); ++i) mn = std::min<int64_t>(mn, as[live[i]].load(std::memory_order_relaxed));
    l = mn;
    if (u8mode && l > 254) return ORC_E_OVERFLOW;
    frontier.clear();
    std::vector<uint64_t> keep;
    for (uint64_t e : live) {
      if (as[e].load(std::memory_order_relaxed) <= l) { frontier.push_back(e); state[e] = 1; }
      else keep.push_back(e);
    }
    live.swap(keep);
    ++levels;
    while (!frontier.empty()) {
      for (auto& p : pushed) p.clear();
#pragma omp parallel
      {
        std::vector<uint64_t>& mine = pushed[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 16)
        for (uint64_t k = 0; k < frontier.size(); ++k) {
          uint64_t e = frontier[k];
          uint64_t u = src[e], v = dst[e];
          uint64_t du = loff[u + 1] - loff[u], dv = loff[v + 1] - loff[v];
          uint64_t small = du <= dv ? u : v, large = small == u ? v : u;
          for (uint64_t si = loff[small]; si < loff[small + 1]; ++si) {
            uint64_t w = lnbr[si];
            if (w == u || w == v) continue;
            uint64_t lo = loff[large], hi = loff[large + 1];
            while (lo < hi) { uint64_t mid = (lo + hi) / 2; if (lnbr[mid] < w) lo = mid + 1; else hi = mid; }
            if (lo == loff[large + 1] || lnbr[lo] != w) continue;
            uint64_t f = leid[si], h = leid[lo];
            if (state[f] == 2 || state[h] == 2) continue;
            bool fin = state[f] == 1, hin = state[h] == 1;
            if (fin && f < e) continue;
            if (hin && h < e) continue;
            auto dec = [&](uint64_t x, int64_t d) {
              int64_t prev = as[x].fetch_sub(d, std::memory_order_relaxed);
              if (prev > l && prev - d <= l) mine.push_back(x);
            };
            if (!fin && as[f].load(std::memory_order_relaxed) > l) dec(f, mu[e] * mu[h]);
            if (!hin && as[h].load(std::memory_order_relaxed) > l) dec(h, mu[e] * mu[f]);
          }
        }
      }
      for (uint64_t e : frontier) { state[e] = 2; s[e] = l; }
      nextf.clear();
      for (auto& p : pushed) nextf.insert(nextf.end(), p.begin(), p.end());
      for (uint64_t e : nextf) state[e] = 1;
      frontier.swap(nextf);
    }
    std::vector<uint64_t> keep2;
    keep2.reserve(live.size());
    for (uint64_t e : live) if (state[e] == 0) keep2.push_back(e);
    live.swap(keep2);
  }
  if (levels_out) *levels_out = levels;
#pragma omp parallel for schedule(static)
  for (uint64_t x = 0; x < W; ++x) {
    uint64_t e = eid[x];
    uint64_t v = (e == UINT64_MAX) ? 2 : (uint64_t)s[e] + 2;
    truss_out[x] = u8mode ? (uint32_t)(v & 0xFF) : (uint32_t)v;
  }
  return ORC_OK;
}

// Multigraph front end of fast_truss_core: distinct neighbours per row with
// their multiplicities, then every copy takes its pair's truss number.
int fast_truss(const Csr& g, bool multi, int T, int u8mode, uint32_t* truss_out, uint64_t* tri_out,
               uint64_t* levels_out) {
  if (!multi) return fast_truss_core(g, nullptr, T, u8mode, truss_out, tri_out, levels_out);
  const uint64_t n = g.n, W = g.width();
  std::vector<uint64_t> off2(n + 1, 0);
  for (uint64_t u = 0; u < n; ++u) {
    uint64_t c = 0;
    for (uint64_t s = g.off[u]; s < g.off[u + 1]; ++s) c += s == g.off[u] || g.nbr[s] != g.nbr[s - 1];
    off2[u + 1] = off2[u] + c;
  }
  std::vector<uint32_t> nbr2(off2[n]), mult(off2[n], 0);
  std::vector<uint64_t> to2(W);
  for (uint64_t u = 0; u < n; ++u) {
    uint64_t p = off2[u];
    for (uint64_t s = g.off[u]; s < g.off[u + 1]; ++s) {
      if (s > g.off[u] && g.nbr[s] == g.nbr[s - 1]) --p;
      nbr2[p] = g.nbr[s];
      ++mult[p];
      to2[s] = p;
      ++p;
    }
  }
  std::vector<uint32_t> t2(off2[n]);
  const int rc = fast_truss_core(Csr{n, off2.data(), nbr2.data()}, mult.data(), T, u8mode, t2.data(), tri_out,
                                 levels_out);
  if (rc) return rc;
  for (uint64_t s = 0; s < W; ++s) truss_out[s] = t2[to2[s]];
  return ORC_OK;
}

}  // namespace

extern "C" {

int orc_validate(uint64_t n, const uint64_t* off, const uint32_t* nbr) {
  return validate(Csr{n, off, nbr});
}

int orc_edge_index(uint64_t n, const uint64_t* off, const uint32_t* nbr, uint64_t* eo, uint64_t* er,
                   int threads) {
  Csr g{n, off, nbr};
  int rc = validate(g);
  if (rc) return rc;
  return edge_index(g, eo, er, threads < 1 ? 1 : threads);
}

// hash = 1 uses std::unordered_map like the reference's HashMap; 0 a dense array.
int orc_triangles(uint64_t n, const uint64_t* off, const uint32_t* nbr, const uint64_t* eo,
                  const uint64_t* er, int threads, int u8mode, int hash, uint32_t* sup) {
  Csr g{n, off, nbr};
  threads = threads < 1 ? 1 : threads;
  if (hash) triangles<HashSlots>(g, eo, er, threads, u8mode, sup);
  else triangles<DenseSlots>(g, eo, er, threads, u8mode, sup);
  return ORC_OK;
}

int orc_pkt(uint64_t n, const uint64_t* off, const uint32_t* nbr, const uint64_t* er,
            const uint32_t* sup, int threads, int u8mode, int hash, uint32_t* truss,
            uint64_t* stats3) {
  Csr g{n, off, nbr};
  PktStats st{};
  threads = threads < 1 ? 1 : threads;
  int rc = hash ? pkt<HashSlots>(g, er, sup, threads, u8mode, truss, &st)
                : pkt<DenseSlots>(g, er, sup, threads, u8mode, truss, &st);
  if (stats3) { stats3[0] = st.levels; stats3[1] = st.sublevels; stats3[2] = st.max_level; }
  return rc;
}

int orc_burkhardt(uint64_t n, const uint64_t* off, const uint32_t* nbr, const uint64_t* er,
                  const uint32_t* sup, int u8mode, int hash, uint32_t* truss) {
  Csr g{n, off, nbr};
  return hash ? burkhardt<HashSlots>(g, er, sup, u8mode, truss)
              : burkhardt<DenseSlots>(g, er, sup, u8mode, truss);
}

uint64_t orc_verify(uint64_t n, const uint64_t* off, const uint32_t* nbr, const uint64_t* er,
                    const uint32_t* truss, int threads) {
  return verify(Csr{n, off, nbr}, er, truss, threads < 1 ? 1 : threads);
}

int orc_fast_truss(uint64_t n, const uint64_t* off, const uint32_t* nbr, int threads, int u8mode,
                   uint32_t* truss, uint64_t* triangles, uint64_t* levels) {
  Csr g{n, off, nbr};
  bool multi = false;
  int rc = validate(g, &multi);
  if (rc) return rc;
  return fast_truss(g, multi, threads < 1 ? 1 : threads, u8mode, truss, triangles, levels);
}

}  // extern "C"
