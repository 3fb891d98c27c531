// Per-child selection and variation of one steady-state round
// (crossover_child / mutate_child / compare_child,
// cpp/src/evolution/repro/gpu/phase_operators.cuh:46-265), one warp per
// child over rows staged in shared memory.  Every lane draws the same random
// numbers (the reference's Warp=true contract); lanes split copies, counts
// and scans.  One whole-program phase per member (slot_count == 1), so the
// uniform-phase draw is bounded(1) and a row is a member.
#pragma once
#include "device_ops.cuh"

namespace gb {

// A tournament entrant: its key, tie-break and member; `live` false for a
// lane that holds no draw.  Keys pack (-fitness, wrong, nodes), smaller is
// better.  For metrics with wrong counts the reference's selection values are
// ranks (evolve.cpp:285,361), and of two members with equal keys the one of
// smaller index holds the better rank; otherwise they are the fitness values,
// and equal keys are equal selection values.
struct Entrant {
  uint64_t key;
  uint32_t tie;
  int member;
  bool live;
};
__device__ __forceinline__ bool entrant_better(const Entrant& a, const Entrant& b) {
  return a.live && (!b.live || a.key < b.key || (a.key == b.key && a.tie < b.tie));
}
__device__ __forceinline__ Entrant warp_best_entrant(Entrant e) {
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    Entrant f;
    f.key = __shfl_xor_sync(kFull, e.key, o);
    f.tie = __shfl_xor_sync(kFull, e.tie, o);
    f.member = __shfl_xor_sync(kFull, e.member, o);
    f.live = __shfl_xor_sync(kFull, int(e.live), o) != 0;
    if (entrant_better(f, e)) e = f;
  }
  return e;
}

// The parent's and the donor's tournaments, one after the other on `random`
// (crossover_child's two tournament calls, phase_operators.cuh:46-50,
// 135-136), with their key loads in flight together.  Every lane draws the
// same 2 x pressure members in order and lane j keeps draw j of each chunk
// of 32.  The sequential tournament replaces its best only by a strictly
// better selection value or, for rank values, an equal one of smaller member
// index, so its winner is the entrant of the smallest (key, tie): tie = the
// member index for rank values, the draw position otherwise.
__device__ inline void warp_tournaments(const SearchDesc& s, Rng& random, int* parent, int* donor) {
  const int lane = lane_id();
  const int p = s.pressure, total = 2 * p;
  if (p <= 16) {
    // both tournaments in aligned power-of-two lane segments (the parent's
    // entrants from lane 0, the donor's from lane `seg`): log2(seg) steps of
    // a segmented shuffle reduction, then each winner from its lane
    int seg = 1;
    while (seg < p) seg <<= 1;
    int mine = 0;
    for (int j = 0; j < total; ++j) {
      const int d = int(random.bounded_fixed(uint64_t(s.P), s.bounded_threshold, s.mod_magic));
      if ((j < p ? j : seg + j - p) == lane) mine = d;
    }
    const int position = lane < seg ? lane : lane - seg;
    const bool live = lane < 2 * seg && position < p;
    uint64_t key = live ? s.key[mine] : ~0ULL;
    uint32_t tie = live ? (s.has_wrong ? uint32_t(mine) : uint32_t(position)) : ~0u;
    int from = lane;
    for (int o = 1; o < seg; o <<= 1) {
      const uint64_t k2 = __shfl_xor_sync(kFull, key, o);
      const uint32_t t2 = __shfl_xor_sync(kFull, tie, o);
      const int f2 = __shfl_xor_sync(kFull, from, o);
      if (k2 < key || (k2 == key && t2 < tie)) {
        key = k2;
        tie = t2;
        from = f2;
      }
    }
    const int parent_lane = __shfl_sync(kFull, from, 0), donor_lane = __shfl_sync(kFull, from, seg);
    *parent = __shfl_sync(kFull, mine, parent_lane);
    *donor = __shfl_sync(kFull, mine, donor_lane);
    return;
  }
  Entrant best[2] = {{0, 0, 0, false}, {0, 0, 0, false}};
  for (int base = 0; base < total; base += 32) {
    const int n = min(32, total - base);
    int mine = 0;
    for (int j = 0; j < n; ++j) {
      const int d = int(random.bounded_fixed(uint64_t(s.P), s.bounded_threshold, s.mod_magic));
      if (j == lane) mine = d;
    }
    const int position = base + lane;
    const int which = position < p ? 0 : 1;
    const uint64_t key = lane < n ? s.key[mine] : 0;
    for (int t = 0; t < 2; ++t) {
      const Entrant e{key, s.has_wrong ? uint32_t(mine) : uint32_t(position - t * p), mine, lane < n && which == t};
      const Entrant w = warp_best_entrant(e);
      if (entrant_better(w, best[t])) best[t] = w;
    }
  }
  *parent = best[0].member;
  *donor = best[1].member;
}

// Shared-memory rows of one warp: parent, donor, child, splice output,
// generated subtree; `pending` is the generator's task stack.
struct WarpRows {
  SRow parent, donor, child, out, gen;
  uint64_t* pending;
};

__host__ __device__ __forceinline__ size_t warp_rows_bytes(int stride) {
  return size_t(5) * stride * (sizeof(uint64_t) + sizeof(int64_t)) + 192 * sizeof(uint64_t);
}
__device__ inline WarpRows carve_rows(char* base, int stride) {
  WarpRows r;
  uint64_t* n = reinterpret_cast<uint64_t*>(base);
  int64_t* c = reinterpret_cast<int64_t*>(n + 5 * stride);
  r.parent = SRow{n, c, 0, 0};
  r.donor = SRow{n + stride, c + stride, 0, 0};
  r.child = SRow{n + 2 * stride, c + 2 * stride, 0, 0};
  r.out = SRow{n + 3 * stride, c + 3 * stride, 0, 0};
  r.gen = SRow{n + 4 * stride, c + 4 * stride, 0, 0};
  r.pending = reinterpret_cast<uint64_t*>(c + 5 * stride);
  return r;
}

// The parent's and the donor's rows into shared memory.  Every member row
// holds `stride` words, so the whole stride is copied without waiting for
// the lengths: the row loads and the length loads are in flight together.
__device__ inline void load_members(const SearchDesc& s, int a, SRow& to_a, int b, SRow& to_b) {
  const int32_t la = s.len[a], lb = s.len[b];
  const uint64_t* na = s.node + size_t(a) * s.stride;
  const uint64_t* nb = s.node + size_t(b) * s.stride;
  const int64_t* ca = s.cval + size_t(a) * s.stride;
  const int64_t* cb = s.cval + size_t(b) * s.stride;
  for (int i = lane_id(); i < s.stride; i += 32) {
    const uint64_t x = na[i], y = nb[i];
    const int64_t u = ca[i], v = cb[i];
    to_a.node[i] = x;
    to_b.node[i] = y;
    to_a.cval[i] = u;
    to_b.cval[i] = v;
  }
  to_a.n = len_nodes(la);
  to_a.nc = len_consts(la);
  to_b.n = len_nodes(lb);
  to_b.nc = len_consts(lb);
  __syncwarp();
}

// Hash of a row's genotype (construction expressions and constants): a
// wrap-around sum over positions of a mixed (value, position) word, so that
// the lanes hash their strided elements independently.  Equality of rows
// decides a reuse; the hash only picks candidates, as the reference's
// serial FNV-style fold does (parent_cache::hash_program,
// parent_fitness_cache.cuh:15-31).  Every lane returns the same hash.
__device__ inline uint64_t warp_row_hash(const uint64_t* node, const int64_t* cval, int n, int nc) {
  const int lane = lane_id();
  uint64_t acc = 0;
  for (int i = lane; i < n; i += 32) acc += mix64(uint64_t(w_origin(node[i])) | (uint64_t(i) << 32));
  for (int i = lane; i < nc; i += 32) acc += mix64(uint64_t(cval[i]) ^ mix64(0x5bd1e995ULL + uint64_t(i)));
#pragma unroll
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
  return mix64(acc ^ (uint64_t(n) << 40) ^ (uint64_t(nc) << 20));
}

// Genotype equality of two rows (parent_cache::equal_program,
// parent_fitness_cache.cuh:33-48): lengths, construction expressions (every
// other node field is a function of them) and constants.
__device__ inline bool warp_rows_equal(const uint64_t* an, const int64_t* ac, int a_n, int a_nc, const uint64_t* bn,
                                       const int64_t* bc, int b_n, int b_nc) {
  if (a_n != b_n || a_nc != b_nc) return false;
  bool same = true;
  for (int i = lane_id(); i < a_n; i += 32) same &= w_origin(an[i]) == w_origin(bn[i]);
  for (int i = lane_id(); i < a_nc; i += 32) same &= ac[i] == bc[i];
  return __all_sync(kFull, same);
}

// Member index slot words: the row hash's top 44 bits and member + 1
// (members below 2^20; 0 marks an empty slot).
__device__ __forceinline__ unsigned long long index_word(uint64_t h, int m) {
  return ((h >> 20) << 20) | (unsigned long long)(m + 1);
}
__device__ __forceinline__ int index_member(unsigned long long w) { return int(w & 0xfffffu) - 1; }
__device__ __forceinline__ bool index_tag_matches(unsigned long long w, uint64_t h) { return (w >> 20) == (h >> 20); }

// A current member identical to `row` (the member_hashes lookup of
// HostPhasePopulation::make_batch, phase_population_cpu.cpp:336-339): the
// round's member index holds one member per distinct row, probed linearly
// from the row's hash up to an empty slot.  Which identical member is found
// does not matter: identical programs score the same.  -1: none.
__device__ inline int warp_find_member(const SearchDesc& s, const SRow& row) {
  const uint64_t h = warp_row_hash(row.node, row.cval, row.n, row.nc);
  const uint32_t mask = uint32_t(s.mtab_mask);
  uint32_t slot = uint32_t(h) & mask;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    const unsigned long long w = s.mtab[slot];
    if (!w) return -1;
    if (index_tag_matches(w, h)) {
      const int m = index_member(w);
      const int32_t l = s.len[m];
      if (warp_rows_equal(s.node + size_t(m) * s.stride, s.cval + size_t(m) * s.stride, len_nodes(l), len_consts(l),
                          row.node, row.cval, row.n, row.nc))
        return m;
    }
    slot = (slot + 1) & mask;
  }
  return -1;
}

// locals_defined of a row of node words, for a statement program (true for
// a value phase, whose reads are inputs and binders only).  Out of line: the
// walk's frame stack stays out of the variation kernel's own frame.
__device__ __noinline__ bool row_locals_defined(const SearchDesc& s, const uint64_t* node, int n) {
  return locals_defined(n, [&](int i) {
    const uint64_t w = node[i];
    const ExprInfo& x = s.info[w_origin(w)];
    return StatementNode{x.kind == EK_OPERATION ? int(x.node_kind) : -1, x.operand, w_arity(w), int(x.type)};
  });
}
// The same for a row in a warp's shared memory: lane 0 walks it and every
// lane returns its answer.
__device__ inline bool warp_locals_defined(const SearchDesc& s, const uint64_t* node, int n) {
  if (!is_statement_tag(s.slot_type)) return true;
  __syncwarp();
  bool ok = false;
  if (lane_id() == 0) ok = row_locals_defined(s, node, n);
  return __shfl_sync(kFull, ok, 0);
}

// One child, by one warp.  Writes the child row, its parent and reuse
// source (the parent when the genotype is unchanged; k_lower looks for an
// identical current member otherwise) and returns the
// reference's OperatorStats error code (0: none).  stamp[0..2]: SM clock
// after selection, after crossover, after the mutation's subtree generation
// (left 0 for phases not reached); stamp[4]: the generation's steps + 1 on
// lane 0 (left 0 without a generation).
__device__ inline int warp_vary_child(const SearchDesc& s, const char* image, int child, uint64_t seed, WarpRows& w,
                                      int* reuse_out, int* parent_out, long long* stamp) {
  const int lane = lane_id();
  *reuse_out = -1;
  // ---- crossover_child
  Rng random(seed ^ (0x617089e168ULL + uint64_t(child)));
  int parent, donor;
  warp_tournaments(s, random, &parent, &donor);
  *parent_out = parent;
  load_members(s, parent, w.parent, donor, w.donor);
  stamp[0] = clock64();
  if (w.parent.n <= 0 || w.parent.n > s.maxv || w.parent.nc > w.parent.n) return 1;
  warp_copy(w.parent.node, w.parent.cval, w.parent.n, w.parent.nc, w.child.node, w.child.cval);
  w.child.n = w.parent.n;
  w.child.nc = w.parent.nc;
  const int total = w.parent.n;
  const bool gated = s.crossover_probability < 1 && random.unit() >= s.crossover_probability;
  if (!gated) {
    if (s.uniform_phase) (void)random.bounded(1);
    for (int attempt = 0; attempt < s.attempts; ++attempt) {
      const int dest = warp_choose_site(w.parent, random, s.counted, kNoClass);
      if (dest < 0) break;
      const int src = warp_choose_site(w.donor, random, s.counted, w_class(w.parent.node[dest]));
      if (src < 0) continue;
      const int ae = warp_subtree_end(w.parent, dest), be = warp_subtree_end(w.donor, src);
      if (ae < 0 || be < 0) return 3;
      if (total - (ae - dest) + (be - src) > s.maxv) continue;
      const GenResult r = warp_splice(w.parent, dest, ae, w.donor, src, be, w.out, s.stride, s.slot_max_depth,
                                      s.site_depth);
      // a splice that reads a grammar local before assigning it is a
      // rejected attempt (crossover_child, phase_operators.cuh:185)
      if (r.status == ST_OK && warp_locals_defined(s, w.out.node, r.nodes)) {
        warp_copy(w.out.node, w.out.cval, r.nodes, r.constants, w.child.node, w.child.cval);
        w.child.n = r.nodes;
        w.child.nc = r.constants;
        break;
      }
    }
  }
  stamp[1] = clock64();
  // ---- mutate_child
  {
    Rng m(seed ^ (0x124ab512bf01ULL + uint64_t(child)));
    if (m.unit() < s.mutation_probability) {
      if (s.uniform_phase) (void)m.bounded(1);
      const int dest = warp_choose_site(w.child, m, s.counted, kNoClass);
      if (dest >= 0) {
        const uint64_t a = w.child.node[dest];
        const int end = warp_subtree_end(w.child, dest), depth = w_depth(a);
        if (end < 0 || depth < 1) return 6;
        const int entry = w_entry(a);
        const int incoming = s.site_depth ? w_sval(a) - 1 : 0;
        if (incoming < 0 || incoming > s.site_depth) return 6;
        const int logical = s.site_depth - incoming;
        const int replaced = end - dest;
        const int whole = s.maxv - (w.child.n - replaced), phase = kCapacity - (w.child.n - replaced);
        const int available = whole < phase ? whole : phase, uncapped = available < kCapacity ? available : kCapacity;
        const bool capped = s.mutation_max_nodes > 0 && s.mutation_max_nodes < uncapped;
        const int bounded = capped ? s.mutation_max_nodes : uncapped;
        const uint64_t gseed = m.next();
        GenResult g{ST_INVALID, 0, 0, 0};
        if (lane == 0) {
          g = generate(s, image, entry, 0, s.slot_max_depth - depth + 1, bounded, gseed, w.gen.node, w.gen.cval,
                       logical, w.pending);
          stamp[4] = (long long)g.steps + 1;
        }
        g.status = __shfl_sync(kFull, g.status, 0);
        g.nodes = __shfl_sync(kFull, g.nodes, 0);
        g.constants = __shfl_sync(kFull, g.constants, 0);
        __syncwarp();
        stamp[2] = clock64();
        if (capped && g.status == ST_CAPACITY) {
          // a configured cap without a feasible derivation skips this mutation
        } else if (g.status != ST_OK) {
          return 7;
        } else {
          w.gen.n = g.nodes;
          w.gen.nc = g.constants;
          const GenResult r = warp_splice(w.child, dest, end, w.gen, 0, w.gen.n, w.out, s.stride, s.slot_max_depth,
                                          s.site_depth);
          if (r.status != ST_OK) return 8;
          // a mutation that reads a grammar local before assigning it is
          // dropped and the crossed child stands (mutate_child,
          // phase_operators.cuh:240-241)
          if (warp_locals_defined(s, w.out.node, r.nodes)) {
            warp_copy(w.out.node, w.out.cval, r.nodes, r.constants, w.child.node, w.child.cval);
            w.child.n = r.nodes;
            w.child.nc = r.constants;
          }
        }
      }
    }
  }
  // ---- the generational schedule's elites (reproduce,
  // phase_population_cpu.cpp:283-290): the first elite_count children are
  // the best members, each reusing its own completed result (an identical
  // program: the same result as the parent or member the reference finds)
  if (s.generational && child < s.elite_count) {
    const int src = s.elites[child];
    const int32_t l = s.len[src];
    for (int i = lane; i < len_nodes(l); i += 32)
      s.cnode[size_t(child) * s.stride + i] = s.node[size_t(src) * s.stride + i];
    for (int i = lane; i < len_consts(l); i += 32)
      s.ccval[size_t(child) * s.stride + i] = s.cval[size_t(src) * s.stride + i];
    if (lane == 0) s.clen[child] = l;
    *reuse_out = src;
    return 0;
  }
  // ---- compare_child: identical construction records and constants
  bool equal = w.child.n == w.parent.n && w.child.nc == w.parent.nc;
  if (equal) {
    bool mine = true;
    for (int i = lane; i < w.child.n; i += 32) mine &= w_origin(w.child.node[i]) == w_origin(w.parent.node[i]);
    for (int i = lane; i < w.child.nc; i += 32) mine &= w.child.cval[i] == w.parent.cval[i];
    equal = __all_sync(kFull, mine);
  }
  if (equal) *reuse_out = parent;
  // ---- publish the child row
  for (int i = lane; i < w.child.n; i += 32) s.cnode[size_t(child) * s.stride + i] = w.child.node[i];
  for (int i = lane; i < w.child.nc; i += 32) s.ccval[size_t(child) * s.stride + i] = w.child.cval[i];
  if (lane == 0) s.clen[child] = make_len(w.child.n, w.child.nc);
  return 0;
}

// Member (or child) node count for ranking: AST nodes (fixed wrapper nodes +
// phase nodes), or the mutable grammar sites under tie_break grammar_sites
// (HostPhasePopulation::nodes, phase_population_cpu.cpp:165-173).
__device__ inline uint32_t ranking_nodes(const SearchDesc& s, const uint64_t* node, int n) {
  if (!s.grammar_sites) return uint32_t(s.fixed_nodes + n);
  uint32_t count = 0;
  for (int i = 0; i < n; ++i) count += w_site(node[i]);
  return count;
}

}  // namespace gb
