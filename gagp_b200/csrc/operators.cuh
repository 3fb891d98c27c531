// Per-child selection and variation of one steady-state round
// (crossover_child / mutate_child / compare_child,
// cpp/src/evolution/repro/gpu/phase_operators.cuh:46-265), over the compact
// row layout.  One whole-program phase per member (slot_count == 1), so the
// uniform-phase draw is bounded(1) and a row is a member.
#pragma once
#include "device_ops.cuh"

namespace gb {

// Selection-value comparison of two members.  For metrics with wrong counts
// the reference's selection values are ranks (evolve.cpp:285,361), so a
// larger selection value is exactly a better rank; otherwise they are the
// fitness values.  Keys pack (-fitness, wrong, nodes) so smaller is better.
__device__ __forceinline__ bool selection_greater(const SearchDesc& s, const uint64_t* key, int c, int b) {
  const uint64_t kc = key[c], kb = key[b];
  return kc < kb || (s.has_wrong && kc == kb && c < b);
}
// Ranking order `better` (evolve.cpp:351-355): strict total order.
__device__ __forceinline__ bool better(const uint64_t* key, int a, int b) {
  const uint64_t ka = key[a], kb = key[b];
  return ka < kb || (ka == kb && a < b);
}

// tournament (phase_operators.cuh:46-50)
__device__ inline int tournament(const SearchDesc& s, Rng& random) {
  int best = int(random.bounded(uint64_t(s.P)));
  for (int i = 1; i < s.pressure; ++i) {
    const int c = int(random.bounded(uint64_t(s.P)));
    if (selection_greater(s, s.key, c, best)) best = c;
  }
  return best;
}

// site_matches (phase_operators.cuh:51-54): a variation site of class `cls`
// (any class when cls < 0); fixed-nonterminal sites never match.
__device__ __forceinline__ bool site_matches(const SearchDesc& s, uint32_t w, int cls) {
  const int e = entry_of(w);
  if (e < 0) return false;
  const int c = s.info[e].site_class;
  return c >= 0 && (cls < 0 || c == cls);
}

// choose_site (phase_operators.cuh:55-83): counted rank draw or reservoir draws.
__device__ inline int choose_site(const SearchDesc& s, const Row& t, Rng& random, bool counted, int cls) {
  if (counted) {
    unsigned count = 0;
    for (int i = 0; i < t.n; ++i) count += site_matches(s, t.node[i], cls);
    if (!count) return -1;
    unsigned rank = unsigned(random.bounded(count));
    for (int i = 0; i < t.n; ++i)
      if (site_matches(s, t.node[i], cls)) {
        if (rank == 0) return i;
        --rank;
      }
    return -1;
  }
  int selected = -1;
  unsigned count = 0;
  for (int i = 0; i < t.n; ++i)
    if (site_matches(s, t.node[i], cls))
      if (random.bounded(++count) == 0) selected = i;
  return selected;
}

// One child: crossover into the child row, then mutation of the child row,
// then the identity check against its first parent.  Returns the error code
// of the reference's OperatorStats (0: none).
__device__ inline int vary_child(const SearchDesc& s, int child, uint64_t seed, int* reuse_out, int* parent_out) {
  const Row none{nullptr, nullptr, 0, 0};
  (void)none;
  *reuse_out = -1;
  MRow crow = mrow_of(s.cnode, s.ccval, s.stride, child);
  MRow tmp = mrow_of(s.tnode, s.tcval, s.stride, child);
  // ---- crossover_child
  Rng random(seed ^ (0x617089e168ULL + uint64_t(child)));
  const int parent = tournament(s, random), donor = tournament(s, random);
  *parent_out = parent;
  const Row prow = row_of(s.node, s.cval, s.len, s.stride, parent);
  const Row drow = row_of(s.node, s.cval, s.len, s.stride, donor);
  if (prow.n <= 0 || prow.n > s.maxv || prow.nc > prow.n) return 1;
  copy_row(prow, crow);
  int n = prow.n, nc = prow.nc;
  const int total = prow.n;
  bool gated = s.crossover_probability < 1 && random.unit() >= s.crossover_probability;
  if (!gated) {
    if (s.uniform_phase) (void)random.bounded(1);
    for (int attempt = 0; attempt < s.attempts; ++attempt) {
      const int dest = choose_site(s, prow, random, s.counted, -1);
      if (dest < 0) break;
      const int cls = s.info[entry_of(prow.node[dest])].site_class;
      const int src = choose_site(s, drow, random, s.counted, cls);
      if (src < 0) continue;
      const int ae = subtree_end(s, prow, dest), be = subtree_end(s, drow, src);
      if (ae < 0 || be < 0) return 3;
      if (total - (ae - dest) + (be - src) > s.maxv) continue;
      const GenResult r = splice(s, prow, dest, drow, src, tmp, s.slot_max_depth, s.site_depth);
      if (r.status == ST_OK) {
        copy_row(Row{tmp.node, tmp.cval, r.nodes, r.constants}, crow);
        n = r.nodes;
        nc = r.constants;
        break;
      }
    }
  }
  s.clen[child] = make_len(n, nc);
  // ---- mutate_child
  {
    const Row c{crow.node, crow.cval, n, nc};
    Rng m(seed ^ (0x124ab512bf01ULL + uint64_t(child)));
    if (m.unit() < s.mutation_probability) {
      if (s.uniform_phase) (void)m.bounded(1);
      const int dest = choose_site(s, c, m, s.counted, -1);
      if (dest >= 0) {
        const int end = subtree_end(s, c, dest), depth = node_depth(s, c, dest);
        if (end < 0 || depth < 0) return 6;
        const int entry = entry_of(c.node[dest]);
        const int incoming = s.site_depth ? site_depth_of(s, c.node, c.n, dest) : 0;
        if (incoming < 0 || incoming > s.site_depth) return 6;
        const int logical = s.site_depth - incoming;
        const int replaced = end - dest;
        const int whole = s.maxv - (c.n - replaced), phase = kCapacity - (c.n - replaced);
        const int available = whole < phase ? whole : phase, uncapped = available < kCapacity ? available : kCapacity;
        const bool capped = s.mutation_max_nodes > 0 && s.mutation_max_nodes < uncapped;
        const int bounded = capped ? s.mutation_max_nodes : uncapped;
        uint32_t* gnode = s.gnode + size_t(child) * s.stride;
        int64_t* gcval = s.gcval + size_t(child) * s.stride;
        // parent_scope of a site: scoped nonterminals are declined at admission
        const GenResult g = generate(s, entry, 0, s.slot_max_depth - depth + 1, bounded, m.next(), gnode, gcval,
                                     logical, true);
        if (capped && g.status == ST_CAPACITY) {
          // a configured cap without a feasible derivation skips this mutation
        } else if (g.status != ST_OK) {
          return 7;
        } else {
          const Row gen{gnode, gcval, g.nodes, g.constants};
          const GenResult r = splice(s, c, dest, gen, 0, tmp, s.slot_max_depth, s.site_depth);
          if (r.status != ST_OK) return 8;
          copy_row(Row{tmp.node, tmp.cval, r.nodes, r.constants}, crow);
          n = r.nodes;
          nc = r.constants;
          s.clen[child] = make_len(n, nc);
        }
      }
    }
  }
  // ---- compare_child: identical genotype (construction records + constants)
  if (n == prow.n && nc == prow.nc) {
    bool equal = true;
    for (int i = 0; i < n && equal; ++i) equal = origin_of(crow.node[i]) == origin_of(prow.node[i]);
    for (int i = 0; i < nc && equal; ++i) equal = crow.cval[i] == prow.cval[i];
    if (equal) *reuse_out = parent;
  }
  return 0;
}

// Member (or child) node count for ranking: AST nodes (fixed wrapper nodes +
// phase nodes), or the mutable grammar sites under tie_break grammar_sites
// (HostPhasePopulation::nodes, phase_population_cpu.cpp:165-173).
__device__ inline uint32_t ranking_nodes(const SearchDesc& s, const uint32_t* node, int n) {
  if (!s.grammar_sites) return uint32_t(s.fixed_nodes + n);
  uint32_t count = 0;
  for (int i = 0; i < n; ++i) count += entry_of(node[i]) >= 0;
  return count;
}

}  // namespace gb
