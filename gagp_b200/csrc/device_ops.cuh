// Device building blocks of the resident search: the grammar RNG, phase-row
// primitives, typed subtree generation and splicing over the compact row
// layout of search_state.h.  Each function names the reference function whose
// semantics it reproduces exactly (paths relative to the reference root).
#pragma once
#include <cstdint>

#include "search_state.h"

namespace gb {

// PhaseExpressionKind / PhaseTreeKind / status codes (reference enums).
enum { EK_OPERATION = 0, EK_CONSTANT = 1, EK_BOUND = 2, EK_REFERENCE = 3, EK_INPUT = 4, EK_ALIAS = 5 };
enum { TK_CONSTANT = 0, TK_LOCAL = 1, TK_OPERATION = 2, TK_IF = 3, TK_AND = 4, TK_OR = 5 };
enum { ST_OK = 0, ST_INVALID = 1, ST_UNSUPPORTED = 2, ST_CAPACITY = 3 };
constexpr int kFixedSite = 1 << 30;

// ---------------------------------------------------------------- RNG
// SplitMix64 stream with rejection-sampled bounds
// (DGrammarRandom, cpp/src/evolution/repro/gpu/device/grammar_random.cuh:10-51).
struct Rng {
  uint64_t state;
  __device__ explicit Rng(uint64_t seed) : state(seed) {}
  __device__ __forceinline__ uint64_t next() {
    uint64_t v = (state += 0x9e3779b97f4a7c15ULL);
    v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ULL;
    v = (v ^ (v >> 27)) * 0x94d049bb133111ebULL;
    return v ^ (v >> 31);
  }
  __device__ __forceinline__ uint64_t bounded(uint64_t upper) {
    const uint64_t threshold = (0 - upper) % upper;
    for (;;) {
      const uint64_t v = next();
      if (v >= threshold) return v % upper;
    }
  }
  __device__ __forceinline__ int64_t integer(int64_t lo, int64_t hi) {
    const uint64_t sign = 1ULL << 63;
    const uint64_t first = uint64_t(lo) ^ sign, last = uint64_t(hi) ^ sign;
    const uint64_t width = last - first + 1;
    const uint64_t bits = (first + (width ? bounded(width) : next())) ^ sign;
    if (bits < sign) return int64_t(bits);
    return INT64_MIN + int64_t(bits - sign);
  }
  // 53-bit uniform in [0,1): exact (a power-of-two scale)
  __device__ __forceinline__ double unit() { return __dmul_rn(double(next() >> 11), 0x1.0p-53); }
};

__device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

// ---------------------------------------------------------------- rows
__device__ __forceinline__ int origin_of(uint32_t w) { return int(w & 0xffffu); }
__device__ __forceinline__ int entry_of(uint32_t w) { return int(w >> 16) - 1; }
__device__ __forceinline__ uint32_t make_word(int origin, int entry) {
  return uint32_t(origin) | (uint32_t(entry + 1) << 16);
}
__device__ __forceinline__ int len_nodes(int32_t l) { return l & 0xffff; }
__device__ __forceinline__ int len_consts(int32_t l) { return (l >> 16) & 0xffff; }
__device__ __forceinline__ int32_t make_len(int n, int c) { return n | (c << 16); }

struct Row {
  const uint32_t* node;
  const int64_t* cval;
  int n, nc;
};
struct MRow {
  uint32_t* node;
  int64_t* cval;
};

__device__ __forceinline__ Row row_of(const uint32_t* node, const int64_t* cval, const int32_t* len, int stride, int r) {
  const int32_t l = len[r];
  return Row{node + size_t(r) * stride, cval + size_t(r) * stride, len_nodes(l), len_consts(l)};
}
__device__ __forceinline__ MRow mrow_of(uint32_t* node, int64_t* cval, int stride, int r) {
  return MRow{node + size_t(r) * stride, cval + size_t(r) * stride};
}

__device__ __forceinline__ int arity_of(const SearchDesc& s, uint32_t w) { return s.info[origin_of(w)].arity; }
__device__ __forceinline__ bool is_constant(const SearchDesc& s, uint32_t w) {
  return s.info[origin_of(w)].node_kind == TK_CONSTANT;
}
// PhaseGeneSite fields as functions of the site's entry expression.
__device__ __forceinline__ int site_nt(const SearchDesc& s, int entry) { return entry < 0 ? -1 : s.info[entry].site_nt; }
__device__ __forceinline__ int site_scope(const SearchDesc& s, int entry) {
  if (entry < 0) return 0;
  const gagp_expression& e = s.ex[entry];
  const bool fixed = s.nts[e.target].fixed != 0;
  return e.scope_count | (fixed ? kFixedSite : 0);
}

__device__ inline void copy_row(const Row& from, MRow to) {
  for (int i = 0; i < from.n; ++i) to.node[i] = from.node[i];
  for (int i = 0; i < from.nc; ++i) to.cval[i] = from.cval[i];
}

// phase_subtree_end (device/phase_variation.cuh:81-91)
__device__ inline int subtree_end(const SearchDesc& s, const Row& t, int start) {
  if (start < 0 || start >= t.n || t.n > kCapacity) return -1;
  int pending = 1;
  for (int i = start; i < t.n; ++i) {
    const int a = arity_of(s, t.node[i]);
    if (a < 0 || a > 8) return -1;
    pending += a - 1;
    if (!pending) return i + 1;
  }
  return -1;
}
// phase_node_depth (device/phase_variation.cuh:92-105)
__device__ inline int node_depth(const SearchDesc& s, const Row& t, int position) {
  if (position < 0 || position >= t.n || t.n > kCapacity) return -1;
  int pending[64];
  int depth = 1;
  pending[0] = 1;
  for (int i = 0; i <= position; ++i) {
    while (depth && !pending[depth - 1]) --depth;
    if (!depth) return -1;
    if (i == position) return depth;
    --pending[depth - 1];
    const int a = arity_of(s, t.node[i]);
    if (a < 0 || a > 8) return -1;
    if (a) {
      if (depth == 64) return -1;
      pending[depth++] = a;
    }
  }
  return -1;
}
// phase_site_depth (device/phase_variation.cuh:127-142); position < 0 gives
// the height, otherwise the incoming depth at `position`.
__device__ inline int site_depth_of(const SearchDesc& s, const uint32_t* node, int count, int position) {
  if (count <= 0 || count > kCapacity || position >= count) return -1;
  int pending[64], incoming[64];
  int depth = 1, maximum = 0;
  pending[0] = 1;
  incoming[0] = 0;
  for (int i = 0; i < count; ++i) {
    while (depth && !pending[depth - 1]) --depth;
    if (!depth) return -1;
    if (i == position) return incoming[depth - 1];
    const int a = arity_of(s, node[i]);
    if (a < 0 || a > 8) return -1;
    const int value = incoming[depth - 1] + (entry_of(node[i]) >= 0 ? 1 : 0);
    maximum = value > maximum ? value : maximum;
    --pending[depth - 1];
    if (a) {
      if (depth == 64) return -1;
      pending[depth] = a;
      incoming[depth++] = value;
    }
  }
  while (depth && !pending[depth - 1]) --depth;
  return depth ? -1 : maximum;
}

struct GenResult {
  int status, nodes, constants;
};

// splice_phase_tree<FusedDepth=true> (device/phase_variation.cuh:147-207).
// Output constants are base[..dest) ++ donor subtree ++ base[end..), which is
// the prefix renumbering the reference applies node by node.
__device__ inline GenResult splice(const SearchDesc& s, const Row& base, int dest, const Row& donor, int src,
                                   MRow out, int max_depth, int site_limit) {
  GenResult r{ST_INVALID, 0, 0};
  if (max_depth <= 0 || max_depth > 64 || base.n <= 0 || base.n > kCapacity || donor.n <= 0 ||
      donor.n > kCapacity || base.nc < 0 || base.nc > base.n || donor.nc < 0 || donor.nc > donor.n || dest < 0 ||
      dest >= base.n || src < 0 || src >= donor.n)
    return r;
  const int ea = entry_of(base.node[dest]), eb = entry_of(donor.node[src]);
  const int na = site_nt(s, ea), nb = site_nt(s, eb);
  if (na < 0 || na != nb || site_scope(s, ea) != site_scope(s, eb)) return r;
  const int end = subtree_end(s, base, dest), donor_end = subtree_end(s, donor, src);
  if (end < 0 || donor_end < 0) return r;
  const int inserted = donor_end - src;
  const int length = base.n - (end - dest) + inserted;
  if (length > kCapacity) { r.status = ST_CAPACITY; return r; }
  // Callers bound the output by the variable-node budget before splicing
  // (crossover's total check, mutation's generation capacity); the row
  // stride holds that budget.
  if (length > s.stride) { r.status = ST_CAPACITY; return r; }
  int pending[64];
  int depth = 1, maximum = 1;
  pending[0] = 1;
  for (int i = 0; i < length; ++i) {
    const bool incoming = i >= dest && i < dest + inserted;
    uint32_t w = incoming ? donor.node[src + i - dest] : base.node[i < dest ? i : i + (end - dest) - inserted];
    const int a = arity_of(s, w);
    while (depth && !pending[depth - 1]) --depth;
    if (!depth || a < 0 || a > 8) return r;
    maximum = depth > maximum ? depth : maximum;
    --pending[depth - 1];
    if (a) {
      if (depth == 64) return r;
      pending[depth++] = a;
    }
    if (i == dest) w = (w & 0xffffu) | (uint32_t(ea + 1) << 16);
    out.node[i] = w;
  }
  int bb = 0, be = 0, db = 0, dc = 0;
  for (int i = 0; i < end; ++i) {
    const int c = is_constant(s, base.node[i]);
    be += c;
    if (i < dest) bb += c;
  }
  for (int i = 0; i < donor_end; ++i) {
    const int c = is_constant(s, donor.node[i]);
    if (i < src) db += c; else dc += c;
  }
  if (be > base.nc || db + dc > donor.nc) return r;
  int o = 0;
  for (int k = 0; k < bb; ++k) out.cval[o++] = base.cval[k];
  for (int k = 0; k < dc; ++k) out.cval[o++] = donor.cval[db + k];
  for (int k = be; k < base.nc; ++k) out.cval[o++] = base.cval[k];
  while (depth && !pending[depth - 1]) --depth;
  if (depth) return r;
  if (maximum > max_depth) { r.status = ST_CAPACITY; return r; }
  if (site_limit) {
    const int height = site_depth_of(s, out.node, length, -1);
    if (height < 0) return r;
    if (height > site_limit) { r.status = ST_CAPACITY; return r; }
  }
  r.status = ST_OK;
  r.nodes = length;
  r.constants = o;
  return r;
}


// Minimum node cost of (expression, depth, site budget); kNoId when infeasible.
__device__ __forceinline__ unsigned minimum_of(const SearchDesc& s, int e, int d, int l) {
  if (e < 0 || e >= s.n_ex || d < 0 || d >= s.depth_count || l < 0 || l >= s.logical_count) return kNoId;
  return __ldg(&s.minimum[(size_t(e) * s.depth_count + d) * s.logical_count + l]);
}

// generate_phase<CompactTasks=true, EmitSites, Warp=false>
// (cpp/src/evolution/repro/gpu/device/phase_generate.cuh:125-270): a typed
// random subtree with min-cost feasibility and the FP64 weighted production
// draw.  The draw uses round-to-nearest intrinsics so nothing is contracted
// into an FMA; the reference host build rounds every operation the same way.
// Tasks pack (expression:17, depth:7, scope_count:4, logical:4).
__device__ inline GenResult generate(const SearchDesc& s, int root_expression, int scope_count, int depth,
                                     int capacity, uint64_t seed, uint32_t* out_node, int64_t* out_cval,
                                     int logical_depth, bool emit_sites) {
  GenResult result{ST_INVALID, 0, 0};
  int steps = 0;
  int next_site = -1;  // entry expression of a pending site
  const bool site_limited = s.site_depth > 0;
  if (root_expression < 0 || root_expression >= s.n_ex || scope_count < 0 || scope_count > 15 || depth <= 0 ||
      depth >= s.depth_count || depth > 64 || logical_depth < 0 || logical_depth >= s.logical_count ||
      capacity <= 0 || capacity > kCapacity || s.n_ex > 131071)
    return result;
  if (capacity > s.stride) capacity = s.stride;  // never reached: callers pass <= the node budget
  const unsigned unselected = 131071u;
  uint32_t pending[192];
  int count = 1;
  auto pack = [](unsigned e, unsigned d, unsigned n, unsigned l) -> uint32_t {
    return e | (d << 17) | (n << 24) | (l << 28);
  };
  pending[0] = pack(unsigned(root_expression), unsigned(depth), unsigned(scope_count), unsigned(logical_depth));
  unsigned reserved = minimum_of(s, root_expression, depth, logical_depth);
  if (reserved > unsigned(capacity)) { result.status = ST_CAPACITY; return result; }
  Rng random(seed);
  while (count) {
    if (++steps > 8192) { result.status = ST_CAPACITY; return result; }
    const uint32_t task = pending[--count];
    const int t_expr = int(task & 0x1ffffu), t_depth = int((task >> 17) & 0x7fu);
    const int t_scope = int((task >> 24) & 0xfu), t_logical = int(task >> 28);
    const unsigned required = minimum_of(s, t_expr, t_depth, t_logical);
    if (required > reserved) return result;
    reserved -= required;
    const gagp_expression& expression = s.ex[t_expr];
    const ExprInfo info = s.info[t_expr];
    if (info.kind == EK_REFERENCE) {
      if (expression.target < 0 || expression.target >= s.n_nts || expression.scope_count < 0 ||
          expression.scope_count > 8)
        return result;
      if (emit_sites) {
        if (next_site >= 0) return result;
        next_site = t_expr;
      }
      const gagp_nonterminal nt = s.nts[expression.target];
      if (nt.scope_count != expression.scope_count || nt.production_offset < 0 || nt.production_count <= 0 ||
          nt.production_offset > s.n_prods || nt.production_count > s.n_prods - nt.production_offset)
        return result;
      if (site_limited && t_logical == 0) { result.status = ST_CAPACITY; return result; }
      const int n_logical = t_logical - (site_limited ? 1 : 0);
      unsigned next_expr = unselected;
      if (reserved > unsigned(capacity - result.nodes)) { result.status = ST_CAPACITY; return result; }
      const unsigned available = unsigned(capacity - result.nodes) - reserved;
      double maximum = nt.normalized_weights ? 1.0 : 0.0, total = 0.0;
      if (!nt.normalized_weights)
        for (int i = 0; i < nt.production_count; ++i) {
          const gagp_production p = s.prods[nt.production_offset + i];
          if (minimum_of(s, p.expression, t_depth, n_logical) <= available && p.weight > maximum) maximum = p.weight;
        }
      if (!(maximum > 0)) { result.status = ST_CAPACITY; return result; }
      for (int i = 0; i < nt.production_count; ++i) {
        const gagp_production p = s.prods[nt.production_offset + i];
        if (minimum_of(s, p.expression, t_depth, n_logical) <= available)
          total = __dadd_rn(total, nt.normalized_weights ? p.weight : __ddiv_rn(p.weight, maximum));
      }
      double choice = __dmul_rn(__dmul_rn(double(random.next() >> 11), 0x1.0p-53), total);
      for (int i = 0; i < nt.production_count; ++i) {
        const gagp_production p = s.prods[nt.production_offset + i];
        if (minimum_of(s, p.expression, t_depth, n_logical) > available) continue;
        if (p.expression < 0 || p.expression >= s.n_ex) return result;
        next_expr = unsigned(p.expression);
        choice = __dsub_rn(choice, nt.normalized_weights ? p.weight : __ddiv_rn(p.weight, maximum));
        if (choice < 0) break;
      }
      if (next_expr == unselected || count >= 192) return result;
      reserved += minimum_of(s, int(next_expr), t_depth, n_logical);
      pending[count++] = pack(next_expr, unsigned(t_depth), unsigned(expression.scope_count), unsigned(n_logical));
      continue;
    }
    if (info.kind == EK_ALIAS) {
      const int child = expression.children[0];
      if (child < 0 || child >= s.n_ex || count >= 192) return result;
      const int scope = expression.child_scope[0] >= 0 ? expression.child_scope[0] : t_scope;
      reserved += minimum_of(s, child, t_depth, t_logical);
      pending[count++] = pack(unsigned(child), unsigned(t_depth), unsigned(scope), unsigned(t_logical));
      continue;
    }
    if (t_depth <= 0 || result.nodes >= capacity) { result.status = ST_CAPACITY; return result; }
    const int arity = info.arity;
    if (arity < 0 || arity > 8) return result;
    if (info.kind == EK_BOUND) {
      if (arity != 0 || expression.operand < 0 || expression.operand >= 16) return result;
    } else if (info.kind == EK_CONSTANT) {
      if (expression.target < 0 || expression.target >= s.n_doms || arity != 0) return result;
      const gagp_domain domain = s.doms[expression.target];
      int64_t value;
      if (domain.integer_range) {
        if (domain.minimum > domain.maximum) return result;
        value = random.integer(domain.minimum, domain.maximum);
      } else {
        if (domain.value_offset < 0 || domain.value_count <= 0 || domain.value_offset > s.n_vals ||
            domain.value_count > s.n_vals - domain.value_offset)
          return result;
        const gagp_value v = s.vals[domain.value_offset + random.bounded(uint64_t(domain.value_count))];
        if (v.tag == GAGP_TAG_INVALID) return result;
        value = v.i;
      }
      out_cval[result.constants++] = value;
    } else if (info.kind != EK_OPERATION && info.kind != EK_INPUT) {
      return result;
    }
    out_node[result.nodes++] = make_word(t_expr, emit_sites ? next_site : -1);
    next_site = -1;
    for (int i = arity - 1; i >= 0; --i) {
      if (count >= 192) { result.status = ST_CAPACITY; return result; }
      const int child = expression.children[i];
      const unsigned need = minimum_of(s, child, t_depth - 1, t_logical);
      if (need > unsigned(capacity - result.nodes) || reserved > unsigned(capacity - result.nodes) - need) {
        result.status = ST_CAPACITY;
        return result;
      }
      const int scope = expression.child_scope[i] >= 0 ? expression.child_scope[i] : t_scope;
      pending[count++] = pack(unsigned(child), unsigned(t_depth - 1), unsigned(scope), unsigned(t_logical));
      reserved += need;
    }
  }
  if (reserved || !result.nodes) return result;
  result.status = ST_OK;
  return result;
}

}  // namespace gb
