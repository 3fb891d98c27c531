// Device building blocks of the resident search: the grammar RNG, the
// self-describing node word, typed subtree generation and warp-cooperative
// row primitives.  Each function names the reference function whose results
// it reproduces exactly (paths relative to the reference root).
//
// Node word (64 bits), B200-first layout of one phase-tree node:
//   [0,16)  construction expression (the reference's origin)
//   [16,32) 1 + the reference expression that opened the node's grammar
//           site (0: no site) -- the whole PhaseGeneSite is a function of it
//   [32,40) depth (root = 1), [40,48) site depth: grammar sites on the path
//           from the root down to and including this node
//   [48,52) arity, [52] constant, [53,64) crossover class of the site
//           (nonterminal and scope; kNoClass: none or variation disabled)
// Storing depth and site depth turns the reference's sequential stack walks
// (phase_node_depth, phase_site_depth, phase_tree_depth) into lookups and
// warp max-reductions: a splice shifts the donor subtree's depths by the
// difference at the splice point and leaves every other node's unchanged.
#pragma once
#include <cstdint>

#include "search_state.h"

namespace gb {

// PhaseExpressionKind / PhaseTreeKind / status codes (reference enums).
enum { EK_OPERATION = 0, EK_CONSTANT = 1, EK_BOUND = 2, EK_REFERENCE = 3, EK_INPUT = 4, EK_ALIAS = 5 };
enum { TK_CONSTANT = 0, TK_LOCAL = 1, TK_OPERATION = 2, TK_IF = 3, TK_AND = 4, TK_OR = 5, TK_PROGRAM = 6,
       TK_BLOCK = 7, TK_NIL = 8, TK_ASSIGN = 9, TK_RETURN = 10, TK_FOR_RANGE = 11, TK_VAR = 12, TK_LET = 13,
       TK_BOUND = 14, TK_REGION = 15, TK_TRAVERSE = 16 };
// Completion tag of a statement (kPhaseStatement,
// cpp/src/evolution/repro/gpu/device/phase_compile.cuh:23): a node or phase
// type, never a runtime value.  Tables narrowed to int8_t keep it as -16.
constexpr int kStatementTag = 0xF0;
__host__ __device__ __forceinline__ bool is_statement_tag(int t) { return (t & 0xff) == kStatementTag; }
constexpr int kNamedLocals = 16;  // grammar locals a phase can name (kPhaseNamedLocals)
enum { ST_OK = 0, ST_INVALID = 1, ST_UNSUPPORTED = 2, ST_CAPACITY = 3 };
constexpr int kFixedSite = 1 << 30;
constexpr uint32_t kNoClass = 0x7ffu;
constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------- RNG
// Ranges up to kSmallBound (site counts, value lists, small integer
// domains) draw with 32-bit arithmetic only (Rng::bounded).
constexpr uint64_t kSmallBound = uint64_t(1) << 16;

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
    if (upper - 1 < uint64_t(kSmallBound)) {
      // the same rejection bound and residue from 32-bit arithmetic, with no
      // table load on the generator's dependent chain: m = 2^32 mod u, so
      // the bound (2^64 - u) mod u = 2^64 mod u = m^2 mod u, and a draw
      // v = hi * 2^32 + lo has v mod u = ((hi mod u) * m + lo mod u) mod u
      // (every intermediate below 2^32 for u <= 2^16)
      const uint32_t u = uint32_t(upper);
      const uint32_t m = (0u - u) % u;
      const uint32_t threshold = (m * m) % u;
      for (;;) {
        const uint64_t v = next();
        if (v >= threshold) return ((uint32_t(v >> 32) % u) * m + uint32_t(v) % u) % u;
      }
    }
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
  // bounded(upper) for a fixed upper with its rejection bound
  // ((2^64 - upper) mod upper) and magic floor((2^64 - 1) / upper) given:
  // the residue comes from a multiply-high quotient estimate, at most two
  // below the true quotient, and at most two corrections
  __device__ __forceinline__ uint64_t bounded_fixed(uint64_t upper, uint64_t threshold, uint64_t magic) {
    for (;;) {
      const uint64_t v = next();
      if (v >= threshold) {
        uint64_t r = v - __umul64hi(v, magic) * upper;
        while (r >= upper) r -= upper;
        return r;
      }
    }
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

// ---------------------------------------------------------------- node words
__host__ __device__ __forceinline__ int w_origin(uint64_t w) { return int(w & 0xffffu); }
__host__ __device__ __forceinline__ int w_entry(uint64_t w) { return int((w >> 16) & 0xffffu) - 1; }
__host__ __device__ __forceinline__ int w_depth(uint64_t w) { return int((w >> 32) & 0xffu); }
__host__ __device__ __forceinline__ int w_sval(uint64_t w) { return int((w >> 40) & 0xffu); }
__host__ __device__ __forceinline__ int w_arity(uint64_t w) { return int((w >> 48) & 0xfu); }
__host__ __device__ __forceinline__ bool w_const(uint64_t w) { return (w >> 52) & 1u; }
__host__ __device__ __forceinline__ uint32_t w_class(uint64_t w) { return uint32_t(w >> 53); }
__host__ __device__ __forceinline__ bool w_site(uint64_t w) { return ((w >> 16) & 0xffffu) != 0; }
__host__ __device__ __forceinline__ uint64_t w_make(int origin, int entry, int depth, int sval, int arity, bool constant,
                                           uint32_t cls) {
  return uint64_t(uint32_t(origin) & 0xffffu) | (uint64_t(uint32_t(entry + 1) & 0xffffu) << 16) |
         (uint64_t(uint32_t(depth) & 0xffu) << 32) | (uint64_t(uint32_t(sval) & 0xffu) << 40) |
         (uint64_t(uint32_t(arity) & 0xfu) << 48) | (uint64_t(constant) << 52) | (uint64_t(cls & 0x7ffu) << 53);
}
// Shifts depth and site depth (a donor subtree moved under another parent).
__host__ __device__ __forceinline__ uint64_t w_shift(uint64_t w, int ddepth, int dsval) {
  const int d = w_depth(w) + ddepth, v = w_sval(w) + dsval;
  return (w & ~(0xffffULL << 32)) | (uint64_t(uint32_t(d) & 0xffu) << 32) | (uint64_t(uint32_t(v) & 0xffu) << 40);
}
// Replaces the site (entry and class) of a word by another word's site.
__host__ __device__ __forceinline__ uint64_t w_with_site(uint64_t w, uint64_t site_from) {
  const uint64_t mask = (0xffffULL << 16) | (0x7ffULL << 53);
  return (w & ~mask) | (site_from & mask);
}
__host__ __device__ __forceinline__ int len_nodes(int32_t l) { return l & 0xffff; }
__host__ __device__ __forceinline__ int len_consts(int32_t l) { return (l >> 16) & 0xffff; }
__host__ __device__ __forceinline__ int32_t make_len(int n, int c) { return n | (c << 16); }

// Crossover class of sites opened by reference expression `entry`.
__device__ __forceinline__ uint32_t class_of_entry(const SearchDesc& s, int entry) {
  return entry < 0 ? kNoClass : uint32_t(s.info[entry].site_class);
}

// Definite assignment of grammar locals in a statement program
// (phase_locals_defined, cpp/src/evolution/repro/gpu/device/phase_compile.cuh:170-200):
// a grammar local may be read after an assignment to it, inside a for_range
// body that names it, and after a statement if only when both branches
// assigned it; a loop body's assignments do not outlive the loop, and inputs
// are always defined.  `at(i)` gives node i's tree kind, operand, arity and
// type.  False also for a tree deeper than 64 open nodes or one that ends
// early.
struct StatementNode {
  int kind, operand, arity, type;
};
// (`at` may be host-only: the engine's host code checks imported rows with it)
#pragma nv_exec_check_disable
template <class At>
__host__ __device__ inline bool locals_defined(int n, At at) {
  struct Frame {
    int16_t index, seen;
    uint16_t saved, branch;
  };
  Frame frames[64];
  int depth = 0;
  unsigned mask = 0;
  auto bit = [](int operand) -> unsigned { return operand >= 0 && operand < kNamedLocals ? 1u << operand : 0u; };
  for (int i = 0; i < n; ++i) {
    const StatementNode x = at(i);
    if (x.kind == TK_VAR && !(mask & bit(x.operand))) return false;
    if (x.arity > 0) {
      if (depth == 64) return false;
      frames[depth++] = Frame{int16_t(i), 0, uint16_t(mask), 0};
      continue;
    }
    while (depth) {
      Frame& f = frames[depth - 1];
      const StatementNode owner = at(f.index);
      ++f.seen;
      if (owner.kind == TK_FOR_RANGE && f.seen == 1) {
        f.saved = uint16_t(mask);
        mask |= bit(owner.operand);
      } else if (owner.kind == TK_IF && is_statement_tag(owner.type)) {
        if (f.seen == 1) {
          f.saved = uint16_t(mask);
        } else if (f.seen == 2) {
          f.branch = uint16_t(mask);
          mask = f.saved;
        } else {
          mask &= f.branch;
        }
      }
      if (f.seen < owner.arity) break;
      if (owner.kind == TK_ASSIGN) mask |= bit(owner.operand);
      else if (owner.kind == TK_FOR_RANGE) mask = f.saved;
      --depth;
    }
  }
  return depth == 0;
}

struct GenResult {
  int status, nodes, constants;
  int steps;  // tasks processed
};

// The subtree generator's tables: the sections of a search's GenImage, in
// shared memory (the variation kernel's staged copy) or in global memory.
// Read with plain loads, which serve either.
struct GenTables {
  const GenExpr* gx;
  const GenNt* gnt;
  const uint32_t* head;
  const GenLevel* level;
  const GenEntry* entry;
  const gagp_domain* doms;
  const gagp_value* vals;
  const uint16_t* minimum;
  const int4* extra;  // children 4..7 and their scopes, two int4 per expression (arity above 4 only)
};
__device__ __forceinline__ GenTables gen_tables(const SearchDesc& s, const char* image) {
  return GenTables{reinterpret_cast<const GenExpr*>(image), reinterpret_cast<const GenNt*>(image + s.gi.nt),
                   reinterpret_cast<const uint32_t*>(image + s.gi.head),
                   reinterpret_cast<const GenLevel*>(image + s.gi.level),
                   reinterpret_cast<const GenEntry*>(image + s.gi.entry),
                   reinterpret_cast<const gagp_domain*>(image + s.gi.doms),
                   reinterpret_cast<const gagp_value*>(image + s.gi.vals),
                   reinterpret_cast<const uint16_t*>(image + s.gi.minimum),
                   reinterpret_cast<const int4*>(image + s.gi.extra)};
}

// A precomputed draw level (GenLevel) in registers.
struct LevelView {
  double total;
  unsigned bound, entry;
  int last, below;
};
__device__ __forceinline__ LevelView load_level(const GenLevel* p) {
  const int4 a = *reinterpret_cast<const int4*>(p);
  const int2 b = *(reinterpret_cast<const int2*>(p) + 2);
  return LevelView{__hiloint2double(a.y, a.x), unsigned(a.z), unsigned(a.w), b.x, b.y};
}

// generate_phase<CompactTasks=true, EmitSites=true, Warp=false>
// (cpp/src/evolution/repro/gpu/device/phase_generate.cuh:125-270): a typed
// random subtree with min-cost feasibility and the FP64 weighted production
// draw.  The draw uses round-to-nearest intrinsics so nothing is contracted
// into an FMA; the reference's host build rounds every operation alike.
// Tasks pack (expression:17, depth:7, scope_count:4, logical:4) in `pending`
// (192 entries).  Emitted words carry depth relative to the generated root
// (root = 1) and site depth relative to the budget `logical_depth`.
__device__ inline GenResult generate(const SearchDesc& s, const char* image, int root_expression, int scope_count,
                                     int depth, int capacity, uint64_t seed, uint64_t* out_node, int64_t* out_cval,
                                     int logical_depth, uint64_t* pending) {
  GenResult result{ST_INVALID, 0, 0, 0};
  const GenTables tables = gen_tables(s, image);
  // the tables (staged in shared memory by the variation kernel), read once
  // into registers; the sequential draw's production tables stay global
  const GenExpr* __restrict__ gx = tables.gx;
  const GenNt* __restrict__ gnt = tables.gnt;
  const uint32_t* __restrict__ head = tables.head;
  const GenLevel* __restrict__ gen_level = tables.level;
  const GenEntry* __restrict__ gen_entry = tables.entry;
  const gagp_domain* __restrict__ doms = tables.doms;
  const gagp_value* __restrict__ vals = tables.vals;
  const uint16_t* __restrict__ minimum = tables.minimum;
  const gagp_production* __restrict__ prods = s.prods;
  const uint32_t* __restrict__ prod_minimum = s.prod_minimum;
  const int n_ex = s.n_ex, n_nts = s.n_nts, n_prods = s.n_prods;
  const int depth_count = s.depth_count, logical_count = s.logical_count;
  const bool site_limited = s.site_depth > 0;
  // minimum cost of (expression, depth, site budget); admission has checked
  // every expression id a table holds, and the generator keeps depth and site
  // budget inside the table, so only the root's lookup is range-checked
  auto min_at = [&](int e, int d, int l) -> unsigned {
    const unsigned v = minimum[(e * depth_count + d) * logical_count + l];
    return v == kNoMinimum16 ? kNoId : v;
  };
  int next_site = -1;  // entry expression of a pending site
  uint32_t next_class = kNoClass;
  if (root_expression < 0 || root_expression >= n_ex || scope_count < 0 || scope_count > 15 || depth <= 0 ||
      depth >= depth_count || depth > 64 || logical_depth < 0 || logical_depth >= logical_count ||
      capacity <= 0 || capacity > kCapacity || n_ex > 131071)
    return result;
  if (capacity > s.stride) capacity = s.stride;  // callers pass at most the node budget
  // a task: expression, depth, scope, site budget and its minimum cost (the
  // reservation made when it was pushed).  The task to run next is kept in a
  // register (`next`, when have_next) rather than pushed and popped at once;
  // `count` is what the reference's stack holds below it.
  auto pack = [](unsigned e, unsigned d, unsigned n, unsigned l, unsigned required) -> uint64_t {
    return uint64_t(e | (d << 17) | (n << 24) | (l << 28)) | (uint64_t(required) << 32);
  };
  unsigned reserved = min_at(root_expression, depth, logical_depth);
  uint64_t next = pack(unsigned(root_expression), unsigned(depth), unsigned(scope_count), unsigned(logical_depth),
                       reserved);
  bool have_next = true;
  int count = 0;
  if (reserved > unsigned(capacity)) { result.status = ST_CAPACITY; return result; }
  Rng random(seed);
  while (have_next || count) {
    if (++result.steps > 8192) { result.status = ST_CAPACITY; return result; }
    const uint64_t task = have_next ? next : pending[--count];
    have_next = false;
    const int t_expr = int(task & 0x1ffffu), t_depth = int((task >> 17) & 0x7fu);
    const int t_scope = int((task >> 24) & 0xfu), t_logical = int((task >> 28) & 0xfu);
    const unsigned required = unsigned(task >> 32);
    if (required > reserved) return result;
    reserved -= required;
    const int4 ra = *reinterpret_cast<const int4*>(gx + t_expr);      // children
    const int4 rb = *(reinterpret_cast<const int4*>(gx + t_expr) + 1);  // target, class, kinds, scopes
    const int kind = int(int8_t(rb.z & 0xff)), arity = int(int8_t((rb.z >> 8) & 0xff));
    const int target = rb.x;
    if (kind == EK_REFERENCE) {
      // admission: the target nonterminal exists, is unscoped (as is every
      // reference) and its productions are in range
      if (next_site >= 0) return result;
      next_site = t_expr;
      next_class = uint32_t(rb.y);
      const int4 nt = *reinterpret_cast<const int4*>(gnt + target);
      const int nt_offset = nt.x, nt_count = nt.y;
      const bool normalized = nt.w != 0;
      if (site_limited && t_logical == 0) { result.status = ST_CAPACITY; return result; }
      const int n_logical = t_logical - (site_limited ? 1 : 0);
      if (reserved > unsigned(capacity - result.nodes)) { result.status = ST_CAPACITY; return result; }
      const unsigned available = unsigned(capacity - result.nodes) - reserved;
      unsigned next_expr, need;
      // the widest precomputed level whose productions all fit
      LevelView lv = load_level(gen_level + head[(t_depth * logical_count + n_logical) * n_nts + target]);
      while (lv.bound > available && lv.below >= 0) lv = load_level(gen_level + lv.below);
      if (lv.bound <= available && lv.total == lv.total) {
        const double choice = __dmul_rn(__dmul_rn(double(random.next() >> 11), 0x1.0p-53), lv.total);
        const GenEntry* __restrict__ en = gen_entry + lv.entry;
        int pick = lv.last;
        if (nt_count <= 8) {
          double th[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) th[k] = k < nt_count ? en[k].threshold : 0.0;
#pragma unroll
          for (int k = 7; k >= 0; --k)
            if (k < nt_count && choice < th[k]) pick = k;
        } else {
          for (int i = 0; i < nt_count; ++i)
            if (choice < en[i].threshold) { pick = i; break; }
        }
        const int2 picked = *(reinterpret_cast<const int2*>(en + pick) + 1);  // expression, need
        next_expr = unsigned(picked.x);
        need = unsigned(picked.y);
      } else {
        // the reference's draw step by step (no precomputed level applies)
        const uint32_t* __restrict__ prow = prod_minimum + (t_depth * logical_count + n_logical) * n_prods + nt_offset;
        uint64_t feasible_mask = 0;  // a bit per production for the first 64
        for (int i = 0; i < nt_count && i < 64; ++i)
          if (__ldg(&prow[i]) <= available) feasible_mask |= 1ULL << i;
        auto feasible = [&](int i) -> bool {
          return i < 64 ? (feasible_mask >> i & 1) : __ldg(&prow[i]) <= available;
        };
        double maximum = normalized ? 1.0 : 0.0, total = 0.0;
        if (!normalized)
          for (int i = 0; i < nt_count; ++i) {
            const double w = __ldg(&prods[nt_offset + i].weight);
            if (feasible(i) && w > maximum) maximum = w;
          }
        if (!(maximum > 0)) { result.status = ST_CAPACITY; return result; }
        for (int i = 0; i < nt_count; ++i)
          if (feasible(i)) {
            const double w = __ldg(&prods[nt_offset + i].weight);
            total = __dadd_rn(total, normalized ? w : __ddiv_rn(w, maximum));
          }
        double choice = __dmul_rn(__dmul_rn(double(random.next() >> 11), 0x1.0p-53), total);
        next_expr = 131071u;  // unselected
        for (int i = 0; i < nt_count; ++i) {
          if (!feasible(i)) continue;
          next_expr = unsigned(__ldg(&prods[nt_offset + i].expression));
          const double w = __ldg(&prods[nt_offset + i].weight);
          choice = __dsub_rn(choice, normalized ? w : __ddiv_rn(w, maximum));
          if (choice < 0) break;
        }
        if (next_expr == 131071u) return result;
        need = min_at(int(next_expr), t_depth, n_logical);
      }
      if (count >= 192) return result;
      reserved += need;
      next = pack(next_expr, unsigned(t_depth), 0u, unsigned(n_logical), need);
      have_next = true;
      continue;
    }
    if (t_depth <= 0 || result.nodes >= capacity) { result.status = ST_CAPACITY; return result; }
    if (kind == EK_CONSTANT) {
      // admission: the domain exists and is an Int range or a list of Ints
      const gagp_domain* domain = doms + target;
      int64_t value;
      if (domain->integer_range) {
        value = random.integer(domain->minimum, domain->maximum);
      } else {
        const int v_offset = domain->value_offset, v_count = domain->value_count;
        value = vals[v_offset + random.bounded(uint64_t(v_count))].i;
      }
      out_cval[result.constants++] = value;
    } else if (kind != EK_OPERATION && kind != EK_INPUT && kind != EK_BOUND) {
      return result;  // aliases are declined at admission
    }
    out_node[result.nodes++] = w_make(t_expr, next_site, depth - t_depth + 1, logical_depth - t_logical, arity,
                                      kind == EK_CONSTANT, next_class);
    next_site = -1;
    next_class = kNoClass;
    // the children's minimum costs, loaded together, then pushed last to
    // first (the first child straight into `next`); a traversal has four
    if (arity > 4) {
      // a bounded region: children 4..7 from the image's extra section,
      // pushed last to first as below
      const int4 xa = tables.extra[2 * t_expr], xb = tables.extra[2 * t_expr + 1];
      for (int i = arity - 1; i >= 0; --i) {
        if (count >= 192) { result.status = ST_CAPACITY; return result; }
        const int child = i == 0 ? ra.x : i == 1 ? ra.y : i == 2 ? ra.z : i == 3 ? ra.w : i == 4 ? xa.x
                          : i == 5 ? xa.y : i == 6 ? xa.z : xa.w;
        const unsigned need = min_at(child, t_depth - 1, t_logical);
        if (need > unsigned(capacity - result.nodes) || reserved > unsigned(capacity - result.nodes) - need) {
          result.status = ST_CAPACITY;
          return result;
        }
        const int child_scope = i < 4 ? int(int8_t((rb.w >> (8 * i)) & 0xff)) : int(int8_t((xb.x >> (8 * (i - 4))) & 0xff));
        const int scope = child_scope >= 0 ? child_scope : t_scope;
        const uint64_t t = pack(unsigned(child), unsigned(t_depth - 1), unsigned(scope), unsigned(t_logical), need);
        if (i == 0) {
          next = t;
          have_next = true;
        } else {
          pending[count++] = t;
        }
        reserved += need;
      }
      continue;
    }
    const unsigned need0 = arity > 0 ? min_at(ra.x, t_depth - 1, t_logical) : 0;
    const unsigned need1 = arity > 1 ? min_at(ra.y, t_depth - 1, t_logical) : 0;
    const unsigned need2 = arity > 2 ? min_at(ra.z, t_depth - 1, t_logical) : 0;
    const unsigned need3 = arity > 3 ? min_at(ra.w, t_depth - 1, t_logical) : 0;
    for (int i = arity - 1; i >= 0; --i) {
      if (count >= 192) { result.status = ST_CAPACITY; return result; }
      const int child = i == 0 ? ra.x : i == 1 ? ra.y : i == 2 ? ra.z : ra.w;
      const unsigned need = i == 0 ? need0 : i == 1 ? need1 : i == 2 ? need2 : need3;
      if (need > unsigned(capacity - result.nodes) || reserved > unsigned(capacity - result.nodes) - need) {
        result.status = ST_CAPACITY;
        return result;
      }
      const int child_scope = int(int8_t((rb.w >> (8 * i)) & 0xff));
      const int scope = child_scope >= 0 ? child_scope : t_scope;
      const uint64_t t = pack(unsigned(child), unsigned(t_depth - 1), unsigned(scope), unsigned(t_logical), need);
      if (i == 0) {
        next = t;
        have_next = true;
      } else {
        pending[count++] = t;
      }
      reserved += need;
    }
  }
  if (reserved || !result.nodes) return result;
  result.status = ST_OK;
  return result;
}

// ------------------------------------------------------- warp row primitives
// A row staged in shared memory: node words and constants.
struct SRow {
  uint64_t* node;
  int64_t* cval;
  int n, nc;
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

__device__ inline void warp_copy(const uint64_t* from_node, const int64_t* from_cval, int n, int nc, uint64_t* to_node,
                                 int64_t* to_cval) {
  for (int i = lane_id(); i < n; i += 32) to_node[i] = from_node[i];
  for (int i = lane_id(); i < nc; i += 32) to_cval[i] = from_cval[i];
  __syncwarp();
}

// site_matches (phase_operators.cuh:51-54): a variation site of class `cls`
// (any class when cls == kNoClass).
__device__ __forceinline__ bool site_matches(uint64_t w, uint32_t cls) {
  const uint32_t c = w_class(w);
  return c != kNoClass && (cls == kNoClass || c == cls);
}

// choose_site (phase_operators.cuh:55-83 and the counted warp variant
// :95-117): the same count, draws and prefix-ordered rank; reservoir draws
// visit matching sites in prefix order.  Every lane returns the same site.
__device__ inline int warp_choose_site(const SRow& t, Rng& random, bool counted, uint32_t cls) {
  const int lane = lane_id();
  if (counted) {
    unsigned count = 0;
    for (int chunk = 0; chunk < t.n; chunk += 32) {
      const int i = chunk + lane;
      count += __popc(__ballot_sync(kFull, i < t.n && site_matches(t.node[i], cls)));
    }
    if (!count) return -1;
    unsigned rank = unsigned(random.bounded(count));
    for (int chunk = 0; chunk < t.n; chunk += 32) {
      const int i = chunk + lane;
      unsigned mask = __ballot_sync(kFull, i < t.n && site_matches(t.node[i], cls));
      const unsigned c = __popc(mask);
      if (rank < c) {
        for (unsigned j = 0; j < rank; ++j) mask &= mask - 1;
        return chunk + __ffs(mask) - 1;
      }
      rank -= c;
    }
    return -1;
  }
  int selected = -1;
  unsigned count = 0;
  for (int chunk = 0; chunk < t.n; chunk += 32) {
    const int i = chunk + lane;
    unsigned mask = __ballot_sync(kFull, i < t.n && site_matches(t.node[i], cls));
    while (mask) {
      const int bit = __ffs(mask) - 1;
      mask &= mask - 1;
      if (random.bounded(++count) == 0) selected = chunk + bit;
    }
  }
  return selected;
}

// phase_subtree_end (device/phase_variation.cuh:81-91, warp form :213-229).
__device__ inline int warp_subtree_end(const SRow& t, int start) {
  if (start < 0 || start >= t.n) return -1;
  const int lane = lane_id();
  int pending = 1;
  for (int chunk = start; chunk < t.n; chunk += 32) {
    const int i = chunk + lane;
    const bool live = i < t.n;
    int scan = live ? w_arity(t.node[i]) - 1 : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int up = __shfl_up_sync(kFull, scan, o);
      if (lane >= o) scan += up;
    }
    const unsigned hit = __ballot_sync(kFull, live && pending + scan == 0);
    if (hit) return chunk + __ffs(hit);
    pending += __shfl_sync(kFull, scan, 31);
  }
  return -1;
}

// Constant nodes among row positions [0, first) and [0, second), first <= second.
__device__ __forceinline__ void warp_count_constants2(const SRow& t, int first, int second, int* a, int* b) {
  int ca = 0, cb = 0;
  for (int chunk = 0; chunk < second; chunk += 32) {
    const int i = chunk + lane_id();
    const bool c = i < second && w_const(t.node[i]);
    ca += __popc(__ballot_sync(kFull, c && i < first));
    cb += __popc(__ballot_sync(kFull, c));
  }
  *a = ca;
  *b = cb;
}

template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    const T u = __shfl_xor_sync(kFull, v, o);
    v = u > v ? u : v;
  }
  return v;
}

// splice_phase_tree (device/phase_variation.cuh:147-207): base with the
// subtree [dest, end) replaced by donor's subtree [src, donor_end), into
// `out`; the callers have found both subtree ends already.
// Depth and site-depth limits are maxima of the output words; constants are
// base[..dest) ++ donor subtree ++ base[end..), the prefix renumbering the
// reference performs node by node.  Every lane returns the same result.
__device__ inline GenResult warp_splice(const SRow& base, int dest, int end, const SRow& donor, int src, int donor_end,
                                        SRow out, int stride, int max_depth, int site_limit) {
  GenResult r{ST_INVALID, 0, 0};
  if (max_depth <= 0 || max_depth > 64 || base.n <= 0 || donor.n <= 0 || dest < 0 || dest >= base.n || src < 0 ||
      src >= donor.n)
    return r;
  const uint64_t a = base.node[dest], b = donor.node[src];
  if (!w_site(a) || w_class(a) != w_class(b)) return r;
  if (end <= dest || end > base.n || donor_end <= src || donor_end > donor.n) return r;
  const int inserted = donor_end - src;
  const int length = base.n - (end - dest) + inserted;
  if (length > kCapacity) { r.status = ST_CAPACITY; return r; }
  if (length > stride) { r.status = ST_CAPACITY; return r; }  // never reached: callers bound by the node budget
  const int ddepth = w_depth(a) - w_depth(b), dsval = w_sval(a) - w_sval(b);
  int maxd = 0, maxs = 0;
  for (int i = lane_id(); i < length; i += 32) {
    uint64_t w;
    if (i >= dest && i < dest + inserted) {
      w = w_shift(donor.node[src + i - dest], ddepth, dsval);
      if (i == dest) w = w_with_site(w, a);
    } else {
      w = base.node[i < dest ? i : i + (end - dest) - inserted];
    }
    out.node[i] = w;
    maxd = max(maxd, w_depth(w));
    maxs = max(maxs, w_sval(w));
  }
  int bb, be, db, de;
  warp_count_constants2(base, dest, end, &bb, &be);
  warp_count_constants2(donor, src, donor_end, &db, &de);
  const int dc = de - db;
  for (int k = lane_id(); k < bb; k += 32) out.cval[k] = base.cval[k];
  for (int k = lane_id(); k < dc; k += 32) out.cval[bb + k] = donor.cval[db + k];
  for (int k = lane_id(); k < base.nc - be; k += 32) out.cval[bb + dc + k] = base.cval[be + k];
  maxd = warp_max(maxd);
  maxs = warp_max(maxs);
  __syncwarp();
  if (maxd > max_depth) { r.status = ST_CAPACITY; return r; }
  if (site_limit && maxs > site_limit) { r.status = ST_CAPACITY; return r; }
  r.status = ST_OK;
  r.nodes = length;
  r.constants = bb + dc + (base.nc - be);
  return r;
}

}  // namespace gb
