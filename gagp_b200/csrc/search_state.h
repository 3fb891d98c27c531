// Device-resident state of one search and the descriptor kernels read it by.
//
// Row layout (B200-first, not the reference's): a member is one phase row of
// at most `maxv` nodes.  A node is one 64-bit self-describing word (see
// device_ops.cuh): the construction expression and the expression that
// opened its grammar site -- every other field of the reference's 28-byte
// PhaseTreeNode and 16-byte PhaseGeneSite is a function of those two ids
// (device/phase_compile.cuh:64-74, device/phase_generate.cuh:12-17) -- plus
// depth, site depth, arity, a constant flag and the site's crossover class.
// Constants are int64 payloads in prefix order, which is the operand order
// the reference's generator and splice assign (phase_generate.cuh:253,
// phase_variation.cuh:183-187).  A row is 16 bytes per node slot instead of
// the reference's 64 KB fixed 1024-node rows.
#pragma once
#include <cstdint>

#include "../../include/gagp_b200.h"

namespace gb {

// Elites the generational schedule keeps on the device.
constexpr int kMaxElites = 64;

constexpr int kCapacity = 1024;        // semantic phase capacity (phase_operators.cuh:13)
constexpr unsigned kNoId = 0xffffffffu;
constexpr int kMaxTemps = 6;           // accumulator VM temporaries
constexpr int kMaxCodeWords = 2048;    // accumulator VM instructions per program

// Per-expression facts the kernels need, derived once at admission.
struct ExprInfo {
  int8_t kind;         // PhaseExpressionKind
  int8_t node_kind;    // PhaseTreeKind
  int8_t arity;
  int8_t type;         // ValueTag
  int16_t opcode;
  int16_t reserved;
  int32_t site_class;  // Reference expressions: class of (nonterminal, scope); -1 fixed/none
  int32_t operand;
  int32_t target;
  int32_t site_nt;     // Reference expressions: the nonterminal (site present), else -1
};

// Subtree-generation view of one expression, two 16-byte loads: the first
// four children, then target (nonterminal or domain), the crossover class of
// the sites it opens, kind / arity / scope count and the children's scopes.
struct alignas(16) GenExpr {
  int32_t child[4];
  int32_t target;
  int32_t site_class;
  int8_t kind, arity, scope_count, reserved;
  int8_t child_scope[4];
};
// A nonterminal in one 16-byte load.
struct alignas(16) GenNt {
  int32_t production_offset, production_count, scope_count, normalized_weights;
};
// Precomputed production draw of one nonterminal at one (depth, site
// budget) for one feasibility level: the productions whose minimum cost is at
// most `bound` are the feasible ones, and the draw over them is decided by
// comparing the choice value with per-production thresholds (GenEntry).  A
// nonterminal's levels at one (depth, site budget) form a chain from the
// widest (every production of finite cost) down through `below`.
struct alignas(16) GenLevel {
  double total;     // the draw's weight sum; NaN: no precomputed draw
  uint32_t bound;   // largest minimum cost of a feasible production (kNoId: none)
  uint32_t entry;   // first of the nonterminal's production_count GenEntry
  int32_t last;     // the last feasible production: the pick when no threshold exceeds the choice
  int32_t below;    // the next narrower level, -1: none
  int32_t reserved[2];
};
// One production of a level's draw: the smallest choice value whose running
// difference after this production is not negative (0: never picked), the
// production's expression and its minimum cost at the level's (depth, site
// budget).
struct alignas(16) GenEntry {
  double threshold;
  int32_t expression;
  uint32_t need;
};

// Byte offsets of the subtree generator's image sections (GenExpr[n_ex] at
// offset 0, each section 16-byte aligned): GenNt[n_nts]; head[depth_count *
// logical_count * n_nts], the widest GenLevel of each nonterminal at each
// (depth, site budget) (0: no precomputed draw); the GenLevel table (level 0
// is the empty one) and GenEntry table, each record held once however many
// heads share it; gagp_domain[n_doms]; gagp_value[n_vals]; the minimum cost
// table as uint16 (kNoMinimum16: infeasible).
struct GenImage {
  int32_t nt, head, level, entry, doms, vals, minimum;
  int32_t extra;  // children 4..7 of each expression and their scopes (two int4), when an arity exceeds 4
};
constexpr uint16_t kNoMinimum16 = 0xffff;

// A traversal table entry (the reference's PhaseRegionInfo for a traversal,
// device/phase_compile.cuh:47-60) as lowering reads it: direction, the
// binder numbers of element, index and state, the operand types the
// children must complete with, the binding types and the result type.
struct RegionInfo {
  int8_t traversal;       // 1 forward, 2 reverse; 0 a bounded region
  int8_t ranged;          // 0: (source, start, initial state, body)
  int8_t arity;           // 4, or 6 when ranged; a bounded region: operands + phases
  int8_t result_type;     // ValueTag of the traversal's (or the bounded region's) result
  int8_t binders[3];
  int8_t binding_types[3];
  int8_t operand_types[6];
  // a bounded region: a coordinate recurrence (gagp_region's bounded fields)
  int8_t operands, phases, captures, state_count, request_count, axis_count, inclusive, memoized;
  int8_t capture_kind[8], capture_target[8];
  int8_t phase_type[4], phase_bindings[4];
  int8_t binding_bank[4][8], binding_slot[4][8], phase_binding_types[4][8];
  int8_t transition_kind[8][4], transition_source[8][4];
  int8_t axis_slot[4], lower_kind[4], upper_kind[4];
  uint32_t frames, cells, entry_fuel;
  // a traversal's fuel profile: each event's first instruction carries its
  // charge, the rest none (PhaseFuelEvent numbering); off: every instruction costs 1
  int32_t fuel_profile;
  uint32_t event_cost[26];
  int64_t transition_offset[8][4];
  int64_t lower[4], upper[4];
};
// The device view of a region table entry (gagp_region), traversal or
// bounded region (a bounded one checked by the engine's admission).
inline RegionInfo region_info_of(const gagp_region& x) {
  RegionInfo y{};
  y.fuel_profile = x.fuel_profile ? 1 : 0;
  for (int k = 0; k < 26; ++k) y.event_cost[k] = x.event_cost[k];
  y.traversal = int8_t(x.traversal);
  y.ranged = int8_t(x.ranged);
  y.arity = int8_t(x.ranged ? 6 : 4);
  y.result_type = int8_t(x.result_type);
  for (int k = 0; k < 3; ++k) {
    y.binders[k] = int8_t(x.binders[k]);
    y.binding_types[k] = int8_t(x.binding_types[k]);
  }
  if (x.traversal == 0) {
    // a bounded region (checked by check_tables_and_cases)
    y.arity = int8_t(x.operands + x.phases);
    y.operands = int8_t(x.operands); y.phases = int8_t(x.phases); y.captures = int8_t(x.captures);
    y.state_count = int8_t(x.state_count); y.request_count = int8_t(x.request_count);
    y.axis_count = int8_t(x.axis_count); y.inclusive = int8_t(x.inclusive != 0); y.memoized = int8_t(x.memoized != 0);
    for (int c = 0; c < 8; ++c) { y.capture_kind[c] = int8_t(x.capture_kind[c]); y.capture_target[c] = int8_t(x.capture_target[c]); }
    for (int p = 0; p < 4; ++p) {
      y.phase_type[p] = int8_t(x.phase_type[p]);
      y.phase_bindings[p] = int8_t(x.phase_bindings[p]);
      for (int b = 0; b < 8; ++b) {
        y.binding_bank[p][b] = int8_t(x.binding_bank[p][b]);
        y.binding_slot[p][b] = int8_t(x.binding_slot[p][b]);
        y.phase_binding_types[p][b] = int8_t(x.phase_binding_types[p][b]);
      }
    }
    for (int q = 0; q < 8; ++q)
      for (int k = 0; k < 4; ++k) {
        y.transition_kind[q][k] = int8_t(x.transition_kind[q][k]);
        y.transition_source[q][k] = int8_t(x.transition_source[q][k]);
        y.transition_offset[q][k] = x.transition_offset[q][k];
      }
    for (int a = 0; a < 4; ++a) {
      y.axis_slot[a] = int8_t(x.axis_slot[a]);
      y.lower_kind[a] = int8_t(x.lower_kind[a]); y.upper_kind[a] = int8_t(x.upper_kind[a]);
      y.lower[a] = x.lower[a]; y.upper[a] = x.upper[a];
    }
    y.frames = x.frames; y.cells = x.cells; y.entry_fuel = x.entry_fuel;
    for (int k = 0; k < 4; ++k) y.operand_types[k] = int8_t(k < x.operands ? x.operand_types[k] : 0);
  }
  for (int k = 0; k < 6; ++k) y.operand_types[k] = int8_t(x.operand_types[k]);
  return y;
}

// Frames, memo cells and their int64 words in one lane's bounded-region
// workspace: a frame holds the states, the request results and the next
// request; a cell the states and the value.
__host__ __device__ inline size_t region_lane_words(const RegionInfo& r) {
  return size_t(r.frames) * (r.state_count + r.request_count + 1) + size_t(r.cells) * (r.state_count + 1);
}

// Everything a kernel needs to work on one search (device pointers).
struct SearchDesc {
  // ---- admitted grammar (phase tables)
  const gagp_expression* ex;
  const ExprInfo* info;
  const gagp_production* prods;
  const gagp_nonterminal* nts;
  const gagp_domain* doms;
  const gagp_value* vals;
  const uint32_t* minimum;
  // minimum of each production's expression, production-major per (depth,
  // site budget): prod_minimum[(d * logical_count + l) * n_prods + p]
  const uint32_t* prod_minimum;
  // the subtree generator's tables (GenImage layout), gen_image_bytes long
  const char* gen_image;
  int32_t gen_image_bytes;
  GenImage gi;
  const int32_t* local_types;          // ValueTag of each evaluator input
  const RegionInfo* regions;           // traversal table entries (TK_TRAVERSE operands)
  int32_t n_regions;
  int32_t n_ex, n_prods, n_nts, n_doms, n_vals;
  int32_t depth_count, logical_count, site_depth;
  int32_t root_expression, slot_max_depth, slot_type, local_count;
  int32_t result_type;                 // ValueTag a program returns (slot_type, or a statement program's return type)
  int32_t unit_fuel;                   // every instruction costs 1 (else no program takes the accumulator VM)
  int32_t max_nodes, fixed_nodes;
  uint32_t return_fuel;
  // ---- config
  int32_t P, B, maxv, stride;          // stride: row slots (>= maxv, multiple of 4)
  int32_t pressure, attempts, mutation_max_nodes;
  int32_t counted, uniform_phase, replacement_size, has_wrong, grammar_sites;
  int32_t metric, fuel;
  double crossover_probability, mutation_probability, penalty;
  int64_t penalty_int;                 // |penalty| when integral
  uint64_t seed;
  int32_t rounds_per_epoch;            // P / B (1 for the generational schedule)
  int32_t generations;
  // generational schedule (run_phase_population, evolve.cpp:253-322): every
  // round replaces the whole population (B = P), its first elite_count
  // children by the elites of the ranking
  int32_t generational, elite_count;
  int32_t imported;  // the members were imported (no initial generation)
  // ---- cases (input-major: inputs[j * C + c]); an IntList input's value is
  // the offset in `lists` of its length word, its elements following
  const int64_t* inputs;
  const int64_t* expected;
  const int64_t* lists;
  int64_t n_lists;                     // words in `lists`
  int32_t C, n_inputs, expected_tag, vm_cases_per_lane;
  // ---- population rows (members) and children
  uint64_t* node;     int64_t* cval;     int32_t* len;        // P member rows (node words, constants)
  uint64_t* cnode;    int64_t* ccval;    int32_t* clen;       // B child rows
  // ---- member statistics; key: packed ranking key (smaller is better)
  double* fitness; uint32_t* wrong; uint32_t* nodes; uint64_t* key;
  uint32_t* errors;  // row evaluation only (null otherwise): cases that ended in a runtime error
  // ---- per-child results of one round
  int32_t* c_parent; int32_t* c_reuse; int32_t* c_error;
  double* c_fitness; uint32_t* c_wrong; uint32_t* c_nodes; uint64_t* c_key;
  int32_t* c_eval;                     // 1: evaluate this child
  // ---- member index of one round: open addressing over mtab_mask + 1
  // slots (at least 2P) holding one member per distinct row, each slot
  // word the row hash's top 44 bits << 20 | member + 1 (0: empty)
  unsigned long long* mtab; int32_t mtab_mask;
  // ---- lowered programs (children, or members during the initial evaluation)
  uint2* code; int32_t* code_len; int64_t* kpool;
  int32_t code_stride;                 // accumulator instructions per program slot
  int32_t* code_temps;                 // temporaries; <0: needs the general VM
  // per program slot, the fast VM's tile accumulators: [2 slot] loss (bits
  // 0-39) | wrong cases (40-55) | tiles done (56-63) when the search's case
  // count and penalty fit those fields; otherwise [2 slot] the loss sum and
  // [2 slot + 1] wrong cases (low 32 bits) | tiles done (high 32 bits)
  unsigned long long* vm_acc;
  int32_t* bc;                         // reference bytecode (op,flags,a,b,fuel) per program
  int32_t* bc_len;
  int32_t* bc_locals;                  // per lowered program: locals (inputs + temporaries) | stack bound << 8
  int64_t* bc_consts;
  int32_t bc_stride;                   // instructions per program slot
  // ---- run generator (MT19937-64) and its output stream
  uint64_t* mt;                        // 312 words
  uint64_t* stream;                    // buffered outputs
  uint32_t* stream_mod;                // outputs % P
  long long* stream_head;              // [0]: outputs read, [1]: outputs written (ring positions)
  int32_t stream_capacity;
  uint64_t mod_magic;                  // floor((2^64 - 1) / P): exact residues by multiply-high
  uint64_t bounded_threshold;          // (2^64 - P) mod P: rejection bound of bounded(P)
  uint64_t* round_seed;                // seed of the next round's variation
  // ---- search progress and history
  int32_t* best;                       // tracked best member
  int32_t* elites;                     // generational: the elite_count best members, best first
  int32_t* placed;                     // P: child placed into member, -1
  int32_t* place_state;                // 1: the cluster placement placed this round
  int16_t* child_level;                // B: placement level of each child (k_place_levels)
  int32_t* level_plan;                 // [0] round + 1 the levels belong to, [1] number of levels
  int32_t* round;                      // [0] rounds done, [1] history entries, [2] finished flag, [3] error
  int64_t* hist_sum;                   // per history entry: sum of member fitness (integral)
  double* hist_fitness; uint32_t* hist_wrong; uint32_t* hist_nodes;
  uint64_t* hist_node; int64_t* hist_cval; int32_t* hist_len;
  uint64_t* counters;                  // GAGP_COUNTERS work counters (gagp_b200_search_counters)
  int32_t key_shift_wrong, key_shift_nodes; // packed key layout
  int32_t total_rounds;
};

}  // namespace gb
