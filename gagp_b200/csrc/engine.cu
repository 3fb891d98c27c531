// Host side of the B200 resident GAGP engine: admission, device memory,
// launch sequences and the C ABI of include/gagp_b200.h.
//
// One engine per device.  A search owns one device allocation holding its
// tables, cases, population rows, child rows, lowered programs, run-generator
// stream and history; it stays resident between generations.  A batch is any
// set of searches advanced together: every kernel takes the batch's
// descriptor array and flat item offsets, so one launch sequence advances all
// of them by one round.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <chrono>
#include <deque>
#include <map>
#include <tuple>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "kernels.cuh"

namespace {

thread_local std::string g_error;

gagp_status fail(gagp_status status, const std::string& message) {
  g_error = message;
  return status;
}

#define CUDA_TRY(expr)                                                                    \
  do {                                                                                    \
    const cudaError_t e_ = (expr);                                                        \
    if (e_ != cudaSuccess) return fail(GAGP_DEVICE_ERROR, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
  } while (0)

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Sub-allocation plan of one search's device block.
struct Layout {
  size_t total = 0;
  size_t take(size_t bytes) {
    const size_t at = align_up(total, 256);
    total = at + bytes;
    return at;
  }
};

struct Search {
  int id = 0;
  gb::SearchDesc desc{};
  char* block = nullptr;
  size_t bytes = 0;
  int P = 0, B = 0, G = 0, total_rounds = 0, maxv = 0, stride = 0, fixed_nodes = 0;
  int has_wrong = 0;
  bool started = false;
  // most of its programs need the exact VM (traversals, or operations that
  // can fail); otherwise only the rare program past the accumulator VM's
  // limits does
  bool exact_heavy = false;
  size_t region_words = 0;  // the largest bounded-region plan's workspace per lane (0: none)
  gb::SearchDesc* d_desc = nullptr;   // single-search batch descriptor
  int32_t* d_off = nullptr;           // {0, P, 0, B}: member and child offsets
};

}  // namespace

struct gagp_engine {
  int device = 0;
  cudaStream_t stream = nullptr;
  // side stream of the run-generator top-up, forked from and joined to `stream`
  cudaStream_t side = nullptr;   // member index and history entry
  cudaStream_t draws = nullptr;  // run generator and placement levels
  cudaEvent_t fork = nullptr, join = nullptr, indexed = nullptr, drawn = nullptr;
  // the children of a round in kChunks ranges, each varied, lowered and
  // evaluated on its own stream so that one range's slowest children
  // overlap the other ranges' work
  static constexpr int kChunks = 8;
  cudaStream_t chunk_stream[kChunks] = {};
  cudaEvent_t chunk_fork = nullptr, chunk_done[kChunks] = {};
  std::map<int, std::unique_ptr<Search>> searches;
  int next_id = 1;
  uint64_t arena_limit = 0, arena_used = 0;
  int sm_count = 0;
  size_t max_smem = 0;
  // batch scratch
  gb::ProgramRef* d_fast = nullptr;
  gb::ProgramRef* d_general = nullptr;
  gb::ProgramRef* d_region = nullptr;  // programs with bounded regions, deferred by the exact VM
  int32_t* d_counts = nullptr;
  // the bounded-region kernel's frame and memo workspace: region_ws_words
  // int64 words per lane, region_lanes lanes (sized by the largest plan admitted)
  int64_t* region_ws = nullptr;
  size_t region_ws_words = 0;
  int region_lanes = 0;
  size_t list_capacity = 0;
  gb::SearchDesc* d_batch_desc = nullptr;
  size_t batch_desc_capacity = 0;
  int32_t* d_batch_off = nullptr;
  size_t batch_off_capacity = 0;
  bool poisoned = false;
  // per-kernel CUDA-event timing (bench/profiling)
  bool profiling = false;
  std::vector<cudaEvent_t> event_pool;
  size_t event_next = 0;
  struct Pending { int kernel; cudaEvent_t start, stop; };
  std::vector<Pending> pending;
  // the launches of the last harvested batch of rounds: kernel, start and
  // end (ms after the batch's first timed launch started)
  struct Span { int kernel; float start, end; };
  std::vector<Span> timeline;
  double kernel_ms[16] = {};
  long long kernel_launches[16] = {};
  void* flush_buffer = nullptr;
  size_t flush_bytes = 0;
  // bytes copied host->device and device->host by this engine's API calls
  uint64_t h2d_bytes = 0, d2h_bytes = 0;
  // stream-ordered pool of the searches' device blocks: admission and
  // retirement neither allocate from the driver nor synchronize the device
  cudaMemPool_t pool = nullptr;
  // pinned staging of result downloads (grown on demand)
  char* pinned = nullptr;
  size_t pinned_bytes = 0;
  // VM autotuner: per batch shape, the fast VM's cases per lane, chosen by
  // timing each candidate on live rounds (results do not depend on it)
  struct VmTune {
    double ms[3] = {0, 0, 0};
    int rounds[3] = {0, 0, 0};
    int pending = 0;
    int chosen = -1;
  };
  std::map<uint64_t, VmTune> vm_tune;
  struct TuneMark { uint64_t key; int cand; cudaEvent_t start, stop; };
  std::vector<TuneMark> tune_marks;
};

namespace {
// Engine copies, counted for gagp_b200_engine_transfers.
cudaError_t copy_h2d(gagp_engine* e, void* dst, const void* src, size_t bytes) {
  e->h2d_bytes += bytes;
  return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, e->stream);
}
cudaError_t copy_d2h(gagp_engine* e, void* dst, const void* src, size_t bytes) {
  e->d2h_bytes += bytes;
  return cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost);
}
}  // namespace

namespace {

enum KernelId {
  KN_INIT, KN_LOWER, KN_VM_FAST, KN_KEYS, KN_START, KN_RECORD, KN_VARY, KN_CHILD, KN_PLACE,
  KN_COMMIT, KN_STREAM, KN_LEVELS, KN_VM_GENERAL, KN_INDEX, KN_COUNT
};
const char* const kKernelNames[KN_COUNT] = {"k_init_population", "k_lower", "k_vm_fast",
                                            "k_member_keys", "k_start", "k_record", "k_vary", "k_child_results",
                                            "k_place", "k_commit", "k_stream", "k_place_levels", "k_vm_general",
                                            "k_member_index"};

cudaEvent_t take_event(gagp_engine* e) {
  if (e->event_next == e->event_pool.size()) {
    cudaEvent_t ev;
    cudaEventCreate(&ev);
    e->event_pool.push_back(ev);
  }
  return e->event_pool[e->event_next++];
}
// Brackets one kernel launch with events on the engine stream when profiling.
struct Timed {
  gagp_engine* e;
  int kernel;
  cudaEvent_t stop = nullptr;
  cudaStream_t stream;
  Timed(gagp_engine* engine, int k, cudaStream_t on = nullptr) : e(engine), kernel(k), stream(on ? on : engine->stream) {
    if (!e->profiling) return;
    cudaEvent_t start = take_event(e);
    stop = take_event(e);
    cudaEventRecord(start, stream);
    e->pending.push_back({kernel, start, stop});
  }
  ~Timed() {
    if (stop) cudaEventRecord(stop, stream);
  }
};
// Adds the elapsed times of completed launches (after a stream sync).
// Fast-VM cases per lane, the autotuner's candidates.
constexpr int kVmLanes[3] = {1, 2, 4};
// rounds the VM autotuner times per candidate, in the order 1, 2, 4, 4, 2, 1
// cases per lane (so that a drift over the first rounds favours none)
constexpr int kTuneRounds = 2;

void harvest(gagp_engine* e) {
  if (!e->pending.empty()) e->timeline.clear();
  for (const auto& p : e->pending) {
    float ms = 0, at = 0;
    if (cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
      e->kernel_ms[p.kernel] += ms;
      e->kernel_launches[p.kernel] += 1;
      if (cudaEventElapsedTime(&at, e->pending[0].start, p.start) == cudaSuccess)
        e->timeline.push_back({p.kernel, at, at + ms});
    }
  }
  e->pending.clear();
  // VM autotuner: once every candidate's round has been timed, keep the
  // fastest (mean fast-VM time per round)
  for (const auto& m : e->tune_marks) {
    float ms = 0;
    auto& t = e->vm_tune[m.key];
    if (cudaEventElapsedTime(&ms, m.start, m.stop) == cudaSuccess) t.ms[m.cand] += ms;
    --t.pending;
  }
  for (const auto& m : e->tune_marks) {
    auto& t = e->vm_tune[m.key];
    if (t.chosen >= 0 || t.pending > 0 || t.rounds[0] < kTuneRounds || t.rounds[1] < kTuneRounds ||
        t.rounds[2] < kTuneRounds)
      continue;
    int best = 0;
    for (int c = 1; c < 3; ++c)
      if (t.ms[c] / t.rounds[c] < t.ms[best] / t.rounds[best]) best = c;
    t.chosen = best;
  }
  e->tune_marks.clear();
  e->event_next = 0;
}

// Device counters of a round: per variation range c, [4c] and [4c+1] its
// lowered-program list sizes (fast, exact) and [4c+2] its next child; then
// [4 kChunks + 1] the size of the shared exact-VM list of a round whose
// ranges hand their exact-VM programs to one launch.
constexpr int kCountWords = 4 * gagp_engine::kChunks + 4;
// [4 kChunks + 2]: the size of the deferred bounded-region program list
constexpr int kRegionCount = 4 * gagp_engine::kChunks + 2;
gagp_status ensure_region_workspace(gagp_engine* e, size_t words);

gagp_status ensure_lists(gagp_engine* e, size_t items) {
  if (items <= e->list_capacity) return GAGP_OK;
  if (e->d_fast) cudaFree(e->d_fast);
  if (e->d_general) cudaFree(e->d_general);
  if (e->d_region) cudaFree(e->d_region);
  e->d_fast = e->d_general = e->d_region = nullptr;
  e->list_capacity = 0;
  const size_t cap = std::max<size_t>({items, size_t(1024), 2 * e->list_capacity});
  CUDA_TRY(cudaMalloc(&e->d_fast, cap * sizeof(gb::ProgramRef)));
  CUDA_TRY(cudaMalloc(&e->d_general, cap * sizeof(gb::ProgramRef)));
  CUDA_TRY(cudaMalloc(&e->d_region, cap * sizeof(gb::ProgramRef)));
  if (!e->d_counts) CUDA_TRY(cudaMalloc(&e->d_counts, kCountWords * sizeof(int32_t)));
  e->list_capacity = cap;
  return GAGP_OK;
}

// Cases per lane of the fast VM for `cases` (the fewest warp passes with at
// most 4 cases per lane, the register budget of two resident blocks per SM).
int cases_per_lane(int cases) {
  if (cases <= 32) return 1;
  if (cases <= 64) return 2;
  return 4;
}

// Batch shape of the VM autotuner: case count rounded up to a power of two
// and the input count.
uint64_t vm_key(int max_C, int max_inputs) {
  uint64_t c = 1;
  while (c < uint64_t(max_C)) c <<= 1;
  return (c << 8) | uint64_t(max_inputs & 0xff);
}

int bits_for(uint64_t v) {
  int b = 0;
  while (b < 64 && (v >> b)) ++b;
  return b;
}

// A bounded region's table entry, in the subset the device runs: a
// coordinate recurrence of 1..4 Int states with at most 4 operands and the
// four phases, requests that copy or offset states, literal or operand
// coordinate bounds, at most 128 frames and 256 memo cells, phase bindings
// from the state, parameter and (in the combine phase) request-result
// banks.  The reference's grammar compiler and plan validation
// (region_plan.cpp) have checked the plan itself.
gagp_status check_bounded_region(const gagp_grammar* g, const gagp_region& x) {
  auto value_tag = [](int t) { return t == GAGP_TAG_INT || t == GAGP_TAG_BOOL || t == GAGP_TAG_INTLIST; };
  if (x.state_count < 1 || x.state_count > 4 || x.operands < x.state_count || x.operands > 4 || x.phases != 4)
    return fail(GAGP_DECLINED, "bounded regions other than coordinate recurrences of at most 4 operands");
  if (x.request_count < 1 || x.request_count > 8 || x.axis_count < 1 || x.axis_count > 4)
    return fail(GAGP_DECLINED, "bounded region request or axis count");
  if (x.frames > 128 || x.cells > 256 || x.entry_fuel > 0x7fffffffu)
    return fail(GAGP_DECLINED, "bounded region limits beyond 128 frames and 256 memo cells");
  if ((x.result_type != GAGP_TAG_INT && x.result_type != GAGP_TAG_BOOL) || x.phase_type[0] != GAGP_TAG_BOOL ||
      x.phase_type[1] != x.result_type || x.phase_type[2] != x.result_type || x.phase_type[3] != x.result_type)
    return fail(GAGP_DECLINED, "bounded region phase types");
  for (int k = 0; k < x.operands; ++k)
    if (x.operand_types[k] != GAGP_TAG_INT) return fail(GAGP_DECLINED, "bounded region operands other than Int");
  if (x.captures < 0 || x.captures > 8) return fail(GAGP_INVALID_ARGUMENT, "bounded region captures");
  for (int c = 0; c < x.captures; ++c) {
    const int kind = x.capture_kind[c], t = x.capture_target[c];
    if (!value_tag(x.parameter_types[c])) return fail(GAGP_DECLINED, "bounded region parameter type");
    if ((kind == 0 && (t < 0 || t >= g->local_count)) || (kind == 1 && (t < 0 || t >= gb::kNamedLocals)) ||
        (kind == 2 && (t < 0 || t >= gb::kLowerBinders)) || kind < 0 || kind > 2)
      return fail(GAGP_INVALID_ARGUMENT, "bounded region capture");
  }
  for (int p = 0; p < 4; ++p) {
    if (x.phase_bindings[p] < 0 || x.phase_bindings[p] > 7) return fail(GAGP_DECLINED, "bounded region phase bindings");
    for (int b = 0; b < x.phase_bindings[p]; ++b) {
      const int bank = x.binding_bank[p][b], slot = x.binding_slot[p][b], t = x.phase_binding_types[p][b];
      const bool ok = (bank == 0 && slot >= 0 && slot < x.state_count && t == GAGP_TAG_INT) ||
                      (bank == 1 && slot >= 0 && slot < x.captures && t == x.parameter_types[slot]) ||
                      (bank == 3 && p == 2 && slot >= 0 && slot < x.request_count && t == x.result_type);
      if (!ok) return fail(GAGP_DECLINED, "bounded region binding outside the state, parameter and result banks");
    }
  }
  for (int q = 0; q < x.request_count; ++q)
    for (int k = 0; k < x.state_count; ++k)
      if ((x.transition_kind[q][k] != 0 && x.transition_kind[q][k] != 1) || x.transition_source[q][k] < 0 ||
          x.transition_source[q][k] >= x.state_count)
        return fail(GAGP_DECLINED, "bounded region transitions other than state copies and coordinate offsets");
  for (int a = 0; a < x.axis_count; ++a) {
    if (x.axis_slot[a] < 0 || x.axis_slot[a] >= x.state_count) return fail(GAGP_INVALID_ARGUMENT, "bounded region axis");
    if ((x.lower_kind[a] == 1 && (x.lower[a] < 0 || x.lower[a] >= x.operands)) ||
        (x.upper_kind[a] == 1 && (x.upper[a] < 0 || x.upper[a] >= x.operands)) || x.lower_kind[a] < 0 ||
        x.lower_kind[a] > 1 || x.upper_kind[a] < 0 || x.upper_kind[a] > 1)
      return fail(GAGP_INVALID_ARGUMENT, "bounded region coordinate bound");
  }
  return GAGP_OK;
}

// The value type a program of `g` returns: the phase type of an expression
// entry; for a statement program (a Program entry, whose phase completes as
// a statement) the type its returns carry, which the grammar makes the
// entry's result contract (compiled.cpp:512-513).
int result_type_of(const gagp_grammar* g) {
  if (!gb::is_statement_tag(g->slot_type)) return g->slot_type;
  for (int i = 0; i < g->expression_count; ++i) {
    const gagp_expression& e = g->expressions[i];
    if (e.kind == gb::EK_OPERATION && e.node_kind == gb::TK_RETURN) return e.type;
  }
  return GAGP_TAG_INVALID;
}

// The phase tables, traversal table and cases as the device reads them:
// every id the subtree generator and the lowering follow without a range
// check is in range, and every IntList input lies inside list_values.
// GAGP_DECLINED for constructs outside the resident subset.
gagp_status check_tables_and_cases(const gagp_grammar* g, const gagp_cases* c) {
  // the subtree generator and the lowering read these tables without range
  // checks: every id they hold must be in range
  const int E = g->expression_count, NT = g->nonterminal_count, PR = g->production_count, ND = g->domain_count;
  const int RG = g->region_count;
  if (RG < 0 || RG > 1024 || (RG && !g->regions)) return fail(GAGP_INVALID_ARGUMENT, "traversal table");
  auto value_tag = [](int t) { return t == GAGP_TAG_INT || t == GAGP_TAG_BOOL || t == GAGP_TAG_INTLIST; };
  for (int r = 0; r < RG; ++r) {
    const gagp_region& x = g->regions[r];
    if (x.traversal == 0) {
      if (const gagp_status st = check_bounded_region(g, x); st != GAGP_OK) return st;
      continue;
    }
    if (x.traversal != 1 && x.traversal != 2)
      return fail(GAGP_INVALID_ARGUMENT, "region table entry kind");
    if (x.ranged) return fail(GAGP_DECLINED, "ranged traversals are outside the resident subset");
    if (x.fuel_profile)
      for (int k = 0; k < 26; ++k)
        if (x.event_cost[k] < 1 || x.event_cost[k] > 0x7fffffffu)
          return fail(GAGP_DECLINED, "zero-cost traversal events are outside the resident subset");
    for (int k = 0; k < 3; ++k) {
      if (x.binders[k] < 0 || x.binders[k] >= gb::kLowerBinders) return fail(GAGP_INVALID_ARGUMENT, "traversal binder");
      if (!value_tag(x.binding_types[k])) return fail(GAGP_DECLINED, "traversal binding type");
    }
    for (int k = 0; k < 4; ++k)
      if (!value_tag(x.operand_types[k])) return fail(GAGP_DECLINED, "traversal operand type");
    if (!value_tag(x.result_type)) return fail(GAGP_DECLINED, "traversal result type");
  }
  for (int i = 0; i < E; ++i) {
    const gagp_expression& e = g->expressions[i];
    if (e.kind == gb::EK_ALIAS) return fail(GAGP_DECLINED, "templates are outside the resident subset");
    if (e.kind != gb::EK_REFERENCE && e.kind != gb::EK_CONSTANT && e.kind != gb::EK_OPERATION &&
        e.kind != gb::EK_INPUT && e.kind != gb::EK_BOUND)
      return fail(GAGP_INVALID_ARGUMENT, "expression " + std::to_string(i) + ": unknown kind");
    if (e.kind == gb::EK_REFERENCE && (e.scope_count < 0 || e.scope_count > 15))
      return fail(GAGP_INVALID_ARGUMENT, "reference scope");
    if (e.kind == gb::EK_OPERATION && e.node_kind == gb::TK_TRAVERSE) {
      if (e.arity != 4 || e.operand < 0 || e.operand >= RG || g->regions[e.operand].traversal == 0)
        return fail(GAGP_INVALID_ARGUMENT, "expression " + std::to_string(i) + ": traversal entry");
    } else if (e.kind == gb::EK_OPERATION && e.node_kind == gb::TK_REGION) {
      if (e.operand < 0 || e.operand >= RG || g->regions[e.operand].traversal != 0 ||
          e.arity != g->regions[e.operand].operands + g->regions[e.operand].phases || e.arity > GAGP_MAX_ARITY)
        return fail(GAGP_INVALID_ARGUMENT, "expression " + std::to_string(i) + ": bounded region entry");
    } else if (e.arity < 0 || e.arity > 3) {
      return fail(GAGP_DECLINED, "arity capacity");
    }
    if (e.kind == gb::EK_OPERATION && e.node_kind != gb::TK_OPERATION && e.node_kind != gb::TK_IF &&
        e.node_kind != gb::TK_AND && e.node_kind != gb::TK_OR && e.node_kind != gb::TK_TRAVERSE &&
        e.node_kind != gb::TK_LET && e.node_kind != gb::TK_REGION && !(e.node_kind >= gb::TK_PROGRAM && e.node_kind <= gb::TK_VAR))
      return fail(GAGP_DECLINED, "tree kind outside the resident subset");
    if (e.kind == gb::EK_OPERATION && e.node_kind >= gb::TK_PROGRAM && e.node_kind <= gb::TK_VAR) {
      // statements belong to a Program entry's whole-program phase; a named
      // target is a grammar local or an input (-1 - its position)
      if (!gb::is_statement_tag(g->slot_type)) return fail(GAGP_INVALID_ARGUMENT, "a statement in a value phase");
      const int nk = e.node_kind;
      const int want = nk == gb::TK_NIL || nk == gb::TK_VAR ? 0 : nk == gb::TK_BLOCK || nk == gb::TK_FOR_RANGE ? 2 : 1;
      if (e.arity != want) return fail(GAGP_INVALID_ARGUMENT, "expression " + std::to_string(i) + ": statement arity");
      const bool named = nk == gb::TK_ASSIGN || nk == gb::TK_FOR_RANGE || nk == gb::TK_VAR;
      if (named && (e.operand >= gb::kNamedLocals || e.operand < -g->local_count || (nk == gb::TK_VAR && e.operand < 0)))
        return fail(GAGP_INVALID_ARGUMENT, "expression " + std::to_string(i) + ": statement target");
      if ((nk == gb::TK_RETURN || nk == gb::TK_VAR) && !value_tag(e.type))
        return fail(GAGP_DECLINED, "statement value type outside Int, Bool and IntList");
      if (nk == gb::TK_RETURN && result_type_of(g) != e.type)
        return fail(GAGP_INVALID_ARGUMENT, "returns of one program disagree on its result type");
    }
    if (e.kind == gb::EK_OPERATION && e.node_kind == gb::TK_LET &&
        (e.arity != 2 || e.operand < 0 || e.operand >= gb::kLowerBinders))
      return fail(GAGP_INVALID_ARGUMENT, "expression " + std::to_string(i) + ": let binder");
    if (e.kind == gb::EK_OPERATION && e.node_kind == gb::TK_OPERATION && e.opcode == gb::OP_CALL_BUILTIN &&
        e.operand != gb::B_ABS && e.operand != gb::B_MIN && e.operand != gb::B_MAX && e.operand != gb::B_LEN &&
        e.operand != gb::B_INDEX && e.operand != gb::B_IDIV0 && e.operand != gb::B_IMOD0 &&
        e.operand != gb::B_TRUNC_DIV0 && e.operand != gb::B_TRUNC_MOD0)
      return fail(GAGP_DECLINED, "builtin outside the resident subset");
    if (e.kind == gb::EK_BOUND && (e.arity != 0 || e.node_kind != gb::TK_BOUND || e.operand < 0 ||
                                   e.operand >= gb::kLowerBinders))
      return fail(GAGP_INVALID_ARGUMENT, "expression " + std::to_string(i) + ": bound read");
    if (e.kind == gb::EK_INPUT && (e.operand < 0 || e.operand >= g->local_count))
      return fail(GAGP_INVALID_ARGUMENT, "expression " + std::to_string(i) + ": input position");
    if (e.kind == gb::EK_REFERENCE) {
      if (e.target < 0 || e.target >= NT) return fail(GAGP_INVALID_ARGUMENT, "reference to a missing nonterminal");
      const gagp_nonterminal& n = g->nonterminals[e.target];
      if (n.production_count < 1 || n.production_offset < 0 || n.production_offset > PR ||
          n.production_count > PR - n.production_offset)
        return fail(GAGP_INVALID_ARGUMENT, "nonterminal " + std::to_string(e.target) + ": production range");
      for (int k = 0; k < n.production_count; ++k) {
        const int x = g->productions[n.production_offset + k].expression;
        if (x < 0 || x >= E) return fail(GAGP_INVALID_ARGUMENT, "production of a missing expression");
      }
    } else if (e.kind == gb::EK_CONSTANT) {
      if (e.arity != 0 || e.target < 0 || e.target >= ND) return fail(GAGP_INVALID_ARGUMENT, "constant domain");
    } else {
      for (int k = 0; k < e.arity; ++k)
        if (e.children[k] < 0 || e.children[k] >= E) return fail(GAGP_INVALID_ARGUMENT, "child of a missing expression");
    }
  }
  for (int j = 0; j < g->local_count; ++j)
    if (!value_tag(g->local_types[j])) return fail(GAGP_DECLINED, "input type outside Int, Bool and IntList");
  if (c->expected_tag != GAGP_TAG_INT && c->expected_tag != GAGP_TAG_BOOL)
    return fail(GAGP_DECLINED, "expected outputs other than Int and Bool are outside the resident subset");
  // every IntList input is a length word and its elements inside list_values
  for (int j = 0; j < c->input_count; ++j) {
    if (!c->input_tags || c->input_tags[j] != g->local_types[j])
      return fail(GAGP_INVALID_ARGUMENT, "case input tags must equal the grammar's input types");
    if (c->input_tags[j] != GAGP_TAG_INTLIST) continue;
    if (!c->list_values || c->list_value_count < 1) return fail(GAGP_INVALID_ARGUMENT, "IntList inputs need list_values");
    for (int k = 0; k < c->case_count; ++k) {
      const int64_t at = c->inputs[size_t(k) * c->input_count + j];
      if (at < 0 || at >= c->list_value_count) return fail(GAGP_INVALID_ARGUMENT, "IntList input outside list_values");
      const int64_t len = c->list_values[at];
      if (len < 0 || len > c->list_value_count - at - 1)
        return fail(GAGP_INVALID_ARGUMENT, "IntList input overruns list_values");
    }
  }
  return GAGP_OK;
}

// Admission checks of this engine (a decline reruns on the native path in
// the reference).  Returns GAGP_OK or GAGP_DECLINED with a reason.
gagp_status admit(const gagp_grammar* g, const gagp_cases* c, const gagp_search_config* cfg) {
  if (!g || !c || !cfg) return fail(GAGP_INVALID_ARGUMENT, "null argument");
  if (cfg->population < 1 || cfg->population > 16384) return fail(GAGP_DECLINED, "population/grammar capacity");
  if (cfg->steady_state) {
    // with one member every replacement draw is the best member, which the
    // steady-state loop redraws without end (evolve.cpp:331-441)
    if (cfg->population < 2) return fail(GAGP_INVALID_ARGUMENT, "steady-state replacement needs at least 2 members");
    const int B = cfg->batch > 0 ? cfg->batch : cfg->population;
    if (B > cfg->population || cfg->population % B)
      return fail(GAGP_INVALID_ARGUMENT, "steady-state batch must divide the population");
    if (cfg->replacement_size < 1 || cfg->replacement_size > 64) return fail(GAGP_INVALID_ARGUMENT, "replacement_size");
  } else {
    // reproduce's elite contract (phase_population_cpu.cpp:271)
    if (cfg->elite_count < 0 || cfg->elite_count >= cfg->population)
      return fail(GAGP_INVALID_ARGUMENT, "elite count must be in [0, population)");
    if (cfg->elite_count > gb::kMaxElites) return fail(GAGP_DECLINED, "more elites than the device keeps");
  }
  if (cfg->generations < 1) return fail(GAGP_INVALID_ARGUMENT, "generations must be > 0");
  if (cfg->tournament_size < 1 || cfg->crossover_attempts < 1 || cfg->crossover_attempts > 64)
    return fail(GAGP_INVALID_ARGUMENT, "selection/crossover contract");
  if (!(cfg->mutation_probability >= 0 && cfg->mutation_probability <= 1) ||
      !(cfg->crossover_probability >= 0 && cfg->crossover_probability <= 1))
    return fail(GAGP_INVALID_ARGUMENT, "probabilities must be in [0,1]");
  if (cfg->metric != GAGP_METRIC_ABSOLUTE && cfg->metric != GAGP_METRIC_EXACT)
    return fail(GAGP_DECLINED, "fitness metric outside the resident scalar subset");
  const double pen = std::fabs(cfg->penalty);
  if (pen != std::floor(pen) || pen < 1 || pen > 2147483647.0)
    return fail(GAGP_DECLINED, "a fractional penalty needs the ordered 48-bit reduction");
  if (double(c->case_count) * pen >= 281474976710656.0) return fail(GAGP_DECLINED, "cases * penalty must stay below 2^48");
  if (c->case_count < 1 || c->case_count > (1 << 20)) return fail(GAGP_INVALID_ARGUMENT, "case count");
  if (c->input_count != g->local_count || g->local_count > GAGP_MAX_LOCALS)
    return fail(GAGP_INVALID_ARGUMENT, "case inputs must cover the grammar inputs");
  if (g->expression_count < 1 || g->expression_count > 65534) return fail(GAGP_DECLINED, "expression table capacity");
  if (g->site_depth < 1 || g->site_depth > 15) return fail(GAGP_DECLINED, "the device population is grown under a site-depth limit");
  const int maxv = g->max_nodes - g->fixed_nodes;
  if (maxv < 1 || maxv > gb::kMaxLowerNodes) return fail(GAGP_DECLINED, "variable node budget outside 1..256");
  if (g->slot_max_depth < 1 || g->slot_max_depth >= g->depth_count || g->depth_count > 65)
    return fail(GAGP_DECLINED, "depth budget");
  if (const gagp_status st = check_tables_and_cases(g, c); st != GAGP_OK) return st;
  const int ND = g->domain_count;
  for (int i = 0; i < ND; ++i) {
    const gagp_domain& d = g->domains[i];
    if (d.integer_range) {
      if (d.minimum > d.maximum) return fail(GAGP_INVALID_ARGUMENT, "empty integer domain");
    } else {
      if (d.value_count < 1 || d.value_offset < 0 || d.value_offset > g->value_count ||
          d.value_count > g->value_count - d.value_offset)
        return fail(GAGP_INVALID_ARGUMENT, "domain value range");
      for (int k = 0; k < d.value_count; ++k)
        if (g->values[d.value_offset + k].tag != GAGP_TAG_INT)
          return fail(GAGP_DECLINED, "only Int constants are resident");
    }
  }
  return GAGP_OK;
}

// Precomputed production draws (generate_phase's weighted choice,
// cpp/src/evolution/repro/gpu/device/phase_generate.cuh:125-270).  At a
// given (depth, site budget) a production is feasible when its minimum cost
// fits the room left, so the feasible productions of a nonterminal are
// always those whose cost is at most one of the distinct costs among its
// productions: one level per distinct cost.  For each level the choice
// value c = u * total is compared against thresholds instead of subtracting
// the weights one by one: with f_i(c) = (((c - v_0) - v_1) ... - v_i) over
// the level's productions, each step rounded to nearest in double
// precision, f_i is non-decreasing in c, so f_i(c) < 0 exactly when c is
// below the smallest double T_i with f_i(T_i) >= 0, found by bisection over
// the bit patterns of non-negative doubles.  The first production whose
// threshold exceeds c is the one the sequential loop stops at (the last
// feasible one when none does).  Levels with the same feasible set share
// their draw; past kMaxDrawEntries the remaining nonterminals keep the
// sequential draw.
constexpr size_t kMaxDrawEntries = size_t(1) << 16;

struct DrawTables {
  std::vector<uint32_t> head;  // per (depth, site budget, nonterminal): its widest level (0: none)
  std::vector<gb::GenLevel> level;
  std::vector<gb::GenEntry> entry;
};

// `with_draws` false: only the table sizes (for the memory plan).
DrawTables draw_tables(const gagp_grammar* g, bool with_draws) {
  const int E = g->expression_count, PR = g->production_count, NT = g->nonterminal_count;
  const int DC = g->depth_count, LC = g->logical_depth_count;
  DrawTables t;
  const size_t heads = size_t(std::max(1, NT)) * DC * LC;
  gb::GenLevel none{};
  none.total = std::nan("");
  none.bound = gb::kNoId;
  none.entry = 0;
  none.last = -1;
  none.below = -1;
  t.level.assign(1, none);  // level 0: no precomputed draw
  t.head.assign(heads, 0);
  struct Draw { double total; int last; std::vector<double> threshold; };
  std::map<std::pair<int, std::vector<uint8_t>>, Draw> memo;
  auto from_bits = [](uint64_t b) { double d; std::memcpy(&d, &b, sizeof d); return d; };
  auto draw_of = [&](int nt, const std::vector<uint8_t>& feasible) -> const Draw& {
    auto it = memo.find({nt, feasible});
    if (it != memo.end()) return it->second;
    const gagp_nonterminal& n = g->nonterminals[nt];
    const int off = n.production_offset, cnt = n.production_count;
    Draw dr{std::nan(""), -1, std::vector<double>(cnt, 0.0)};
    double maximum = n.normalized_weights ? 1.0 : 0.0;
    for (int i = 0; i < cnt; ++i)
      if (feasible[i] && !n.normalized_weights && g->productions[off + i].weight > maximum)
        maximum = g->productions[off + i].weight;
    if (maximum > 0) {
      std::vector<double> v(cnt, 0.0);
      double total = 0.0;
      for (int i = 0; i < cnt; ++i)
        if (feasible[i]) {
          const double w = g->productions[off + i].weight;
          v[i] = n.normalized_weights ? w : w / maximum;
          total = total + v[i];
          dr.last = i;
        }
      auto f = [&](double c, int i) {
        double x = c;
        for (int k = 0; k <= i; ++k)
          if (feasible[k]) x = x - v[k];
        return x;
      };
      for (int i = 0; i < cnt; ++i) {
        if (!feasible[i] || f(0.0, i) >= 0) continue;  // threshold 0: never picked
        uint64_t lo = 0, hi = 0x7ff0000000000000ULL;   // f_i(lo) < 0 <= f_i(hi)
        while (hi - lo > 1) {
          const uint64_t mid = lo + (hi - lo) / 2;
          if (f(from_bits(mid), i) >= 0) hi = mid; else lo = mid;
        }
        dr.threshold[i] = from_bits(hi);
      }
      dr.total = total;
    }
    return memo.emplace(std::make_pair(nt, feasible), std::move(dr)).first->second;
  };
  std::map<std::tuple<int, uint32_t, std::vector<uint32_t>>, std::pair<uint32_t, std::pair<double, int>>> entry_memo;
  std::map<std::tuple<uint32_t, uint32_t, int32_t>, int32_t> level_memo;
  for (int nt = 0; nt < NT; ++nt) {
    const gagp_nonterminal& n = g->nonterminals[nt];
    const int off = n.production_offset, cnt = n.production_count;
    if (cnt <= 0 || off < 0 || off > PR || cnt > PR - off) continue;
    bool valid = true;
    for (int i = 0; i < cnt; ++i)
      if (g->productions[off + i].expression < 0 || g->productions[off + i].expression >= E) valid = false;
    if (!valid) continue;
    for (int d = 0; d < DC; ++d)
      for (int l = 0; l < LC; ++l) {
        std::vector<uint32_t> cost(cnt);
        for (int i = 0; i < cnt; ++i)
          cost[i] = g->minimum[(size_t(g->productions[off + i].expression) * DC + d) * LC + l];
        std::vector<uint32_t> bounds;
        for (uint32_t c : cost)
          if (c != gb::kNoId) bounds.push_back(c);
        std::sort(bounds.begin(), bounds.end());
        bounds.erase(std::unique(bounds.begin(), bounds.end()), bounds.end());
        if (bounds.empty() || t.entry.size() + bounds.size() * size_t(cnt) > kMaxDrawEntries) continue;
        // the chain from the narrowest level up: the widest is the head, the
        // narrower ones are shared by every head whose chain holds them.  A
        // level's entries depend only on (nonterminal, bound, costs), and a
        // narrower level on the same plus the levels below it, so equal keys
        // are equal records: the tables hold each once, which keeps the
        // generator's working set small
        int32_t below = -1;
        for (int k = 0; k < int(bounds.size()); ++k) {
          const std::vector<uint32_t> key_costs(cost.begin(), cost.end());
          const auto ekey = std::make_tuple(nt, bounds[k], key_costs);
          auto eit = entry_memo.find(ekey);
          if (eit == entry_memo.end()) {
            std::vector<uint8_t> feasible(cnt);
            for (int i = 0; i < cnt; ++i) feasible[i] = cost[i] <= bounds[k];
            const Draw* dr = with_draws ? &draw_of(nt, feasible) : nullptr;
            const uint32_t at = uint32_t(t.entry.size());
            for (int i = 0; i < cnt; ++i) {
              gb::GenEntry en{};
              en.threshold = dr ? dr->threshold[i] : 0.0;
              en.expression = g->productions[off + i].expression;
              en.need = cost[i];
              t.entry.push_back(en);
            }
            eit = entry_memo.emplace(ekey, std::make_pair(at, dr ? std::make_pair(dr->total, dr->last)
                                                                  : std::make_pair(0.0, -1))).first;
          }
          gb::GenLevel lv = none;
          lv.bound = bounds[k];
          lv.entry = eit->second.first;
          if (with_draws) {
            lv.total = eit->second.second.first;
            lv.last = eit->second.second.second;
          }
          lv.below = below;
          const auto lkey = std::make_tuple(lv.entry, lv.bound, lv.below);
          auto lit = level_memo.find(lkey);
          if (lit == level_memo.end()) {
            lit = level_memo.emplace(lkey, int32_t(t.level.size())).first;
            t.level.push_back(lv);
          }
          below = lit->second;
        }
        t.head[(size_t(d) * LC + l) * NT + nt] = uint32_t(below);  // the widest
      }
  }
  if (t.entry.empty()) t.entry.push_back(gb::GenEntry{});
  return t;
}

// The subtree generator's tables as one image (gb::GenImage sections, each
// 16-byte aligned), which the variation kernel copies into shared memory.
// `with_draws` false: the layout only.
struct GenImageLayout {
  gb::GenImage at;
  size_t bytes = 0;
};
GenImageLayout gen_image_layout(const gagp_grammar* g, const DrawTables& t) {
  GenImageLayout out;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t here = off;
    off = align_up(off + bytes, 16);
    return int32_t(here);
  };
  const int E = g->expression_count, NT = std::max(1, g->nonterminal_count);
  take(sizeof(gb::GenExpr) * size_t(E));  // expressions first: offset 0
  out.at.nt = take(sizeof(gb::GenNt) * size_t(NT));
  out.at.head = take(sizeof(uint32_t) * t.head.size());
  out.at.level = take(sizeof(gb::GenLevel) * t.level.size());
  out.at.entry = take(sizeof(gb::GenEntry) * t.entry.size());
  out.at.doms = take(sizeof(gagp_domain) * size_t(std::max(1, g->domain_count)));
  out.at.vals = take(sizeof(gagp_value) * size_t(std::max(1, g->value_count)));
  out.at.minimum = take(sizeof(uint16_t) * size_t(E) * g->depth_count * g->logical_depth_count);
  // children 4..7 (a bounded region's phases) only when an arity needs them
  int widest = 0;
  for (int i = 0; i < E; ++i)
    if (g->expressions[i].kind != gb::EK_REFERENCE) widest = std::max(widest, g->expressions[i].arity);
  out.at.extra = widest > 4 ? take(2 * sizeof(int4) * size_t(E)) : 0;
  out.bytes = off;
  return out;
}
std::vector<char> gen_image(const gagp_grammar* g, const std::vector<gb::ExprInfo>& info, const DrawTables& t,
                            const GenImageLayout& lay) {
  std::vector<char> img(lay.bytes, 0);
  const int E = g->expression_count;
  auto* gx = reinterpret_cast<gb::GenExpr*>(img.data());
  for (int i = 0; i < E; ++i) {
    const gagp_expression& x = g->expressions[i];
    gb::GenExpr& r = gx[i];
    for (int k = 0; k < 4; ++k) {
      r.child[k] = k < GAGP_MAX_ARITY ? x.children[k] : -1;
      r.child_scope[k] = k < GAGP_MAX_ARITY ? x.child_scope[k] : -1;
    }
    r.target = x.target;
    r.site_class = info[i].site_class;
    r.kind = int8_t(x.kind);
    r.arity = info[i].arity;
    if (lay.at.extra && r.arity > 4) {
      auto* extra = reinterpret_cast<int32_t*>(img.data() + lay.at.extra) + 8 * size_t(i);
      for (int k = 4; k < 8; ++k) {
        extra[k - 4] = x.children[k];
        extra[4] |= int32_t(uint32_t(uint8_t(x.child_scope[k])) << (8 * (k - 4)));
      }
    }
    // out-of-range counts keep their validity (admission bounds them anyway)
    r.scope_count = int8_t(std::min(std::max(x.scope_count, -1), 100));
    r.reserved = 0;
  }
  auto* nt = reinterpret_cast<gb::GenNt*>(img.data() + lay.at.nt);
  for (int i = 0; i < g->nonterminal_count; ++i) {
    const gagp_nonterminal& n = g->nonterminals[i];
    nt[i] = gb::GenNt{n.production_offset, n.production_count, n.scope_count, n.normalized_weights};
  }
  std::memcpy(img.data() + lay.at.head, t.head.data(), sizeof(uint32_t) * t.head.size());
  std::memcpy(img.data() + lay.at.level, t.level.data(), sizeof(gb::GenLevel) * t.level.size());
  std::memcpy(img.data() + lay.at.entry, t.entry.data(), sizeof(gb::GenEntry) * t.entry.size());
  if (g->domain_count) std::memcpy(img.data() + lay.at.doms, g->domains, sizeof(gagp_domain) * g->domain_count);
  if (g->value_count) std::memcpy(img.data() + lay.at.vals, g->values, sizeof(gagp_value) * g->value_count);
  auto* minimum = reinterpret_cast<uint16_t*>(img.data() + lay.at.minimum);
  const size_t cells = size_t(E) * g->depth_count * g->logical_depth_count;
  for (size_t i = 0; i < cells; ++i) {
    const uint32_t v = g->minimum[i];
    minimum[i] = v >= gb::kNoMinimum16 ? gb::kNoMinimum16 : uint16_t(v);
  }
  return img;
}

// Instructions (and constants) the lowering can emit for a row of at most
// `maxv` nodes, the appended RETURN included: a leaf or operation emits 1, a
// value if 2 (its jumps), and/or 5, and a traversal at most 36 of its own
// beside its four children, so at most 8 per node of a row holding
// traversals (36 + 4 children over 5 nodes).  A for_range emits 23 of its
// own; its body's root is a block node that emits none and is no other
// loop's body root, so at most 12 per node of a row holding loops.  A
// bounded region emits its BOUNDED_REGION and at most 13 record
// instructions beside at least five children: at most 3 per node.
// Program, block and nil nodes emit nothing, an if_stmt 2 and an assign,
// a return or a local read 1.
int bytecode_bound(const gagp_grammar* g, int maxv) {
  int per_node = 1;
  for (int i = 0; i < g->expression_count; ++i) {
    const int nk = g->expressions[i].node_kind;
    if (g->expressions[i].kind == gb::EK_OPERATION)
      per_node = std::max(per_node, nk == gb::TK_FOR_RANGE ? 12 : nk == gb::TK_TRAVERSE ? 8 : nk == gb::TK_REGION ? 3
                                    : nk == gb::TK_IF ? 2
                                    : (nk == gb::TK_AND || nk == gb::TK_OR) ? 5 : 1);
  }
  return per_node * maxv + 2;
}

// Whether a grammar's programs mostly need the exact VM: it holds
// traversals or bound reads, or operations that can raise a runtime error
// (modulo and division by zero, list builtins).
// Whether every instruction a program of `g` can emit costs one unit of
// fuel: the accumulator VM's timeout proof counts instructions.
bool unit_fuel(const gagp_grammar* g) {
  if (g->return_fuel != 1) return false;
  for (int r = 0; r < g->region_count; ++r)
    if (g->regions[r].fuel_profile) return false;
  for (int i = 0; i < g->expression_count; ++i)
    if (g->expressions[i].fuel != 1 || g->expressions[i].merge_fuel != 1) return false;
  return true;
}

bool exact_heavy(const gagp_grammar* g) {
  if (gb::is_statement_tag(g->slot_type)) return true;  // statement programs run on the exact VM only
  if (!unit_fuel(g)) return true;                       // so do programs with fuel charges other than 1
  for (int i = 0; i < g->expression_count; ++i) {
    const gagp_expression& e = g->expressions[i];
    if (e.kind == gb::EK_BOUND) return true;
    if (e.kind != gb::EK_OPERATION) continue;
    if (e.node_kind == gb::TK_TRAVERSE) return true;
    if (e.node_kind == gb::TK_OPERATION &&
        gb::accumulator_op_of(e.node_kind, e.opcode, e.operand) == gb::A_COUNT)
      return true;
  }
  return false;
}

// Device copy of the traversal table.
std::vector<gb::RegionInfo> region_infos(const gagp_grammar* g) {
  std::vector<gb::RegionInfo> out(std::max(1, g->region_count));
  for (int r = 0; r < g->region_count; ++r) out[r] = gb::region_info_of(g->regions[r]);
  return out;
}

struct Plan {
  Layout L;
  size_t ex, info, prods, nts, doms, vals, minimum, prod_minimum, gen_image, gen_image_bytes, local_types, regions,
      inputs, expected, lists;
  size_t node, cval, len, cnode, ccval, clen;
  size_t fitness, wrong, nodes, key, c_parent, c_reuse, c_error, c_fitness, c_wrong, c_nodes, c_key, c_eval;
  size_t mtab;
  int mtab_slots = 0;
  size_t code, code_len, kpool, code_temps, vm_acc, bc, bc_len, bc_locals, bc_consts;
  size_t mt, stream, stream_mod, stream_head, round_seed, best, elites, placed, place_state, child_level, level_plan,
      round,
      hist_sum, hist_fitness,
      hist_wrong,
      hist_nodes, hist_node, hist_cval, hist_len, counters;
  int stride, code_stride, bc_stride, stream_capacity, slots;
};

// Children per round: the steady-state batch, or the whole population under
// the generational schedule.
int children_per_round(const gagp_search_config* cfg) {
  if (!cfg->steady_state) return cfg->population;
  return cfg->batch > 0 ? cfg->batch : cfg->population;
}

Plan plan_search(const gagp_grammar* g, const gagp_cases* c, const gagp_search_config* cfg) {
  Plan p{};
  const int P = cfg->population, B = children_per_round(cfg), C = c->case_count;
  const int maxv = g->max_nodes - g->fixed_nodes;
  p.stride = int(align_up(size_t(maxv), 4));
  p.code_stride = 2 * maxv + 8;
  p.bc_stride = bytecode_bound(g, maxv);
  p.slots = std::max(P, B);
  const long long draws = (long long)B * cfg->replacement_size + 1;
  p.stream_capacity = int(((draws + 311) / 312 + 2) * 312);
  const int E = g->expression_count;
  auto& L = p.L;
  p.ex = L.take(sizeof(gagp_expression) * E);
  p.info = L.take(sizeof(gb::ExprInfo) * E);
  p.prods = L.take(sizeof(gagp_production) * std::max(1, g->production_count));
  p.nts = L.take(sizeof(gagp_nonterminal) * std::max(1, g->nonterminal_count));
  p.doms = L.take(sizeof(gagp_domain) * std::max(1, g->domain_count));
  p.vals = L.take(sizeof(gagp_value) * std::max(1, g->value_count));
  p.minimum = L.take(sizeof(uint32_t) * size_t(E) * g->depth_count * g->logical_depth_count);
  p.prod_minimum = L.take(sizeof(uint32_t) * size_t(std::max(1, g->production_count)) * g->depth_count *
                          g->logical_depth_count);
  {
    const DrawTables shape = draw_tables(g, false);
    p.gen_image_bytes = gen_image_layout(g, shape).bytes;
    p.gen_image = L.take(p.gen_image_bytes);
  }
  p.local_types = L.take(sizeof(int32_t) * GAGP_MAX_LOCALS);
  p.regions = L.take(sizeof(gb::RegionInfo) * size_t(std::max(1, g->region_count)));
  p.inputs = L.take(sizeof(int64_t) * size_t(std::max(1, c->input_count)) * C);
  p.expected = L.take(sizeof(int64_t) * C);
  p.lists = L.take(sizeof(int64_t) * size_t(std::max<int64_t>(1, c->list_values ? c->list_value_count : 0)));
  const size_t S = size_t(p.stride);
  p.node = L.take(8 * S * P); p.cval = L.take(8 * S * P); p.len = L.take(4 * size_t(P));
  p.cnode = L.take(8 * S * B); p.ccval = L.take(8 * S * B); p.clen = L.take(4 * size_t(B));
  p.fitness = L.take(8 * size_t(P)); p.wrong = L.take(4 * size_t(P)); p.nodes = L.take(4 * size_t(P));
  p.key = L.take(8 * size_t(P));
  p.c_parent = L.take(4 * size_t(B)); p.c_reuse = L.take(4 * size_t(B)); p.c_error = L.take(4 * size_t(B));
  p.c_fitness = L.take(8 * size_t(B)); p.c_wrong = L.take(4 * size_t(B)); p.c_nodes = L.take(4 * size_t(B));
  p.c_key = L.take(8 * size_t(B)); p.c_eval = L.take(4 * size_t(B));
  p.mtab_slots = 2;
  while (p.mtab_slots < 2 * P) p.mtab_slots *= 2;
  p.mtab = L.take(8 * size_t(p.mtab_slots));
  const size_t slots = size_t(p.slots);
  p.code = L.take(8 * slots * p.code_stride); p.code_len = L.take(4 * slots);
  p.kpool = L.take(8 * slots * S); p.code_temps = L.take(4 * slots); p.vm_acc = L.take(16 * slots);
  p.bc = L.take(20 * slots * p.bc_stride); p.bc_len = L.take(4 * slots); p.bc_locals = L.take(4 * slots);
  p.bc_consts = L.take(8 * slots * p.bc_stride);
  p.mt = L.take(8 * 312); p.stream = L.take(8 * size_t(p.stream_capacity));
  p.stream_mod = L.take(4 * size_t(p.stream_capacity)); p.stream_head = L.take(16);
  p.round_seed = L.take(8); p.best = L.take(4); p.placed = L.take(4 * size_t(P)); p.round = L.take(16);
  p.elites = L.take(4 * size_t(gb::kMaxElites));
  p.place_state = L.take(4);
  p.child_level = L.take(2 * size_t(B)); p.level_plan = L.take(8);
  const size_t H = size_t(cfg->generations);
  p.hist_sum = L.take(8 * H); p.hist_fitness = L.take(8 * H); p.hist_wrong = L.take(4 * H);
  p.hist_nodes = L.take(4 * H); p.hist_node = L.take(8 * S * H); p.hist_cval = L.take(8 * S * H);
  p.hist_len = L.take(4 * H); p.counters = L.take(8 * GAGP_COUNTERS);
  return p;
}

template <class T>
T* at(char* block, size_t off) { return reinterpret_cast<T*>(block + off); }

// The member rows of an imported initial population (`gagp run --init`,
// run.cpp:146-174, imported by import_native_phase_layout): each row's node
// words from its construction expressions, annotated as annotate_phase_tree
// (device/phase_variation.cuh:23-79) annotates a tree -- a node a reference
// expands is a variation site of that reference (its entry and crossover
// class), depth counts tree levels from the root (1) and the site depth the
// sites on the path from the root, the node's own included (0 without a site
// depth limit).  False when a row does not derive from the slot's root, does
// not fit the node budget or exceeds the site depth limit.
bool import_rows(const gagp_grammar* g, const std::vector<gb::ExprInfo>& info, const gagp_rows* rows, int P, int stride,
                 std::vector<uint64_t>* node, std::vector<int64_t>* cval, std::vector<int32_t>* len,
                 std::string* why) {
  const int E = g->expression_count, maxv = g->max_nodes - g->fixed_nodes;
  const bool site_limited = g->site_depth > 0;
  node->assign(size_t(stride) * P, 0);
  cval->assign(size_t(stride) * P, 0);
  len->assign(P, 0);
  struct Task { int expr, entry, depth, sites; uint32_t cls; };
  std::vector<Task> pending;
  for (int r = 0; r < P; ++r) {
    const int n = rows->node_counts[r], nc = rows->constant_counts[r];
    if (n < 1 || n > maxv || n > rows->stride || nc < 0 || nc > n) {
      *why = "row " + std::to_string(r) + " outside the node budget";
      return false;
    }
    const int32_t* origins = rows->origins + size_t(r) * rows->stride;
    pending.assign(1, Task{g->root_expression, -1, 1, 0, gb::kNoClass});
    int cursor = 0, constants = 0, steps = 0;
    while (!pending.empty()) {
      const Task t = pending.back();
      pending.pop_back();
      if (++steps > 8192 || t.expr < 0 || t.expr >= E) break;
      const gagp_expression& e = g->expressions[t.expr];
      if (e.kind == gb::EK_REFERENCE) {
        // one site per node; the node's origin names the production
        if (t.entry >= 0 || cursor >= n || e.target < 0 || e.target >= g->nonterminal_count) break;
        const gagp_nonterminal& nt = g->nonterminals[e.target];
        int production = -1;
        for (int i = 0; i < nt.production_count && production < 0; ++i)
          if (g->productions[nt.production_offset + i].expression == origins[cursor])
            production = origins[cursor];
        if (production < 0) break;
        pending.push_back(Task{production, t.expr, t.depth, t.sites + (site_limited ? 1 : 0),
                               uint32_t(info[t.expr].site_class)});
        continue;
      }
      if (cursor >= n || origins[cursor] != t.expr || t.depth > 255 || t.sites > 255) {
        cursor = -1;
        break;
      }
      if (site_limited && t.sites > g->site_depth) {
        *why = "row " + std::to_string(r) + " exceeds the site depth limit";
        return false;
      }
      const bool constant = e.kind == gb::EK_CONSTANT;
      constants += constant;
      (*node)[size_t(r) * stride + cursor++] =
          gb::w_make(t.expr, t.entry, t.depth, t.sites, info[t.expr].arity, constant, t.cls);
      for (int i = info[t.expr].arity - 1; i >= 0; --i)
        pending.push_back(Task{e.children[i], -1, t.depth + 1, t.sites, gb::kNoClass});
    }
    if (cursor != n || !pending.empty() || constants != nc) {
      *why = "row " + std::to_string(r) + " does not derive from the grammar's root";
      return false;
    }
    // a statement program reads only definitely assigned grammar locals
    // (the native verifier's definite assignment, ast_type_verify)
    if (gb::is_statement_tag(g->slot_type) && !gb::locals_defined(n, [&](int i) {
          const gagp_expression& x = g->expressions[origins[i]];
          return gb::StatementNode{x.kind == gb::EK_OPERATION ? x.node_kind : -1, x.operand,
                                   info[origins[i]].arity, x.type};
        })) {
      *why = "row " + std::to_string(r) + " reads a grammar local before assigning it";
      return false;
    }
    for (int k = 0; k < nc; ++k) (*cval)[size_t(r) * stride + k] = rows->constants[size_t(r) * rows->stride + k];
    (*len)[r] = gb::make_len(n, nc);
  }
  return true;
}

// Whether two productions of one nonterminal may derive the same program:
// their root expressions emit the same node (operations of one opcode and
// shape, constants with overlapping domains, the same input or binder).
// Only then can a program have two derivations.
bool same_root_possible(const gagp_grammar* g, const gagp_expression& x, const gagp_expression& y) {
  if (x.kind != y.kind) return false;
  switch (x.kind) {
    case gb::EK_INPUT: case gb::EK_BOUND: return x.operand == y.operand;
    case gb::EK_CONSTANT: {
      const gagp_domain& a = g->domains[x.target];
      const gagp_domain& b = g->domains[y.target];
      auto has = [&](const gagp_domain& d, int64_t v) {
        if (d.integer_range) return d.minimum <= v && v <= d.maximum;
        for (int k = 0; k < d.value_count; ++k)
          if (g->values[d.value_offset + k].i == v) return true;
        return false;
      };
      if (a.integer_range && b.integer_range) return std::max(a.minimum, b.minimum) <= std::min(a.maximum, b.maximum);
      const gagp_domain& list = a.integer_range ? b : a;
      const gagp_domain& other = a.integer_range ? a : b;
      for (int k = 0; k < list.value_count; ++k)
        if (has(other, g->values[list.value_offset + k].i)) return true;
      return false;
    }
    case gb::EK_OPERATION:
      return x.node_kind == y.node_kind && x.opcode == y.opcode && x.arity == y.arity && x.type == y.type &&
             (x.operand == y.operand || x.node_kind == gb::TK_REGION || x.node_kind == gb::TK_LET ||
              x.node_kind == gb::TK_TRAVERSE);
    default: return true;
  }
}
bool possibly_ambiguous(const gagp_grammar* g) {
  for (int t = 0; t < g->nonterminal_count; ++t) {
    const gagp_nonterminal& nt = g->nonterminals[t];
    for (int a = 0; a < nt.production_count; ++a)
      for (int b = a + 1; b < nt.production_count; ++b)
        if (same_root_possible(g, g->expressions[g->productions[nt.production_offset + a].expression],
                               g->expressions[g->productions[nt.production_offset + b].expression]))
          return true;
  }
  return false;
}

// The derivation the reference's import gives a generated program
// (reconstruct_derivation, cpp/src/evolution/grammar/membership.cpp:330-360):
// at every nonterminal the first production, in production order, whose
// expression matches the whole subtree.  `origins` and `value` (a constant
// node's value) describe the program's nodes; out[i] receives node i's
// expression.  Returns the subtree's end, or -1 (also past `budget` steps).
int first_match(const gagp_grammar* g, int e, const int32_t* origins, const int64_t* value, int n, int i,
                int32_t* out, long* budget) {
  if (--*budget < 0 || i < 0) return -1;
  const gagp_expression& x = g->expressions[e];
  if (x.kind == gb::EK_REFERENCE) {
    const gagp_nonterminal& nt = g->nonterminals[x.target];
    for (int k = 0; k < nt.production_count; ++k) {
      const int end = first_match(g, g->productions[nt.production_offset + k].expression, origins, value, n, i, out,
                                  budget);
      if (end >= 0) return end;
    }
    return -1;
  }
  if (i >= n) return -1;
  const gagp_expression& y = g->expressions[origins[i]];
  if (x.kind != y.kind) return -1;
  if (x.kind == gb::EK_CONSTANT) {
    const gagp_domain& d = g->domains[x.target];
    bool in = d.integer_range && d.minimum <= value[i] && value[i] <= d.maximum;
    for (int k = 0; !d.integer_range && k < d.value_count && !in; ++k) in = g->values[d.value_offset + k].i == value[i];
    if (!in) return -1;
  } else if (x.kind == gb::EK_OPERATION) {
    if (x.node_kind != y.node_kind || x.opcode != y.opcode || x.operand != y.operand || x.arity != y.arity ||
        x.type != y.type)
      return -1;
  } else if (x.operand != y.operand) {
    return -1;
  }
  out[i] = e;
  int j = i + 1;
  for (int k = 0; k < (x.kind == gb::EK_OPERATION ? x.arity : 0); ++k) {
    j = first_match(g, x.children[k], origins, value, n, j, out, budget);
    if (j < 0) return -1;
  }
  return j;
}

// The device's initial population of a search whose grammar may be
// ambiguous, re-derived as the reference's import re-derives its generated
// programs: generated on the device (k_init_population), then each row's
// first-match derivation annotated on the host (import_rows) and uploaded
// as an imported population.
gagp_status canonical_initial(gagp_engine* e, Search* s, const gagp_grammar* g, const std::vector<gb::ExprInfo>& info,
                              gb::SearchDesc* d) {
  const int P = s->P, S = s->stride;
  gb::k_init_population<<<(P + 127) / 128, 128, 0, e->stream>>>(s->d_desc, s->d_off, 1);
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  std::vector<uint64_t> node(size_t(P) * S);
  std::vector<int64_t> cval(size_t(P) * S);
  std::vector<int32_t> len(P);
  CUDA_TRY(copy_d2h(e, node.data(), d->node, 8 * node.size()));
  CUDA_TRY(copy_d2h(e, cval.data(), d->cval, 8 * cval.size()));
  CUDA_TRY(copy_d2h(e, len.data(), d->len, 4 * len.size()));
  std::vector<int32_t> origins(size_t(P) * S), counts(P), ccounts(P);
  std::vector<int64_t> value(S);
  for (int r = 0; r < P; ++r) {
    const int n = gb::len_nodes(len[r]), nc = gb::len_consts(len[r]);
    if (n < 1 || n > S) return fail(GAGP_DEVICE_ERROR, "initial population row length");
    int32_t* o = origins.data() + size_t(r) * S;
    for (int i = 0, k = 0; i < n; ++i) {
      const uint64_t w = node[size_t(r) * S + i];
      o[i] = gb::w_origin(w);
      value[i] = gb::w_const(w) && k < nc ? cval[size_t(r) * S + k++] : 0;
    }
    std::vector<int32_t> canon(o, o + n);
    long budget = 1 << 20;
    if (first_match(g, g->root_expression, o, value.data(), n, 0, canon.data(), &budget) == n)
      std::copy(canon.begin(), canon.end(), o);
    counts[r] = n;
    ccounts[r] = nc;
  }
  // the rows' constants are read while the annotated rows are written: separate buffers
  const std::vector<int64_t> constants(cval);
  gagp_rows rows{P, S, counts.data(), origins.data(), ccounts.data(), const_cast<int64_t*>(constants.data())};
  std::string why;
  if (!import_rows(g, info, &rows, P, S, &node, &cval, &len, &why))
    return fail(GAGP_DEVICE_ERROR, "re-derived initial population: " + why);
  CUDA_TRY(cudaMemcpyAsync(d->node, node.data(), 8 * node.size(), cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(cudaMemcpyAsync(d->cval, cval.data(), 8 * cval.size(), cudaMemcpyHostToDevice, e->stream));
  CUDA_TRY(cudaMemcpyAsync(d->len, len.data(), 4 * len.size(), cudaMemcpyHostToDevice, e->stream));
  d->imported = 1;
  CUDA_TRY(copy_h2d(e, s->d_desc, d, sizeof(gb::SearchDesc)));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  return GAGP_OK;
}

}  // namespace

// ======================================================================= C ABI
extern "C" {

const char* gagp_b200_last_error(void) { return g_error.c_str(); }
const char* gagp_b200_version(void) { return "gagp_b200 1.0 (sm_100a)"; }

gagp_status gagp_b200_engine_create(int32_t device, uint64_t arena_bytes, gagp_engine** out) {
  if (!out) return fail(GAGP_INVALID_ARGUMENT, "null engine pointer");
  *out = nullptr;
  // a round runs on 11 streams (the engine stream, 8 variation ranges and 2
  // side streams); with the default 8 hardware work queues some of them
  // would share a queue and wait on each other's kernels.  The setting only
  // takes effect when this call creates the process's CUDA context.
  setenv("CUDA_DEVICE_MAX_CONNECTIONS", "32", 0);
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return fail(GAGP_DEVICE_ERROR, "no CUDA device");
  if (device < 0 || device >= count) return fail(GAGP_INVALID_ARGUMENT, "device index");
  CUDA_TRY(cudaSetDevice(device));
  auto e = std::make_unique<gagp_engine>();
  e->device = device;
  // the variation ranges take the SMs first and the member index and
  // history entry (needed by the lowering and the placement) fill what is
  // left; the run generator and the placement levels, a chain of few blocks
  // that the placement waits for, go first
  int least = 0, greatest = 0;
  CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
  CUDA_TRY(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
  CUDA_TRY(cudaStreamCreateWithPriority(&e->side, cudaStreamNonBlocking, least));
  CUDA_TRY(cudaStreamCreateWithPriority(&e->draws, cudaStreamNonBlocking, greatest));
  CUDA_TRY(cudaEventCreateWithFlags(&e->drawn, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&e->join, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&e->indexed, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&e->chunk_fork, cudaEventDisableTiming));
  for (int c = 0; c < gagp_engine::kChunks; ++c) {
    CUDA_TRY(cudaStreamCreateWithPriority(&e->chunk_stream[c], cudaStreamNonBlocking, greatest));
    CUDA_TRY(cudaEventCreateWithFlags(&e->chunk_done[c], cudaEventDisableTiming));
  }
  cudaDeviceProp prop;
  CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  e->sm_count = prop.multiProcessorCount;
  e->max_smem = prop.sharedMemPerBlockOptin;
  size_t free_bytes = 0, total = 0;
  CUDA_TRY(cudaMemGetInfo(&free_bytes, &total));
  e->arena_limit = arena_bytes ? arena_bytes : uint64_t(0.8 * double(free_bytes));
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  CUDA_TRY(cudaMemPoolCreate(&e->pool, &props));
  uint64_t keep = ~0ULL;  // freed blocks stay in the pool for the next admission
  CUDA_TRY(cudaMemPoolSetAttribute(e->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  CUDA_TRY(cudaFuncSetAttribute(gb::k_place, cudaFuncAttributeMaxDynamicSharedMemorySize, int(e->max_smem) - 16384));
  CUDA_TRY(cudaFuncSetAttribute(gb::k_vm_fast<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(e->max_smem) - 1024));
  CUDA_TRY(cudaFuncSetAttribute(gb::k_vm_fast<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(e->max_smem) - 1024));
  CUDA_TRY(cudaFuncSetAttribute(gb::k_vm_fast<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(e->max_smem) - 1024));
  CUDA_TRY(cudaFuncSetAttribute(gb::k_vary, cudaFuncAttributeMaxDynamicSharedMemorySize, int(e->max_smem) - 1024));
  CUDA_TRY(cudaFuncSetAttribute(gb::k_vm_general, cudaFuncAttributeMaxDynamicSharedMemorySize, int(e->max_smem) - 1024));
  *out = e.release();
  return GAGP_OK;
}

void gagp_b200_engine_destroy(gagp_engine* e) {
  if (!e) return;
  cudaSetDevice(e->device);
  cudaStreamSynchronize(e->stream);
  for (auto& kv : e->searches) {
    cudaFreeAsync(kv.second->block, e->stream);
    cudaFreeAsync(kv.second->d_desc, e->stream);
    cudaFreeAsync(kv.second->d_off, e->stream);
  }
  cudaStreamSynchronize(e->stream);
  if (e->pool) cudaMemPoolDestroy(e->pool);
  if (e->pinned) cudaFreeHost(e->pinned);
  cudaFree(e->d_fast);
  cudaFree(e->d_general);
  cudaFree(e->d_region);
  cudaFree(e->region_ws);
  cudaFree(e->d_counts);
  cudaFree(e->d_batch_desc);
  cudaFree(e->d_batch_off);
  cudaFree(e->flush_buffer);
  for (cudaEvent_t ev : e->event_pool) cudaEventDestroy(ev);
  cudaStreamDestroy(e->stream);
  if (e->side) cudaStreamDestroy(e->side);
  if (e->draws) cudaStreamDestroy(e->draws);
  if (e->drawn) cudaEventDestroy(e->drawn);
  if (e->fork) cudaEventDestroy(e->fork);
  if (e->join) cudaEventDestroy(e->join);
  if (e->indexed) cudaEventDestroy(e->indexed);
  if (e->chunk_fork) cudaEventDestroy(e->chunk_fork);
  for (int c = 0; c < gagp_engine::kChunks; ++c) {
    if (e->chunk_stream[c]) cudaStreamDestroy(e->chunk_stream[c]);
    if (e->chunk_done[c]) cudaEventDestroy(e->chunk_done[c]);
  }
  delete e;
}

gagp_status gagp_b200_search_bytes(const gagp_grammar* g, const gagp_cases* c, const gagp_search_config* cfg,
                                   uint64_t* out_bytes) {
  const gagp_status st = admit(g, c, cfg);
  if (st != GAGP_OK) return st;
  *out_bytes = plan_search(g, c, cfg).L.total;
  return GAGP_OK;
}

gagp_status gagp_b200_search_create(gagp_engine* e, const gagp_grammar* g, const gagp_cases* c,
                                    const gagp_search_config* cfg, const gagp_rows* initial, int32_t* out_search) {
  if (!e || !out_search) return fail(GAGP_INVALID_ARGUMENT, "null argument");
  if (e->poisoned) return fail(GAGP_DEVICE_ERROR, "engine is poisoned by an earlier device error");
  const gagp_status st = admit(g, c, cfg);
  if (st != GAGP_OK) return st;
  if (initial && (initial->count < cfg->population || initial->stride < 1 || !initial->node_counts ||
                  !initial->origins || !initial->constant_counts || (!initial->constants && initial->count)))
    return fail(GAGP_INVALID_ARGUMENT, "an imported population needs population rows");
  CUDA_TRY(cudaSetDevice(e->device));
  Plan p = plan_search(g, c, cfg);
  if (e->arena_used + p.L.total > e->arena_limit)
    return fail(GAGP_OUT_OF_MEMORY, "search does not fit the engine's device-memory budget");
  auto s = std::make_unique<Search>();
  s->P = cfg->population;
  s->B = children_per_round(cfg);
  s->G = cfg->generations;
  s->total_rounds = int((long long)s->P * s->G / s->B);
  s->maxv = g->max_nodes - g->fixed_nodes;
  s->stride = p.stride;
  s->fixed_nodes = g->fixed_nodes;
  s->has_wrong = cfg->metric != GAGP_METRIC_LEGACY;
  s->exact_heavy = exact_heavy(g);
  s->region_words = 0;
  for (int r = 0; r < g->region_count; ++r)
    if (g->regions[r].traversal == 0)
      s->region_words = std::max(s->region_words, gb::region_lane_words(gb::region_info_of(g->regions[r])));
  if (s->region_words)
    if (const gagp_status st = ensure_region_workspace(e, s->region_words); st != GAGP_OK) return st;
  s->bytes = p.L.total;
  CUDA_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&s->block), s->bytes, e->pool, e->stream));
  CUDA_TRY(cudaMemsetAsync(s->block, 0, s->bytes, e->stream));
  char* b = s->block;
  const int E = g->expression_count;
  // derived per-expression facts
  std::vector<gb::ExprInfo> info(E);
  for (int i = 0; i < E; ++i) {
    const gagp_expression& x = g->expressions[i];
    gb::ExprInfo& f = info[i];
    f.kind = int8_t(x.kind);
    f.node_kind = int8_t(x.node_kind);
    f.arity = int8_t(x.kind == gb::EK_REFERENCE ? 0 : x.arity);
    f.type = int8_t(x.type);
    f.opcode = int16_t(x.opcode);
    f.operand = x.operand;
    f.target = x.target;
    f.site_nt = x.kind == gb::EK_REFERENCE ? x.target : -1;
    f.site_class = -1;
    if (x.kind == gb::EK_REFERENCE && x.target >= 0 && x.target < g->nonterminal_count &&
        !g->nonterminals[x.target].fixed)
      f.site_class = x.target * 16 + x.scope_count;
  }
  // cases, input-major.  With IntList inputs the cases are ordered by their
  // lists' total length, so that the 32 cases of a VM warp loop about as
  // many times (a program's loss and wrong count are integer sums, which
  // the case order does not change)
  const int C = c->case_count, NI = c->input_count;
  std::vector<int> order(C);
  std::iota(order.begin(), order.end(), 0);
  if (c->list_values) {
    std::vector<int64_t> length(C, 0);
    for (int k = 0; k < C; ++k)
      for (int j = 0; j < NI; ++j)
        if (c->input_tags[j] == GAGP_TAG_INTLIST) length[k] += c->list_values[c->inputs[size_t(k) * NI + j]];
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return length[x] < length[y]; });
  }
  std::vector<int64_t> inputs(size_t(std::max(1, NI)) * C, 0), expected(C);
  for (int k = 0; k < C; ++k) {
    for (int j = 0; j < NI; ++j) inputs[size_t(j) * C + k] = c->inputs[size_t(order[k]) * NI + j];
    expected[k] = c->expected[order[k]];
  }
  std::vector<int32_t> local_types(GAGP_MAX_LOCALS, GAGP_TAG_INVALID);
  for (int j = 0; j < g->local_count; ++j) local_types[j] = g->local_types[j];
  auto up = [&](size_t off, const void* src, size_t bytes) {
    return copy_h2d(e, b + off, src, bytes);
  };
  CUDA_TRY(up(p.ex, g->expressions, sizeof(gagp_expression) * E));
  CUDA_TRY(up(p.info, info.data(), sizeof(gb::ExprInfo) * E));
  if (g->production_count) CUDA_TRY(up(p.prods, g->productions, sizeof(gagp_production) * g->production_count));
  if (g->nonterminal_count) CUDA_TRY(up(p.nts, g->nonterminals, sizeof(gagp_nonterminal) * g->nonterminal_count));
  if (g->domain_count) CUDA_TRY(up(p.doms, g->domains, sizeof(gagp_domain) * g->domain_count));
  if (g->value_count) CUDA_TRY(up(p.vals, g->values, sizeof(gagp_value) * g->value_count));
  CUDA_TRY(up(p.minimum, g->minimum, sizeof(uint32_t) * size_t(E) * g->depth_count * g->logical_depth_count));
  // production-major copy of the minimum table: a nonterminal's productions
  // are adjacent for each (depth, site budget)
  const int PR = g->production_count, DC = g->depth_count, LC = g->logical_depth_count;
  std::vector<uint32_t> prod_minimum(size_t(std::max(1, PR)) * DC * LC, gb::kNoId);
  for (int d = 0; d < DC; ++d)
    for (int l = 0; l < LC; ++l)
      for (int q = 0; q < PR; ++q) {
        const int pe = g->productions[q].expression;
        if (pe >= 0 && pe < E) prod_minimum[(size_t(d) * LC + l) * PR + q] = g->minimum[(size_t(pe) * DC + d) * LC + l];
      }
  CUDA_TRY(up(p.prod_minimum, prod_minimum.data(), sizeof(uint32_t) * prod_minimum.size()));
  const DrawTables draw = draw_tables(g, true);
  const GenImageLayout lay = gen_image_layout(g, draw);
  if (lay.bytes != p.gen_image_bytes) return fail(GAGP_DEVICE_ERROR, "generator table plan mismatch");
  const std::vector<char> image = gen_image(g, info, draw, lay);
  CUDA_TRY(up(p.gen_image, image.data(), image.size()));
  CUDA_TRY(up(p.local_types, local_types.data(), sizeof(int32_t) * GAGP_MAX_LOCALS));
  const std::vector<gb::RegionInfo> regions = region_infos(g);
  CUDA_TRY(up(p.regions, regions.data(), sizeof(gb::RegionInfo) * regions.size()));
  CUDA_TRY(up(p.inputs, inputs.data(), sizeof(int64_t) * inputs.size()));
  CUDA_TRY(up(p.expected, expected.data(), sizeof(int64_t) * C));
  const int64_t n_lists = c->list_values ? c->list_value_count : 0;
  if (n_lists) CUDA_TRY(up(p.lists, c->list_values, sizeof(int64_t) * size_t(n_lists)));

  gb::SearchDesc& d = s->desc;
  d.ex = at<gagp_expression>(b, p.ex);
  d.info = at<gb::ExprInfo>(b, p.info);
  d.prods = at<gagp_production>(b, p.prods);
  d.nts = at<gagp_nonterminal>(b, p.nts);
  d.doms = at<gagp_domain>(b, p.doms);
  d.vals = at<gagp_value>(b, p.vals);
  d.minimum = at<uint32_t>(b, p.minimum);
  d.prod_minimum = at<uint32_t>(b, p.prod_minimum);
  d.gen_image = at<char>(b, p.gen_image);
  d.gen_image_bytes = int32_t(lay.bytes);
  d.gi = lay.at;
  d.local_types = at<int32_t>(b, p.local_types);
  d.regions = at<gb::RegionInfo>(b, p.regions);
  d.n_regions = g->region_count;
  d.n_ex = E; d.n_prods = g->production_count; d.n_nts = g->nonterminal_count;
  d.n_doms = g->domain_count; d.n_vals = g->value_count;
  d.depth_count = g->depth_count; d.logical_count = g->logical_depth_count; d.site_depth = g->site_depth;
  d.root_expression = g->root_expression; d.slot_max_depth = g->slot_max_depth; d.slot_type = g->slot_type;
  d.result_type = result_type_of(g);
  d.unit_fuel = unit_fuel(g) ? 1 : 0;
  d.local_count = g->local_count; d.max_nodes = g->max_nodes; d.fixed_nodes = g->fixed_nodes;
  d.return_fuel = g->return_fuel;
  d.P = s->P; d.B = s->B; d.maxv = s->maxv; d.stride = p.stride;
  d.pressure = std::clamp(cfg->tournament_size, 1, s->P);
  d.attempts = cfg->crossover_attempts; d.mutation_max_nodes = cfg->mutation_max_nodes;
  d.counted = cfg->counted_sites; d.uniform_phase = cfg->uniform_phase; d.replacement_size = cfg->replacement_size;
  d.has_wrong = s->has_wrong; d.grammar_sites = cfg->grammar_site_ranking;
  d.metric = cfg->metric; d.fuel = cfg->fuel;
  d.crossover_probability = cfg->crossover_probability; d.mutation_probability = cfg->mutation_probability;
  d.penalty = cfg->penalty; d.penalty_int = (int64_t)std::fabs(cfg->penalty);
  d.seed = cfg->seed;
  d.rounds_per_epoch = s->P / s->B;
  d.generational = !cfg->steady_state;
  d.elite_count = cfg->steady_state ? 0 : cfg->elite_count;
  d.generations = s->G;
  d.inputs = at<int64_t>(b, p.inputs); d.expected = at<int64_t>(b, p.expected);
  d.lists = at<int64_t>(b, p.lists); d.n_lists = n_lists;
  d.C = C; d.n_inputs = NI; d.expected_tag = c->expected_tag; d.vm_cases_per_lane = cases_per_lane(C);
  d.node = at<uint64_t>(b, p.node); d.cval = at<int64_t>(b, p.cval); d.len = at<int32_t>(b, p.len);
  d.cnode = at<uint64_t>(b, p.cnode); d.ccval = at<int64_t>(b, p.ccval); d.clen = at<int32_t>(b, p.clen);
  d.fitness = at<double>(b, p.fitness); d.wrong = at<uint32_t>(b, p.wrong); d.nodes = at<uint32_t>(b, p.nodes);
  d.key = at<uint64_t>(b, p.key);
  d.c_parent = at<int32_t>(b, p.c_parent); d.c_reuse = at<int32_t>(b, p.c_reuse); d.c_error = at<int32_t>(b, p.c_error);
  d.c_fitness = at<double>(b, p.c_fitness); d.c_wrong = at<uint32_t>(b, p.c_wrong);
  d.c_nodes = at<uint32_t>(b, p.c_nodes); d.c_key = at<uint64_t>(b, p.c_key); d.c_eval = at<int32_t>(b, p.c_eval);
  d.mtab = at<unsigned long long>(b, p.mtab); d.mtab_mask = p.mtab_slots - 1;
  d.code = at<uint2>(b, p.code); d.code_len = at<int32_t>(b, p.code_len); d.kpool = at<int64_t>(b, p.kpool);
  d.code_stride = p.code_stride; d.code_temps = at<int32_t>(b, p.code_temps);
  d.vm_acc = at<unsigned long long>(b, p.vm_acc);
  d.bc = at<int32_t>(b, p.bc); d.bc_len = at<int32_t>(b, p.bc_len); d.bc_locals = at<int32_t>(b, p.bc_locals);
  d.bc_consts = at<int64_t>(b, p.bc_consts);
  d.bc_stride = p.bc_stride;
  d.mt = at<uint64_t>(b, p.mt); d.stream = at<uint64_t>(b, p.stream); d.stream_mod = at<uint32_t>(b, p.stream_mod);
  d.stream_head = at<long long>(b, p.stream_head); d.stream_capacity = p.stream_capacity;
  d.mod_magic = ~0ULL / uint64_t(s->P);
  d.bounded_threshold = (0 - uint64_t(s->P)) % uint64_t(s->P);
  d.round_seed = at<uint64_t>(b, p.round_seed);
  d.best = at<int32_t>(b, p.best); d.placed = at<int32_t>(b, p.placed); d.round = at<int32_t>(b, p.round);
  d.elites = at<int32_t>(b, p.elites);
  d.place_state = at<int32_t>(b, p.place_state);
  d.child_level = at<int16_t>(b, p.child_level); d.level_plan = at<int32_t>(b, p.level_plan);
  d.hist_sum = at<int64_t>(b, p.hist_sum); d.hist_fitness = at<double>(b, p.hist_fitness);
  d.hist_wrong = at<uint32_t>(b, p.hist_wrong); d.hist_nodes = at<uint32_t>(b, p.hist_nodes);
  d.hist_node = at<uint64_t>(b, p.hist_node); d.hist_cval = at<int64_t>(b, p.hist_cval);
  d.hist_len = at<int32_t>(b, p.hist_len); d.counters = at<uint64_t>(b, p.counters);
  // packed ranking key: loss | wrong | nodes
  const int node_bits = bits_for(uint64_t(g->max_nodes));
  const int wrong_bits = bits_for(uint64_t(C));
  const int loss_bits = bits_for(uint64_t(double(C) * std::fabs(cfg->penalty)));
  if (s->has_wrong && node_bits + wrong_bits + loss_bits > 64) {
    cudaFreeAsync(s->block, e->stream);
    return fail(GAGP_DECLINED, "ranking key wider than 64 bits");
  }
  d.key_shift_nodes = node_bits;
  d.key_shift_wrong = node_bits + wrong_bits;
  d.total_rounds = s->total_rounds;
  if (initial) {
    // the caller's population replaces the generated one (its first
    // population rows, in order)
    std::vector<uint64_t> node;
    std::vector<int64_t> cval;
    std::vector<int32_t> len;
    std::string why;
    if (!import_rows(g, info, initial, s->P, p.stride, &node, &cval, &len, &why)) {
      cudaFreeAsync(s->block, e->stream);
      return fail(GAGP_INVALID_ARGUMENT, "imported population: " + why);
    }
    CUDA_TRY(up(p.node, node.data(), 8 * node.size()));
    CUDA_TRY(up(p.cval, cval.data(), 8 * cval.size()));
    CUDA_TRY(up(p.len, len.data(), 4 * len.size()));
    d.imported = 1;
  }
  CUDA_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&s->d_desc), sizeof(gb::SearchDesc), e->pool, e->stream));
  CUDA_TRY(copy_h2d(e, s->d_desc, &d, sizeof(gb::SearchDesc)));
  const int32_t off[4] = {0, s->P, 0, s->B};
  CUDA_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&s->d_off), sizeof(off), e->pool, e->stream));
  CUDA_TRY(copy_h2d(e, s->d_off, off, sizeof(off)));
  if (!d.imported && possibly_ambiguous(g))
    if (const gagp_status st = canonical_initial(e, s.get(), g, info, &d); st != GAGP_OK) {
      cudaFreeAsync(s->block, e->stream);
      return st;
    }
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  s->id = e->next_id++;
  e->arena_used += s->bytes;
  *out_search = s->id;
  e->searches[s->id] = std::move(s);
  return GAGP_OK;
}

gagp_status gagp_b200_search_destroy(gagp_engine* e, int32_t id) {
  if (!e) return fail(GAGP_INVALID_ARGUMENT, "null engine");
  auto it = e->searches.find(id);
  if (it == e->searches.end()) return fail(GAGP_INVALID_ARGUMENT, "unknown search");
  cudaSetDevice(e->device);
  // stream-ordered: the blocks return to the pool after the work queued on
  // the engine stream (every kernel of the search) has run
  cudaFreeAsync(it->second->block, e->stream);
  cudaFreeAsync(it->second->d_desc, e->stream);
  cudaFreeAsync(it->second->d_off, e->stream);
  e->arena_used -= it->second->bytes;
  e->searches.erase(it);
  return GAGP_OK;
}

}  // extern "C"

// ======================================================================= batches
namespace {

struct BatchView {
  gb::SearchDesc* d_desc = nullptr;
  int32_t* d_member_off = nullptr;   // n + 1
  int32_t* d_child_off = nullptr;    // n + 1
  int n = 0, total_members = 0, total_children = 0, max_P = 0, max_lanes = 1, max_rounds = 0, max_stride = 4;
  long long max_draws = 0;
  int max_code_stride = 2, max_bc_stride = 2;
  int max_C = 1, max_inputs = 0;
  int min_B = 1 << 30;               // the smallest round of the batch
  bool exact_heavy = false;          // some search's programs mostly need the exact VM
  bool regions = false;              // some search's grammar has bounded regions
  bool generational = false;         // the batch's schedule (one per batch)
  std::vector<int> child_off;        // host copy of the child offsets (n + 1)
  std::vector<size_t> image_bytes;   // each search's generator image
};

// Generator images up to this size are staged in the variation kernel's
// shared memory (beside 4 warps' rows, 6 blocks still fit an SM).
constexpr size_t kMaxStagedImage = size_t(12) << 10;

gagp_status make_batch_view(gagp_engine* e, const std::vector<Search*>& list, BatchView* v) {
  const int n = int(list.size());
  v->n = n;
  v->generational = n > 0 && list[0]->desc.generational;
  for (Search* s : list)
    if (bool(s->desc.generational) != v->generational)
      return fail(GAGP_INVALID_ARGUMENT, "a batch holds searches of one schedule (steady-state or generational)");
  if (n == 1) {
    v->d_desc = list[0]->d_desc;
    v->d_member_off = list[0]->d_off;
    v->d_child_off = list[0]->d_off + 2;
  } else {
    // grown geometrically (batches change size while serving); a failed
    // allocation leaves no stale pointer or capacity behind
    if (size_t(n) > e->batch_desc_capacity) {
      const size_t cap = std::max<size_t>(size_t(n), 2 * e->batch_desc_capacity);
      cudaFree(e->d_batch_desc);
      e->d_batch_desc = nullptr;
      e->batch_desc_capacity = 0;
      CUDA_TRY(cudaMalloc(&e->d_batch_desc, sizeof(gb::SearchDesc) * cap));
      e->batch_desc_capacity = cap;
    }
    if (size_t(2 * (n + 1)) > e->batch_off_capacity) {
      const size_t cap = std::max<size_t>(size_t(2 * (n + 1)), 2 * e->batch_off_capacity);
      cudaFree(e->d_batch_off);
      e->d_batch_off = nullptr;
      e->batch_off_capacity = 0;
      CUDA_TRY(cudaMalloc(&e->d_batch_off, sizeof(int32_t) * cap));
      e->batch_off_capacity = cap;
    }
    std::vector<gb::SearchDesc> descs(n);
    std::vector<int32_t> off(2 * (n + 1), 0);
    for (int i = 0; i < n; ++i) {
      descs[i] = list[i]->desc;
      off[i + 1] = off[i] + list[i]->P;
      off[n + 1 + i + 1] = off[n + 1 + i] + list[i]->B;
    }
    CUDA_TRY(copy_h2d(e, e->d_batch_desc, descs.data(), sizeof(gb::SearchDesc) * n));
    CUDA_TRY(copy_h2d(e, e->d_batch_off, off.data(), sizeof(int32_t) * off.size()));
    v->d_desc = e->d_batch_desc;
    v->d_member_off = e->d_batch_off;
    v->d_child_off = e->d_batch_off + n + 1;
  }
  v->total_members = v->total_children = v->max_P = v->max_rounds = 0;
  v->max_stride = 4;
  v->max_draws = 0;
  v->max_code_stride = 2;
  v->max_bc_stride = 2;
  v->max_lanes = 1;
  v->max_C = 1;
  v->max_inputs = 0;
  v->exact_heavy = false;
  v->regions = false;
  v->child_off.assign(1, 0);
  v->image_bytes.clear();
  for (Search* s : list) {
    v->child_off.push_back(v->child_off.back() + s->B);
    v->image_bytes.push_back(size_t(s->desc.gen_image_bytes));
    v->exact_heavy |= s->exact_heavy;
    v->regions |= s->region_words > 0;
    v->max_C = std::max(v->max_C, s->desc.C);
    v->max_inputs = std::max(v->max_inputs, s->desc.n_inputs);
    v->total_members += s->P;
    v->total_children += s->B;
    v->max_P = std::max(v->max_P, s->P);
    v->max_lanes = std::max(v->max_lanes, s->desc.vm_cases_per_lane);
    v->max_rounds = std::max(v->max_rounds, s->total_rounds);
    v->max_stride = std::max(v->max_stride, s->stride);
    v->max_code_stride = std::max(v->max_code_stride, s->desc.code_stride);
    v->max_bc_stride = std::max(v->max_bc_stride, s->desc.bc_stride);
    v->max_draws = std::max(v->max_draws, (long long)s->B * s->desc.replacement_size + 1);
    v->min_B = std::min(v->min_B, s->B);
  }
  return ensure_lists(e, size_t(std::max(v->total_members, v->total_children)));
}

int blocks_for(int items, int threads) { return std::max(1, (items + threads - 1) / threads); }

// Evaluates lowered programs listed by k_lower: counts[0] programs on the
// fast (accumulator) VM, counts[1] on the exact VM.
// Fast-VM launch of one instantiation.
void vm_fast_launch(int lanes, int blocks, int threads, size_t smem, cudaStream_t stream, const gb::SearchDesc* descs,
                    int mode, const gb::ProgramRef* list, const int32_t* counts, int temp_stride, int code_stride,
                    int const_stride, int max_C) {
  const int tiles = (max_C + 32 * lanes - 1) / (32 * lanes);
  switch (lanes) {
    case 1: gb::k_vm_fast<1><<<blocks, threads, smem, stream>>>(descs, mode, list, counts, temp_stride, code_stride, const_stride, tiles); break;
    case 2: gb::k_vm_fast<2><<<blocks, threads, smem, stream>>>(descs, mode, list, counts, temp_stride, code_stride, const_stride, tiles); break;
    default: gb::k_vm_fast<4><<<blocks, threads, smem, stream>>>(descs, mode, list, counts, temp_stride, code_stride, const_stride, tiles); break;
  }
}

// Exact-VM launch over counts[1] programs: persistent blocks of 8 warps,
// each program's bytecode staged in dynamic shared memory with the warp-SIMD
// VM's slots (gb::general_smem_bytes).
constexpr int kGeneralThreads = gb::kGeneralWarps * 32;
size_t vm_general_smem(int bc_stride_max) { return gb::general_smem_bytes(bc_stride_max); }
// `heavy`: most programs may be on the list, so the grid fills every SM;
// otherwise the list is rarely more than a handful of programs and a
// quarter of the SMs take them (an empty launch of a full grid costs a few
// microseconds on every range's critical path).
gagp_status vm_general_launch(int sm_count, cudaStream_t stream, const gb::SearchDesc* descs, int mode,
                              const gb::ProgramRef* list, const int32_t* counts, int bc_stride_max, bool heavy,
                              gb::ProgramRef* deferred, int32_t* deferred_count) {
  const size_t smem = vm_general_smem(bc_stride_max);
  int blocks = std::max(1, sm_count / 4);
  if (heavy) {
    int per_sm = 0;
    const cudaError_t occ = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gb::k_vm_general, kGeneralThreads,
                                                                          smem);
    if (occ != cudaSuccess) return fail(GAGP_DEVICE_ERROR, std::string("exact VM occupancy: ") + cudaGetErrorString(occ));
    blocks = sm_count * std::max(1, per_sm);
  }
  gb::k_vm_general<<<blocks, kGeneralThreads, smem, stream>>>(descs, mode, list, counts + 1, bc_stride_max, deferred,
                                                              deferred_count);
  return GAGP_OK;
}

// The bounded-region workspace for plans of up to `words` int64 words per
// lane (grown, never shrunk; the device is idle between API calls).
gagp_status ensure_region_workspace(gagp_engine* e, size_t words) {
  const int lanes = 2 * e->sm_count * gb::kRegionThreads;
  if (e->region_ws && words <= e->region_ws_words && lanes <= e->region_lanes) return GAGP_OK;
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  if (e->region_ws) cudaFree(e->region_ws);
  e->region_ws = nullptr;
  e->region_ws_words = 0;
  const size_t w = std::max(words, e->region_ws_words);
  if (cudaMalloc(&e->region_ws, w * size_t(lanes) * sizeof(int64_t)) != cudaSuccess) {
    cudaGetLastError();
    return fail(GAGP_OUT_OF_MEMORY, "bounded-region workspace");
  }
  e->region_ws_words = w;
  e->region_lanes = lanes;
  return GAGP_OK;
}

// The deferred programs with bounded regions: a fixed grid of the region
// workspace's lanes, after every exact-VM launch that deferred to it.
gagp_status vm_region_launch(gagp_engine* e, cudaStream_t stream, const gb::SearchDesc* descs, int mode,
                             const gb::ProgramRef* list, const int32_t* count) {
  if (!e->region_ws) return fail(GAGP_DEVICE_ERROR, "bounded regions without a workspace");
  gb::k_vm_region<<<e->region_lanes / gb::kRegionThreads, gb::kRegionThreads, 0, stream>>>(
      descs, mode, list, count, e->region_ws, e->region_ws_words);
  return GAGP_OK;
}


// The VM configuration of one round: the tuned cases per lane, or the next
// candidate to time (measure_key != 0) while the shape is being tuned.
struct VmPlan {
  int lanes = 4;
  uint64_t measure_key = 0;
  int cand = 0;
};
VmPlan plan_vm(gagp_engine* e, const BatchView& v, bool may_measure) {
  VmPlan p;
  const uint64_t key = vm_key(v.max_C, v.max_inputs);
  auto& t = e->vm_tune[key];
  if (t.chosen >= 0) { p.lanes = kVmLanes[t.chosen]; return p; }
  p.lanes = v.max_lanes;  // the heuristic until the candidates are timed
  if (!may_measure || e->profiling) return p;
  const int n = t.rounds[0] + t.rounds[1] + t.rounds[2];
  if (n >= 3 * kTuneRounds) return p;
  const int c = (n / 3) % 2 == 0 ? n % 3 : 2 - n % 3;
  p.lanes = kVmLanes[c];
  p.cand = c;
  p.measure_key = key;
  ++t.rounds[c];
  return p;
}

gagp_status launch_vm_fast(gagp_engine* e, const BatchView& v, int mode, cudaStream_t stream, const gb::ProgramRef* fast,
                           const int32_t* counts, const VmPlan& plan) {
  const int warps = 8;
  const int temp_stride = gb::kMaxTemps * plan.lanes * 32;
  const int code_stride = (v.max_code_stride + 1) & ~1;  // uint2 slots, in int64 units
  const int const_stride = v.max_stride;
  const size_t smem = size_t(warps) * (temp_stride + code_stride + const_stride) * sizeof(int64_t);
  // persistent: as many blocks as fit on every SM at once
  int per_sm = 0;
  const cudaError_t occ = plan.lanes == 1 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gb::k_vm_fast<1>, warps * 32, smem)
                          : plan.lanes == 2 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gb::k_vm_fast<2>, warps * 32, smem)
                                            : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gb::k_vm_fast<4>, warps * 32, smem);
  if (occ != cudaSuccess) return fail(GAGP_DEVICE_ERROR, std::string("VM occupancy: ") + cudaGetErrorString(occ));
  const int blocks = e->sm_count * std::max(1, per_sm);
  cudaEvent_t mark_start = nullptr, mark_stop = nullptr;
  if (plan.measure_key) {
    mark_start = take_event(e);
    mark_stop = take_event(e);
    cudaEventRecord(mark_start, stream);
  }
  {
    Timed t(e, KN_VM_FAST, stream);
    vm_fast_launch(plan.lanes, blocks, warps * 32, smem, stream, v.d_desc, mode, fast, counts, temp_stride,
                   code_stride, const_stride, v.max_C);
  }
  if (plan.measure_key) {
    cudaEventRecord(mark_stop, stream);
    e->tune_marks.push_back({plan.measure_key, plan.cand, mark_start, mark_stop});
    ++e->vm_tune[plan.measure_key].pending;
  }
  return GAGP_OK;
}

// Both VMs over one range's lists: counts[0] fast programs, counts[1] exact.
gagp_status launch_vm(gagp_engine* e, const BatchView& v, int mode, cudaStream_t stream, const gb::ProgramRef* fast,
                      const gb::ProgramRef* general, const int32_t* counts, const VmPlan& plan) {
  if (const gagp_status st = launch_vm_fast(e, v, mode, stream, fast, counts, plan); st != GAGP_OK) return st;
  Timed t(e, KN_VM_GENERAL, stream);
  return vm_general_launch(e->sm_count, stream, v.d_desc, mode, general, counts, v.max_bc_stride, v.exact_heavy,
                           e->d_region, e->d_counts + kRegionCount);
}

gagp_status launch_start(gagp_engine* e, const BatchView& v) {
  { Timed t(e, KN_INIT); gb::k_init_population<<<blocks_for(v.total_members, 128), 128, 0, e->stream>>>(v.d_desc, v.d_member_off, v.n); }
  CUDA_TRY(cudaMemsetAsync(e->d_counts, 0, 2 * sizeof(int32_t), e->stream));
  CUDA_TRY(cudaMemsetAsync(e->d_counts + kRegionCount, 0, sizeof(int32_t), e->stream));
  {
    Timed t(e, KN_LOWER);
    gb::k_lower<<<blocks_for(v.total_members, gb::kLowerWarps), gb::kLowerWarps * 32, 0, e->stream>>>(
        v.d_desc, v.d_member_off, v.n, 0, e->d_fast, e->d_general, e->d_counts, e->d_counts + 1, 0, v.total_members);
  }
  VmPlan start_plan;
  start_plan.lanes = v.max_lanes;
  if (const gagp_status st = launch_vm(e, v, 0, e->stream, e->d_fast, e->d_general, e->d_counts, start_plan);
      st != GAGP_OK)
    return st;
  if (v.regions)
    if (const gagp_status st = vm_region_launch(e, e->stream, v.d_desc, 0, e->d_region, e->d_counts + kRegionCount);
        st != GAGP_OK)
      return st;
  { Timed t(e, KN_KEYS); gb::k_member_keys<<<blocks_for(v.total_members, 128), 128, 0, e->stream>>>(v.d_desc, v.d_member_off, v.n); }
  { Timed t(e, KN_START); gb::k_start<<<v.n, 256, 0, e->stream>>>(v.d_desc, v.n); }
  return cudaPeekAtLastError() == cudaSuccess ? GAGP_OK : fail(GAGP_DEVICE_ERROR, cudaGetErrorString(cudaGetLastError()));
}

gagp_status launch_round(gagp_engine* e, const BatchView& v, bool may_measure = true) {
  const VmPlan vm = plan_vm(e, v, may_measure);
  // the run-generator top-up overlaps everything up to the placement
  CUDA_TRY(cudaEventRecord(e->fork, e->stream));
  CUDA_TRY(cudaStreamWaitEvent(e->side, e->fork, 0));
  // the round's member index (one member per distinct row), built beside
  // the variation: the lowering probes it for the children their parents
  // do not cover, so every range's lowering waits for it
  {
    Timed t(e, KN_INDEX, e->side);
    gb::k_member_index<<<blocks_for(v.total_members, 8), 256, 0, e->side>>>(v.d_desc, v.d_member_off, v.n);
  }
  CUDA_TRY(cudaEventRecord(e->indexed, e->side));
  // the history entry reads only what the placement later rewrites
  { Timed t(e, KN_RECORD, e->side); gb::k_record<<<v.n, 1024, 0, e->side>>>(v.d_desc, v.n, 1); }
  CUDA_TRY(cudaEventRecord(e->join, e->side));
  // the run generator's top-up and the placement levels, on their own
  // stream beside the variation; the generational round draws one
  // run-generator output at its end instead (k_gen_finish)
  if (!v.generational) {
    CUDA_TRY(cudaStreamWaitEvent(e->draws, e->fork, 0));
    { Timed t(e, KN_STREAM, e->draws); gb::k_stream<<<v.n, 256, 0, e->draws>>>(v.d_desc, v.n); }
    if (v.total_children >= gb::kClusterMinChildren) {
      // the placement levels follow from the draws alone: found here, beside
      // the variation, so the placement itself only compares and writes keys
      Timed t(e, KN_LEVELS, e->draws);
      const int local_P = (v.max_P + gb::kPlaceCtas - 1) / gb::kPlaceCtas;
      gb::k_place_levels<<<v.n * gb::kPlaceCtas, gb::kClusterThreads, 2 * size_t(local_P) * sizeof(int32_t) + 16,
                           e->draws>>>(v.d_desc, v.n);
    }
    CUDA_TRY(cudaEventRecord(e->drawn, e->draws));
  }
  // per range c: counts[4c] / [4c+1] lowered-program list sizes, [4c+2] the
  // next child of the variation warps; range c's lists start at item lo
  CUDA_TRY(cudaMemsetAsync(e->d_counts, 0, kCountWords * sizeof(int32_t), e->stream));
  CUDA_TRY(cudaEventRecord(e->chunk_fork, e->stream));
  const int chunks = v.total_children >= 4096 ? gagp_engine::kChunks : 1;
  const int warps = 4;
  // a range whose children all belong to one search stages that search's
  // generator image in shared memory (when it is small enough to keep the
  // variation kernel's occupancy)
  auto range_of = [&](int c) {
    return std::make_pair(int(int64_t(v.total_children) * c / chunks),
                          int(int64_t(v.total_children) * (c + 1) / chunks));
  };
  int staged[gagp_engine::kChunks];
  size_t image_max = 0;
  for (int c = 0; c < chunks; ++c) {
    const auto [lo, hi] = range_of(c);
    staged[c] = -1;
    const int si = int(std::upper_bound(v.child_off.begin(), v.child_off.end(), lo) - v.child_off.begin()) - 1;
    if (si >= 0 && si < v.n && hi <= v.child_off[si + 1] && v.image_bytes[si] <= kMaxStagedImage) {
      staged[c] = si;
      image_max = std::max(image_max, v.image_bytes[si]);
    }
  }
  const size_t vary_smem = warps * gb::warp_rows_bytes(v.max_stride) + image_max;
  // With ranges, the VM that a round rarely needs gets one launch for all
  // ranges once they have joined: the exact VM in rounds of mostly
  // accumulator programs, and in rounds of mostly exact-VM programs (list
  // programs) both, so that the exact VM's persistent blocks see every
  // program at once.  A per-range launch, mostly empty, still waits for SM
  // room (shared memory) behind the other ranges' VM blocks, on its range's
  // critical path.  The lowering then lists those programs in one shared
  // list (counts at shared_count: [0] fast, [1] exact).
  const bool shared_exact = chunks > 1;
  const bool shared_fast = chunks > 1 && v.exact_heavy;
  int32_t* shared_count = e->d_counts + 4 * gagp_engine::kChunks;
  int per_sm = 0;
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gb::k_vary, warps * 32, vary_smem));
  for (int c = 0; c < chunks; ++c) {
    const auto [lo, hi] = range_of(c);
    cudaStream_t st = chunks == 1 ? e->stream : e->chunk_stream[c];
    if (chunks > 1) CUDA_TRY(cudaStreamWaitEvent(st, e->chunk_fork, 0));
    int32_t* counts = e->d_counts + 4 * c;
    {
      Timed t(e, KN_VARY, st);
      // each range gets its share of the GPU, so that all ranges start at once
      // and the slowest children of every range overlap one another
      const int share = std::max(1, std::max(1, per_sm) * e->sm_count / chunks);
      const int blocks = std::min(blocks_for(hi - lo, warps), share);
      gb::k_vary<<<blocks, warps * 32, vary_smem, st>>>(v.d_desc, v.d_child_off, v.n, v.max_stride, counts + 2, lo,
                                                        hi, e->profiling ? 1 : 0, staged[c],
                                                        staged[c] >= 0 ? int(v.image_bytes[staged[c]]) : 0);
    }
    CUDA_TRY(cudaStreamWaitEvent(st, e->indexed, 0));
    {
      Timed t(e, KN_LOWER, st);
      gb::k_lower<<<blocks_for(hi - lo, gb::kLowerWarps), gb::kLowerWarps * 32, 0, st>>>(
          v.d_desc, v.d_child_off, v.n, 1, shared_fast ? e->d_fast : e->d_fast + lo,
          shared_exact ? e->d_general : e->d_general + lo, shared_fast ? shared_count : counts,
          shared_exact ? shared_count + 1 : counts + 1, lo, hi);
    }
    if (shared_fast) {
      // both VMs after the join
    } else if (shared_exact) {
      if (const gagp_status st2 = launch_vm_fast(e, v, 1, st, e->d_fast + lo, counts, vm); st2 != GAGP_OK) return st2;
    } else {
      if (const gagp_status st2 = launch_vm(e, v, 1, st, e->d_fast + lo, e->d_general + lo, counts, vm);
          st2 != GAGP_OK)
        return st2;
    }
    if (chunks > 1) {
      CUDA_TRY(cudaEventRecord(e->chunk_done[c], st));
      CUDA_TRY(cudaStreamWaitEvent(e->stream, e->chunk_done[c], 0));
    }
  }
  if (shared_exact) {
    // all ranges' exact-VM programs (and, in exact-heavy rounds, their
    // accumulator programs) at once
    if (shared_fast)
      if (const gagp_status st2 = launch_vm_fast(e, v, 1, e->stream, e->d_fast, shared_count, vm); st2 != GAGP_OK)
        return st2;
    Timed t(e, KN_VM_GENERAL);
    if (const gagp_status st2 = vm_general_launch(e->sm_count, e->stream, v.d_desc, 1, e->d_general, shared_count,
                                                  v.max_bc_stride, v.exact_heavy, e->d_region,
                                                  e->d_counts + kRegionCount);
        st2 != GAGP_OK)
      return st2;
  }
  if (v.regions)
    if (const gagp_status st2 = vm_region_launch(e, e->stream, v.d_desc, 1, e->d_region, e->d_counts + kRegionCount);
        st2 != GAGP_OK)
      return st2;
  if (v.generational) {
    // every child becomes the member of its index (reproduce's swap), after
    // the reused children have read their sources' results and the history
    // entry has read the members
    {
      Timed t(e, KN_CHILD);
      gb::k_child_results<<<blocks_for(v.total_children, 128), 128, 0, e->stream>>>(v.d_desc, v.d_child_off, v.n);
    }
    CUDA_TRY(cudaStreamWaitEvent(e->stream, e->join, 0));
    {
      Timed t(e, KN_PLACE);
      gb::k_gen_place<<<blocks_for(v.total_members, 256), 256, 0, e->stream>>>(v.d_desc, v.d_member_off, v.n);
    }
    {
      Timed t(e, KN_COMMIT);
      gb::k_commit<<<blocks_for(size_t(v.total_members) * gb::kCommitLanes, 256), 256, 0, e->stream>>>(
          v.d_desc, v.d_member_off, v.n);
    }
    { Timed t(e, KN_STREAM); gb::k_gen_finish<<<v.n, 256, 0, e->stream>>>(v.d_desc, v.n); }
    return cudaPeekAtLastError() == cudaSuccess ? GAGP_OK : fail(GAGP_DEVICE_ERROR, cudaGetErrorString(cudaGetLastError()));
  }
  // rounds of kClusterMinChildren or more children get their results from
  // the cluster placement itself
  if (v.min_B < gb::kClusterMinChildren) {
    Timed t(e, KN_CHILD);
    gb::k_child_results<<<blocks_for(v.total_children, 128), 128, 0, e->stream>>>(v.d_desc, v.d_child_off, v.n);
  }
  {
    Timed t(e, KN_PLACE);
    // member keys plus as many 16-bit staged draws as fit (B * replacement + slack)
    const size_t limit = e->max_smem - 16384;  // static shared memory of k_place: ~13 KB
    // keys, then either the level owners (4 bytes per member) or the staged draws
    size_t bytes = size_t(v.max_P + 1) * sizeof(uint64_t) +
                   std::max(size_t(v.max_P) * sizeof(int32_t) + 64, size_t(v.max_draws + 64) * sizeof(uint16_t));
    bytes = std::min(bytes, limit);
    CUDA_TRY(cudaStreamWaitEvent(e->stream, e->join, 0));
    CUDA_TRY(cudaStreamWaitEvent(e->stream, e->drawn, 0));
    // the cluster placement first; the single-block kernel replays what it could not place
    const int local_P = (v.max_P + gb::kPlaceCtas - 1) / gb::kPlaceCtas;
    const size_t cluster_bytes = size_t(local_P + 2) * (sizeof(uint64_t) + sizeof(int32_t)) + 16;
    gb::k_place_cluster<<<v.n * gb::kPlaceCtas, gb::kClusterThreads, cluster_bytes, e->stream>>>(v.d_desc, v.n);
    gb::k_place<<<v.n, gb::kPlaceThreads, bytes, e->stream>>>(v.d_desc, v.n, int(bytes), 1);
  }
  { Timed t(e, KN_COMMIT); gb::k_commit<<<blocks_for(size_t(v.total_members) * gb::kCommitLanes, 256), 256, 0, e->stream>>>(v.d_desc, v.d_member_off, v.n); }
  return cudaPeekAtLastError() == cudaSuccess ? GAGP_OK : fail(GAGP_DEVICE_ERROR, cudaGetErrorString(cudaGetLastError()));
}

// The searches of `ids`, each at most once: a repeated id would put one
// search's device state into a batch twice, and both copies would write it.
gagp_status collect(gagp_engine* e, const std::vector<int32_t>& ids, std::vector<Search*>* list) {
  std::vector<int32_t> sorted(ids);
  std::sort(sorted.begin(), sorted.end());
  if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
    return fail(GAGP_INVALID_ARGUMENT, "a search id is listed more than once");
  for (int32_t id : ids) {
    auto it = e->searches.find(id);
    if (it == e->searches.end()) return fail(GAGP_INVALID_ARGUMENT, "unknown search " + std::to_string(id));
    list->push_back(it->second.get());
  }
  return GAGP_OK;
}

gagp_status check_errors(gagp_engine* e, const std::vector<Search*>& list) {
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  harvest(e);
  for (Search* s : list) {
    int32_t round[4];
    CUDA_TRY(copy_d2h(e, round, s->desc.round, sizeof(round)));
    if (round[3]) return fail(GAGP_DEVICE_ERROR, "search " + std::to_string(s->id) + " failed on the device (code " + std::to_string(round[3]) + ")");
  }
  return GAGP_OK;
}

// One round of a fixed batch captured as a CUDA graph (its fork/join over the
// side and range streams included), so that a sequence of rounds costs one
// graph launch each instead of ~30 stream operations.  The round's kernels
// read everything that changes between rounds from device memory, so the
// same graph serves every round of the batch.
struct RoundGraph {
  cudaGraphExec_t exec = nullptr;
  ~RoundGraph() { if (exec) cudaGraphExecDestroy(exec); }
};
gagp_status capture_round(gagp_engine* e, const BatchView& v, RoundGraph* out) {
  CUDA_TRY(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  const gagp_status st = launch_round(e, v, false);
  cudaGraph_t graph = nullptr;
  const cudaError_t ended = cudaStreamEndCapture(e->stream, &graph);  // always leaves capture mode
  if (st != GAGP_OK) {
    if (graph) cudaGraphDestroy(graph);
    return st;
  }
  if (ended != cudaSuccess) return fail(GAGP_DEVICE_ERROR, std::string("round capture: ") + cudaGetErrorString(ended));
  const cudaError_t made = cudaGraphInstantiate(&out->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (made != cudaSuccess) return fail(GAGP_DEVICE_ERROR, std::string("round graph: ") + cudaGetErrorString(made));
  return GAGP_OK;
}
// `rounds` rounds of a batch: graph replays, or direct launches while
// per-kernel timing is on (its events are recorded per launch).
gagp_status launch_rounds(gagp_engine* e, const BatchView& v, int rounds) {
  if (rounds <= 0) return GAGP_OK;
  if (e->profiling || rounds == 1) {
    for (int r = 0; r < rounds; ++r) {
      const gagp_status st = launch_round(e, v);
      if (st != GAGP_OK) return st;
    }
    return GAGP_OK;
  }
  // an untuned batch shape times its VM candidates on the first rounds
  int r = 0;
  while (r < rounds && e->vm_tune[vm_key(v.max_C, v.max_inputs)].chosen < 0 && r < 3 * kTuneRounds) {
    const gagp_status st = launch_round(e, v);
    if (st != GAGP_OK) return st;
    ++r;
  }
  if (r) {
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    harvest(e);
  }
  if (r >= rounds) return GAGP_OK;
  RoundGraph g;
  const gagp_status st = capture_round(e, v, &g);
  if (st != GAGP_OK) return st;
  for (; r < rounds; ++r) CUDA_TRY(cudaGraphLaunch(g.exec, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));  // the graph is destroyed on return
  return GAGP_OK;
}

gagp_status run_batch(gagp_engine* e, const std::vector<Search*>& list) {
  BatchView v;
  gagp_status st = make_batch_view(e, list, &v);
  if (st != GAGP_OK) return st;
  std::vector<Search*> fresh;
  for (Search* s : list) if (!s->started) fresh.push_back(s);
  if (!fresh.empty()) {
    BatchView fv;
    if (fresh.size() == list.size()) fv = v;
    else if ((st = make_batch_view(e, fresh, &fv)) != GAGP_OK) return st;
    if ((st = launch_start(e, fv)) != GAGP_OK) return st;
    for (Search* s : fresh) s->started = true;
    if (fresh.size() != list.size() && (st = make_batch_view(e, list, &v)) != GAGP_OK) return st;
  }
  if ((st = launch_rounds(e, v, v.max_rounds)) != GAGP_OK) return st;
  return check_errors(e, list);
}

}  // namespace

// ======================================================================= row evaluation
namespace {

// Device layout of one row evaluation: grammar tables, cases, the rows as
// node words, lowered programs, program lists and outputs, all carved from
// one caller-provided device region.
struct EvalPlan {
  Layout L;
  size_t desc, ex, info, minimum, local_types, regions, inputs, expected, lists, node, cval, len, code, code_len, kpool,
      code_temps, vm_acc, bc, bc_len, bc_locals, bc_consts, fitness, wrong, errors, counters, round, fast, general,
      counts, off, region_list, region_ws;
  int stride, code_stride, bc_stride;
  size_t region_words;  // bounded-region workspace per lane (0: the grammar has none)
};
// Lanes of a row evaluation's bounded-region kernel.
constexpr int kRowRegionBlocks = 64;

EvalPlan plan_eval(const gagp_grammar* g, const gagp_cases* c, int rows) {
  EvalPlan p{};
  const int maxv = g->max_nodes - g->fixed_nodes;
  p.stride = int(align_up(size_t(std::max(1, maxv)), 4));
  p.code_stride = 2 * maxv + 8;
  p.bc_stride = bytecode_bound(g, maxv);
  const int E = g->expression_count, C = c->case_count;
  const size_t R = size_t(std::max(1, rows)), S = size_t(p.stride);
  auto& L = p.L;
  p.desc = L.take(sizeof(gb::SearchDesc));
  p.ex = L.take(sizeof(gagp_expression) * E);
  p.info = L.take(sizeof(gb::ExprInfo) * E);
  p.minimum = L.take(sizeof(uint32_t));
  p.local_types = L.take(sizeof(int32_t) * GAGP_MAX_LOCALS);
  p.regions = L.take(sizeof(gb::RegionInfo) * size_t(std::max(1, g->region_count)));
  p.inputs = L.take(sizeof(int64_t) * size_t(std::max(1, c->input_count)) * C);
  p.expected = L.take(sizeof(int64_t) * C);
  p.lists = L.take(sizeof(int64_t) * size_t(std::max<int64_t>(1, c->list_values ? c->list_value_count : 0)));
  p.node = L.take(8 * S * R); p.cval = L.take(8 * S * R); p.len = L.take(4 * R);
  p.code = L.take(8 * R * p.code_stride); p.code_len = L.take(4 * R); p.kpool = L.take(8 * R * S);
  p.code_temps = L.take(4 * R); p.vm_acc = L.take(16 * R);
  p.bc = L.take(20 * R * p.bc_stride); p.bc_len = L.take(4 * R); p.bc_locals = L.take(4 * R);
  p.bc_consts = L.take(8 * R * p.bc_stride);
  p.fitness = L.take(8 * R); p.wrong = L.take(4 * R); p.errors = L.take(4 * R);
  p.counters = L.take(8 * GAGP_COUNTERS); p.round = L.take(16);
  p.fast = L.take(sizeof(gb::ProgramRef) * R); p.general = L.take(sizeof(gb::ProgramRef) * R);
  p.counts = L.take(16); p.off = L.take(8);
  p.region_words = 0;
  for (int r = 0; r < g->region_count; ++r)
    if (g->regions[r].traversal == 0)
      p.region_words = std::max(p.region_words, gb::region_lane_words(gb::region_info_of(g->regions[r])));
  p.region_list = L.take(sizeof(gb::ProgramRef) * R);
  p.region_ws = L.take(8 * std::max<size_t>(1, p.region_words * kRowRegionBlocks * gb::kRegionThreads));
  return p;
}

gagp_status eval_check(const gagp_grammar* g, const gagp_cases* c, const gagp_search_config* cfg,
                       const gagp_rows* rows) {
  if (!g || !c || !cfg || !rows) return fail(GAGP_INVALID_ARGUMENT, "null argument");
  if (cfg->metric != GAGP_METRIC_ABSOLUTE && cfg->metric != GAGP_METRIC_EXACT)
    return fail(GAGP_DECLINED, "fitness metric outside the resident scalar subset");
  const double pen = std::fabs(cfg->penalty);
  if (pen != std::floor(pen) || pen < 1 || pen > 2147483647.0)
    return fail(GAGP_DECLINED, "a fractional penalty needs the ordered 48-bit reduction");
  if (c->case_count < 1 || double(c->case_count) * pen >= 281474976710656.0)
    return fail(GAGP_DECLINED, "cases * penalty must stay below 2^48");
  if (c->input_count != g->local_count || g->local_count > GAGP_MAX_LOCALS)
    return fail(GAGP_INVALID_ARGUMENT, "case inputs must cover the grammar inputs");
  if (g->expression_count < 1 || g->expression_count > 65534) return fail(GAGP_DECLINED, "expression table capacity");
  const int maxv = g->max_nodes - g->fixed_nodes;
  if (maxv < 1 || maxv > gb::kMaxLowerNodes) return fail(GAGP_DECLINED, "variable node budget outside 1..256");
  if (const gagp_status st = check_tables_and_cases(g, c); st != GAGP_OK) return st;
  if (rows->count < 0 || (rows->count && (!rows->node_counts || !rows->origins || !rows->constant_counts)))
    return fail(GAGP_INVALID_ARGUMENT, "rows");
  for (int r = 0; r < rows->count; ++r) {
    const int n = rows->node_counts[r], nc = rows->constant_counts[r];
    if (n < 1 || n > maxv || nc < 0 || nc > n || n > rows->stride)
      return fail(GAGP_INVALID_ARGUMENT, "row " + std::to_string(r) + " outside the node budget");
    for (int i = 0; i < n; ++i) {
      const int o = rows->origins[size_t(r) * rows->stride + i];
      if (o < 0 || o >= g->expression_count) return fail(GAGP_INVALID_ARGUMENT, "row origin out of range");
    }
  }
  return GAGP_OK;
}

// Fills `region` (device, plan.L.total bytes) and evaluates every row on
// `stream`; results are copied to the host arrays (`wrong` and `errors`, the
// cases that ended in a runtime error, may be null).  No device allocation.
gagp_status eval_rows_in(char* region, const EvalPlan& p, const gagp_grammar* g, const gagp_cases* c,
                         const gagp_search_config* cfg, const gagp_rows* rows, double* fitness, uint32_t* wrong,
                         uint32_t* errors, cudaStream_t stream, int sm_count, size_t max_smem) {
  const int E = g->expression_count, C = c->case_count, NI = c->input_count, R = rows->count;
  if (R == 0) return GAGP_OK;
  char* b = region;
  std::vector<gb::ExprInfo> info(E);
  for (int i = 0; i < E; ++i) {
    const gagp_expression& x = g->expressions[i];
    gb::ExprInfo& f = info[i];
    f.kind = int8_t(x.kind);
    f.node_kind = int8_t(x.node_kind);
    f.arity = int8_t(x.kind == gb::EK_REFERENCE ? 0 : x.arity);
    f.type = int8_t(x.type);
    f.opcode = int16_t(x.opcode);
    f.operand = x.operand;
    f.target = x.target;
    f.site_nt = -1;
    f.site_class = -1;
  }
  std::vector<int64_t> inputs(size_t(std::max(1, NI)) * C, 0);
  for (int j = 0; j < NI; ++j)
    for (int k = 0; k < C; ++k) inputs[size_t(j) * C + k] = c->inputs[size_t(k) * NI + j];
  std::vector<int32_t> local_types(GAGP_MAX_LOCALS, GAGP_TAG_INVALID);
  for (int j = 0; j < g->local_count; ++j) local_types[j] = g->local_types[j];
  // rows as node words: evaluation reads the construction expression, arity
  // and constant flag only
  const size_t S = size_t(p.stride);
  std::vector<uint64_t> node(S * R, 0);
  std::vector<int64_t> cval(S * R, 0);
  std::vector<int32_t> len(R);
  for (int r = 0; r < R; ++r) {
    const int n = rows->node_counts[r], nc = rows->constant_counts[r];
    for (int i = 0; i < n; ++i) {
      const int o = rows->origins[size_t(r) * rows->stride + i];
      const gagp_expression& x = g->expressions[o];
      node[S * r + i] = uint64_t(uint32_t(o)) | (uint64_t(uint32_t(x.arity) & 0xfu) << 48) |
                        (uint64_t(x.kind == gb::EK_CONSTANT) << 52) | (uint64_t(gb::kNoClass) << 53);
    }
    for (int k = 0; k < nc; ++k) cval[S * r + k] = rows->constants[size_t(r) * rows->stride + k];
    len[r] = n | (nc << 16);
  }
  gb::SearchDesc d{};
  d.ex = at<gagp_expression>(b, p.ex);
  d.info = at<gb::ExprInfo>(b, p.info);
  d.minimum = at<uint32_t>(b, p.minimum);
  d.prod_minimum = d.minimum;  // no subtree generation in row evaluation
  d.local_types = at<int32_t>(b, p.local_types);
  d.regions = at<gb::RegionInfo>(b, p.regions);
  d.n_regions = g->region_count;
  d.n_ex = E;
  d.slot_type = g->slot_type;
  d.result_type = result_type_of(g);
  d.unit_fuel = unit_fuel(g) ? 1 : 0;
  d.local_count = g->local_count;
  d.max_nodes = g->max_nodes;
  d.fixed_nodes = g->fixed_nodes;
  d.return_fuel = g->return_fuel;
  d.P = R;
  d.B = 1;
  d.maxv = g->max_nodes - g->fixed_nodes;
  d.stride = p.stride;
  d.has_wrong = 1;
  d.metric = cfg->metric;
  d.fuel = cfg->fuel;
  d.penalty = cfg->penalty;
  d.penalty_int = (int64_t)std::fabs(cfg->penalty);
  d.inputs = at<int64_t>(b, p.inputs);
  d.expected = at<int64_t>(b, p.expected);
  const int64_t n_lists = c->list_values ? c->list_value_count : 0;
  d.lists = at<int64_t>(b, p.lists);
  d.n_lists = n_lists;
  d.C = C;
  d.n_inputs = NI;
  d.expected_tag = c->expected_tag;
  d.vm_cases_per_lane = cases_per_lane(C);
  d.node = at<uint64_t>(b, p.node);
  d.cval = at<int64_t>(b, p.cval);
  d.len = at<int32_t>(b, p.len);
  d.code = at<uint2>(b, p.code);
  d.code_len = at<int32_t>(b, p.code_len);
  d.kpool = at<int64_t>(b, p.kpool);
  d.code_stride = p.code_stride;
  d.code_temps = at<int32_t>(b, p.code_temps);
  d.vm_acc = at<unsigned long long>(b, p.vm_acc);
  d.bc = at<int32_t>(b, p.bc);
  d.bc_len = at<int32_t>(b, p.bc_len);
  d.bc_locals = at<int32_t>(b, p.bc_locals);
  d.bc_consts = at<int64_t>(b, p.bc_consts);
  d.bc_stride = p.bc_stride;
  d.fitness = at<double>(b, p.fitness);
  d.wrong = at<uint32_t>(b, p.wrong);
  d.errors = at<uint32_t>(b, p.errors);
  d.counters = at<uint64_t>(b, p.counters);
  d.round = at<int32_t>(b, p.round);
  const int32_t off[2] = {0, R};
  auto up = [&](size_t at_off, const void* src, size_t bytes) {
    return cudaMemcpyAsync(b + at_off, src, bytes, cudaMemcpyHostToDevice, stream);
  };
  CUDA_TRY(up(p.desc, &d, sizeof d));
  CUDA_TRY(up(p.ex, g->expressions, sizeof(gagp_expression) * E));
  CUDA_TRY(up(p.info, info.data(), sizeof(gb::ExprInfo) * E));
  CUDA_TRY(up(p.local_types, local_types.data(), sizeof(int32_t) * GAGP_MAX_LOCALS));
  const std::vector<gb::RegionInfo> regions = region_infos(g);
  CUDA_TRY(up(p.regions, regions.data(), sizeof(gb::RegionInfo) * regions.size()));
  CUDA_TRY(up(p.inputs, inputs.data(), sizeof(int64_t) * inputs.size()));
  CUDA_TRY(up(p.expected, c->expected, sizeof(int64_t) * C));
  if (n_lists) CUDA_TRY(up(p.lists, c->list_values, sizeof(int64_t) * size_t(n_lists)));
  CUDA_TRY(up(p.node, node.data(), 8 * node.size()));
  CUDA_TRY(up(p.cval, cval.data(), 8 * cval.size()));
  CUDA_TRY(up(p.len, len.data(), 4 * len.size()));
  CUDA_TRY(up(p.off, off, sizeof off));
  CUDA_TRY(cudaMemsetAsync(b + p.counters, 0, 8 * GAGP_COUNTERS, stream));
  CUDA_TRY(cudaMemsetAsync(b + p.round, 0, 16, stream));
  CUDA_TRY(cudaMemsetAsync(b + p.counts, 0, 16, stream));
  const gb::SearchDesc* dd = at<gb::SearchDesc>(b, p.desc);
  const int32_t* doff = at<int32_t>(b, p.off);
  gb::ProgramRef* fast = at<gb::ProgramRef>(b, p.fast);
  gb::ProgramRef* general = at<gb::ProgramRef>(b, p.general);
  int32_t* counts = at<int32_t>(b, p.counts);
  gb::k_lower<<<blocks_for(R, gb::kLowerWarps), gb::kLowerWarps * 32, 0, stream>>>(dd, doff, 1, 0, fast, general, counts,
                                                                                  counts + 1, 0, R);
  const int warps = 8;
  const int lanes = d.vm_cases_per_lane;
  const int temp_stride = gb::kMaxTemps * lanes * 32;
  const int code_stride = (p.code_stride + 1) & ~1;
  const size_t smem = size_t(warps) * (temp_stride + code_stride + p.stride) * sizeof(int64_t);
  if (smem > max_smem - 1024) return fail(GAGP_DECLINED, "program too long for the VM's shared memory");
  const int per_sm = std::max(1, std::min(4, int((max_smem - 1024) / smem)));
  vm_fast_launch(lanes, sm_count * per_sm, warps * 32, smem, stream, dd, 0, fast, counts, temp_stride, code_stride,
                 p.stride, C);
  if (vm_general_smem(p.bc_stride) > max_smem - 1024) return fail(GAGP_DECLINED, "program too long for the exact VM");
  gb::ProgramRef* region_list = at<gb::ProgramRef>(b, p.region_list);
  if (const gagp_status st = vm_general_launch(sm_count, stream, dd, 0, general, counts, p.bc_stride, true,
                                               region_list, counts + 2);
      st != GAGP_OK)
    return st;
  if (p.region_words)
    gb::k_vm_region<<<kRowRegionBlocks, gb::kRegionThreads, 0, stream>>>(dd, 0, region_list, counts + 2,
                                                                          at<int64_t>(b, p.region_ws), p.region_words);
  CUDA_TRY(cudaGetLastError());
  int32_t round[4];
  CUDA_TRY(cudaMemcpyAsync(round, b + p.round, sizeof round, cudaMemcpyDeviceToHost, stream));
  CUDA_TRY(cudaMemcpyAsync(fitness, b + p.fitness, 8 * size_t(R), cudaMemcpyDeviceToHost, stream));
  if (wrong) CUDA_TRY(cudaMemcpyAsync(wrong, b + p.wrong, 4 * size_t(R), cudaMemcpyDeviceToHost, stream));
  if (errors) CUDA_TRY(cudaMemcpyAsync(errors, b + p.errors, 4 * size_t(R), cudaMemcpyDeviceToHost, stream));
  CUDA_TRY(cudaStreamSynchronize(stream));
  if (round[3]) return fail(GAGP_DEVICE_ERROR, "row evaluation failed on the device (code " + std::to_string(round[3]) + ")");
  return GAGP_OK;
}

}  // namespace

// ======================================================================= evaluation without device allocation
namespace {

// Device scratch of gagp_b200_evaluate_rows_static: every device that loads
// this library holds these bytes until the process exits.  In host code the
// name is only a handle for the symbol; its device address comes from
// cudaGetSymbolAddress (static_scratch_on).
constexpr size_t kStaticScratchBytes = size_t(32) << 20;
static __device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

struct StaticDevice {
  bool ready = false;
  char* scratch = nullptr;  // device address of g_static_scratch on this device
  int sm_count = 0;
  size_t max_smem = 0;
};
std::mutex g_static_mutex;
std::map<int, StaticDevice> g_static_devices;

// Once per device, with that device current: the scratch's device address,
// the SM count and the VM kernel's shared-memory opt-in.
gagp_status static_scratch_on(int device, StaticDevice** out) {
  std::lock_guard<std::mutex> lock(g_static_mutex);
  StaticDevice& d = g_static_devices[device];
  if (!d.ready) {
    void* ptr = nullptr;
    const cudaError_t rc = cudaGetSymbolAddress(&ptr, g_static_scratch);
    if (rc != cudaSuccess) return fail(GAGP_DEVICE_ERROR, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(rc));
    int sms = 0, smem = 0;
    CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    CUDA_TRY(cudaDeviceGetAttribute(&smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    CUDA_TRY(cudaFuncSetAttribute(gb::k_vm_fast<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem - 1024));
    CUDA_TRY(cudaFuncSetAttribute(gb::k_vm_fast<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem - 1024));
    CUDA_TRY(cudaFuncSetAttribute(gb::k_vm_fast<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem - 1024));
    CUDA_TRY(cudaFuncSetAttribute(gb::k_vm_general, cudaFuncAttributeMaxDynamicSharedMemorySize, smem - 1024));
    d.scratch = static_cast<char*>(ptr);
    d.sm_count = sms;
    d.max_smem = size_t(smem);
    d.ready = true;
  }
  *out = &d;
  return GAGP_OK;
}

}  // namespace

extern "C" {

gagp_status gagp_b200_search_run(gagp_engine* e, int32_t id) {
  if (!e) return fail(GAGP_INVALID_ARGUMENT, "null engine");
  if (e->poisoned) return fail(GAGP_DEVICE_ERROR, "engine is poisoned by an earlier device error");
  CUDA_TRY(cudaSetDevice(e->device));
  std::vector<Search*> list;
  gagp_status st = collect(e, {id}, &list);
  if (st != GAGP_OK) return st;
  st = run_batch(e, list);
  if (st == GAGP_DEVICE_ERROR && cudaGetLastError() != cudaSuccess) e->poisoned = true;
  return st;
}

gagp_status gagp_b200_batch_run(gagp_engine* e, const int32_t* ids, int32_t count) {
  if (!e || (!ids && count)) return fail(GAGP_INVALID_ARGUMENT, "null argument");
  if (e->poisoned) return fail(GAGP_DEVICE_ERROR, "engine is poisoned by an earlier device error");
  CUDA_TRY(cudaSetDevice(e->device));
  std::vector<Search*> list;
  gagp_status st = collect(e, std::vector<int32_t>(ids, ids + count), &list);
  if (st != GAGP_OK || list.empty()) return st;
  st = run_batch(e, list);
  if (st == GAGP_DEVICE_ERROR && cudaGetLastError() != cudaSuccess) e->poisoned = true;
  return st;
}

static gagp_status batch_step_body(gagp_engine* e, const int32_t* ids, int32_t count, int32_t* finished) {
  CUDA_TRY(cudaSetDevice(e->device));
  std::vector<Search*> list;
  gagp_status st = collect(e, std::vector<int32_t>(ids, ids + count), &list);
  if (st != GAGP_OK || list.empty()) return st;
  BatchView v;
  std::vector<Search*> fresh;
  for (Search* s : list) if (!s->started) fresh.push_back(s);
  if (!fresh.empty()) {
    if ((st = make_batch_view(e, fresh, &v)) != GAGP_OK) return st;
    if ((st = launch_start(e, v)) != GAGP_OK) return st;
    for (Search* s : fresh) s->started = true;
  }
  if ((st = make_batch_view(e, list, &v)) != GAGP_OK) return st;
  if ((st = launch_round(e, v)) != GAGP_OK) return st;
  if ((st = check_errors(e, list)) != GAGP_OK) return st;
  if (finished)
    for (int i = 0; i < count; ++i) {
      int32_t round[4];
      CUDA_TRY(copy_d2h(e, round, list[i]->desc.round, sizeof(round)));
      finished[i] = round[2];
    }
  return GAGP_OK;
}

static gagp_status batch_start_body(gagp_engine* e, const int32_t* ids, int32_t count) {
  CUDA_TRY(cudaSetDevice(e->device));
  std::vector<Search*> list, fresh;
  gagp_status st = collect(e, std::vector<int32_t>(ids, ids + count), &list);
  if (st != GAGP_OK) return st;
  for (Search* s : list) if (!s->started) fresh.push_back(s);
  if (fresh.empty()) return GAGP_OK;
  BatchView v;
  if ((st = make_batch_view(e, fresh, &v)) != GAGP_OK) return st;
  if ((st = launch_start(e, v)) != GAGP_OK) return st;
  for (Search* s : fresh) s->started = true;
  return check_errors(e, fresh);
}

// Round timing events of one batch_advance call, destroyed on every return.
struct RoundMarks {
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> marks;
  ~RoundMarks() {
    for (auto& m : marks) {
      if (m.first) cudaEventDestroy(m.first);
      if (m.second) cudaEventDestroy(m.second);
    }
  }
};

static gagp_status batch_advance_body(gagp_engine* e, const int32_t* ids, int32_t count, int32_t rounds,
                                      int32_t flush_l2, double* device_ms) {
  CUDA_TRY(cudaSetDevice(e->device));
  std::vector<Search*> list;
  gagp_status st = collect(e, std::vector<int32_t>(ids, ids + count), &list);
  if (st != GAGP_OK || list.empty()) return st;
  for (Search* s : list)
    if (!s->started) return fail(GAGP_INVALID_ARGUMENT, "start the searches first (gagp_b200_batch_start)");
  BatchView v;
  if ((st = make_batch_view(e, list, &v)) != GAGP_OK) return st;
  if (flush_l2 && !e->flush_buffer) {
    e->flush_bytes = size_t(256) << 20;  // twice the B200's 126 MB L2
    CUDA_TRY(cudaMalloc(&e->flush_buffer, e->flush_bytes));
  }
  RoundMarks marks;
  RoundGraph graph;
  const bool replay = !e->profiling && rounds > 1 && e->vm_tune[vm_key(v.max_C, v.max_inputs)].chosen >= 0;
  if (replay && (st = capture_round(e, v, &graph)) != GAGP_OK) return st;
  for (int r = 0; r < rounds; ++r) {
    if (flush_l2) CUDA_TRY(cudaMemsetAsync(e->flush_buffer, r & 0xff, e->flush_bytes, e->stream));
    marks.marks.push_back({nullptr, nullptr});
    auto& m = marks.marks.back();
    CUDA_TRY(cudaEventCreate(&m.first));
    CUDA_TRY(cudaEventCreate(&m.second));
    CUDA_TRY(cudaEventRecord(m.first, e->stream));
    if (replay) CUDA_TRY(cudaGraphLaunch(graph.exec, e->stream));
    else if ((st = launch_round(e, v)) != GAGP_OK) return st;
    CUDA_TRY(cudaEventRecord(m.second, e->stream));
  }
  st = check_errors(e, list);
  double total = 0;
  for (auto& m : marks.marks) {
    float ms = 0;
    cudaEventElapsedTime(&ms, m.first, m.second);
    total += ms;
  }
  if (device_ms) *device_ms = total;
  return st;
}

// Entry points that launch work refuse a poisoned engine and poison it
// after a device error that left a CUDA error pending, as search_run does.
static gagp_status poison_after(gagp_engine* e, gagp_status st) {
  if (st == GAGP_DEVICE_ERROR && cudaGetLastError() != cudaSuccess) e->poisoned = true;
  return st;
}

gagp_status gagp_b200_batch_step(gagp_engine* e, const int32_t* ids, int32_t count, int32_t* finished) {
  if (!e || (!ids && count)) return fail(GAGP_INVALID_ARGUMENT, "null argument");
  if (e->poisoned) return fail(GAGP_DEVICE_ERROR, "engine is poisoned by an earlier device error");
  return poison_after(e, batch_step_body(e, ids, count, finished));
}

gagp_status gagp_b200_batch_start(gagp_engine* e, const int32_t* ids, int32_t count) {
  if (!e || (!ids && count)) return fail(GAGP_INVALID_ARGUMENT, "null argument");
  if (e->poisoned) return fail(GAGP_DEVICE_ERROR, "engine is poisoned by an earlier device error");
  return poison_after(e, batch_start_body(e, ids, count));
}

gagp_status gagp_b200_batch_advance(gagp_engine* e, const int32_t* ids, int32_t count, int32_t rounds,
                                    int32_t flush_l2, double* device_ms) {
  if (!e || (!ids && count) || rounds < 0) return fail(GAGP_INVALID_ARGUMENT, "bad argument");
  if (e->poisoned) return fail(GAGP_DEVICE_ERROR, "engine is poisoned by an earlier device error");
  return poison_after(e, batch_advance_body(e, ids, count, rounds, flush_l2, device_ms));
}

gagp_status gagp_b200_engine_transfers(gagp_engine* e, uint64_t* h2d_bytes, uint64_t* d2h_bytes) {
  if (!e) return fail(GAGP_INVALID_ARGUMENT, "null engine");
  if (h2d_bytes) *h2d_bytes = e->h2d_bytes;
  if (d2h_bytes) *d2h_bytes = e->d2h_bytes;
  return GAGP_OK;
}

gagp_status gagp_b200_search_counters(gagp_engine* e, int32_t id, uint64_t* out, int32_t count) {
  if (!e || !out || count < 0) return fail(GAGP_INVALID_ARGUMENT, "null argument or negative count");
  if (count > GAGP_COUNTERS) count = GAGP_COUNTERS;
  auto it = e->searches.find(id);
  if (it == e->searches.end()) return fail(GAGP_INVALID_ARGUMENT, "unknown search");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  CUDA_TRY(copy_d2h(e, out, it->second->desc.counters, size_t(count) * sizeof(uint64_t)));
  return GAGP_OK;
}

gagp_status gagp_b200_engine_profile(gagp_engine* e, int32_t enable) {
  if (!e) return fail(GAGP_INVALID_ARGUMENT, "null engine");
  e->profiling = enable != 0;
  std::fill(std::begin(e->kernel_ms), std::end(e->kernel_ms), 0.0);
  std::fill(std::begin(e->kernel_launches), std::end(e->kernel_launches), 0LL);
  e->pending.clear();
  e->event_next = 0;
  return GAGP_OK;
}

gagp_status gagp_b200_engine_kernel_stats(gagp_engine* e, int32_t kernel, const char** name, double* total_ms,
                                          int64_t* launches) {
  if (!e || kernel < 0 || kernel >= KN_COUNT) return fail(GAGP_INVALID_ARGUMENT, "kernel index");
  if (name) *name = kKernelNames[kernel];
  if (total_ms) *total_ms = e->kernel_ms[kernel];
  if (launches) *launches = e->kernel_launches[kernel];
  return GAGP_OK;
}

gagp_status gagp_b200_engine_timeline(gagp_engine* e, int32_t capacity, int32_t* kernel, float* start_ms,
                                      float* end_ms, int32_t* count) {
  if (!e || !count || capacity < 0 || (capacity && (!kernel || !start_ms || !end_ms)))
    return fail(GAGP_INVALID_ARGUMENT, "null argument or negative capacity");
  *count = int32_t(e->timeline.size());
  const int32_t n = std::min(capacity, *count);
  for (int32_t i = 0; i < n; ++i) {
    kernel[i] = e->timeline[i].kernel;
    start_ms[i] = e->timeline[i].start;
    end_ms[i] = e->timeline[i].end;
  }
  return GAGP_OK;
}

gagp_status gagp_b200_search_progress(gagp_engine* e, int32_t id, int32_t* rounds_done, int32_t* total_rounds,
                                      int32_t* finished) {
  if (!e) return fail(GAGP_INVALID_ARGUMENT, "null engine");
  auto it = e->searches.find(id);
  if (it == e->searches.end()) return fail(GAGP_INVALID_ARGUMENT, "unknown search");
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  int32_t round[4];
  CUDA_TRY(copy_d2h(e, round, it->second->desc.round, sizeof(round)));
  if (rounds_done) *rounds_done = round[0];
  if (total_rounds) *total_rounds = it->second->total_rounds;
  if (finished) *finished = round[2];
  if (round[3]) return fail(GAGP_DEVICE_ERROR, "search failed on the device (code " + std::to_string(round[3]) + ")");
  return GAGP_OK;
}

gagp_status gagp_b200_evaluate_rows(gagp_engine* e, const gagp_grammar* grammar, const gagp_cases* cases,
                                    const gagp_search_config* config, const gagp_rows* rows, double* fitness,
                                    uint32_t* wrong) {
  if (!e || !fitness) return fail(GAGP_INVALID_ARGUMENT, "null argument");
  if (e->poisoned) return fail(GAGP_DEVICE_ERROR, "engine is poisoned by an earlier device error");
  gagp_status st = eval_check(grammar, cases, config, rows);
  if (st != GAGP_OK) return st;
  CUDA_TRY(cudaSetDevice(e->device));
  const EvalPlan p = plan_eval(grammar, cases, rows->count);
  char* region = nullptr;
  CUDA_TRY(cudaMalloc(&region, p.L.total));
  st = eval_rows_in(region, p, grammar, cases, config, rows, fitness, wrong, nullptr, e->stream, e->sm_count,
                    e->max_smem);
  cudaFree(region);
  return st;
}

gagp_status gagp_b200_judge_rows(gagp_engine* e, const gagp_grammar* grammar, const gagp_cases* cases,
                                 const gagp_search_config* config, const gagp_rows* rows, gagp_verdict* out) {
  if (!e || !out) return fail(GAGP_INVALID_ARGUMENT, "null argument");
  if (e->poisoned) return fail(GAGP_DEVICE_ERROR, "engine is poisoned by an earlier device error");
  gagp_status st = eval_check(grammar, cases, config, rows);
  if (st != GAGP_OK) return st;
  CUDA_TRY(cudaSetDevice(e->device));
  const int R = rows->count, C = cases->case_count;
  std::vector<double> fitness(size_t(std::max(1, R)));
  std::vector<uint32_t> wrong(size_t(std::max(1, R))), errors(size_t(std::max(1, R)));
  const EvalPlan p = plan_eval(grammar, cases, R);
  char* region = nullptr;
  CUDA_TRY(cudaMalloc(&region, p.L.total));
  st = eval_rows_in(region, p, grammar, cases, config, rows, fitness.data(), wrong.data(), errors.data(), e->stream,
                    e->sm_count, e->max_smem);
  cudaFree(region);
  if (st != GAGP_OK) return st;
  // run.cpp's judge_case from the fitness terms: a case is correct exactly
  // when it is not wrong; an Int-expected case whose value is not an Int is
  // an error as a runtime failure is; a correct case loses 0, so with Bool
  // expectations under the absolute metric (whose case score is the ceiling
  // whatever the value) the correct cases' ceilings come off the loss
  const bool type_errors = cases->expected_tag == GAGP_TAG_INT && result_type_of(grammar) != GAGP_TAG_INT;
  const int64_t cap = int64_t(std::fabs(config->penalty));
  for (int r = 0; r < R; ++r) {
    gagp_verdict& v = out[r];
    v.cases = C;
    v.correct = C - int32_t(wrong[r]);
    v.runtime_errors = type_errors ? C : int32_t(errors[r]);
    int64_t loss = int64_t(-fitness[r]);
    if (config->metric == GAGP_METRIC_ABSOLUTE && cases->expected_tag != GAGP_TAG_INT) loss -= int64_t(v.correct) * cap;
    v.loss = double(loss);
  }
  return GAGP_OK;
}

// Row evaluation for callers that may not allocate device memory: it runs the
// same lowering and VM kernels as gagp_b200_evaluate_rows, but every device
// buffer lives in the static scratch above.  See include/gagp_b200.h.
gagp_status gagp_b200_evaluate_rows_static(const gagp_grammar* grammar, const gagp_cases* cases,
                                           const gagp_search_config* config, const gagp_rows* rows,
                                           double* fitness, uint32_t* wrong, void* stream) {
  if (!fitness) return fail(GAGP_INVALID_ARGUMENT, "null fitness output");
  gagp_status st = eval_check(grammar, cases, config, rows);
  if (st != GAGP_OK) return st;
  const EvalPlan p = plan_eval(grammar, cases, rows->count);
  if (p.L.total > kStaticScratchBytes)
    return fail(GAGP_INVALID_ARGUMENT, "this evaluation needs " + std::to_string(p.L.total) +
                                           " bytes of device scratch; the static scratch holds " +
                                           std::to_string(kStaticScratchBytes) +
                                           " bytes: evaluate fewer rows or cases per call");
  int device = 0;
  CUDA_TRY(cudaGetDevice(&device));
  StaticDevice* d = nullptr;
  if ((st = static_scratch_on(device, &d)) != GAGP_OK) return st;
  return eval_rows_in(d->scratch, p, grammar, cases, config, rows, fitness, wrong, nullptr,
                      static_cast<cudaStream_t>(stream), d->sm_count, d->max_smem);
}

gagp_status gagp_b200_search_result(gagp_engine* e, int32_t id, gagp_search_result* out) {
  if (!e || !out) return fail(GAGP_INVALID_ARGUMENT, "null argument");
  auto it = e->searches.find(id);
  if (it == e->searches.end()) return fail(GAGP_INVALID_ARGUMENT, "unknown search");
  Search* s = it->second.get();
  CUDA_TRY(cudaSetDevice(e->device));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  const gb::SearchDesc& d = s->desc;
  int32_t round[4];
  CUDA_TRY(copy_d2h(e, round, d.round, sizeof(round)));
  if (round[3]) return fail(GAGP_DEVICE_ERROR, "search failed on the device (code " + std::to_string(round[3]) + ")");
  if (!round[2]) return fail(GAGP_NOT_READY, "search has not finished");
  const int H = std::min(round[1], out->generations);
  const int P = s->P, S = s->stride;
  // the final population ranked and in transport form on the device, so the
  // host only copies it out
  const int W = S;
  Layout D;
  const size_t d_rank = D.take(4 * size_t(P)), d_fit = D.take(8 * size_t(P)), d_wr = D.take(4 * size_t(P)),
               d_nodes = D.take(4 * size_t(P)), d_nc = D.take(4 * size_t(P)), d_cc = D.take(4 * size_t(P)),
               d_org = D.take(4 * size_t(P) * W), d_con = D.take(8 * size_t(P) * W);
  char* db = nullptr;
  CUDA_TRY(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&db), D.total, e->pool, e->stream));
  gb::k_rank_members<<<blocks_for(P, 128), 128, 0, e->stream>>>(s->d_desc, at<int32_t>(db, d_rank));
  gb::k_export_members<<<blocks_for(size_t(P) * 32, 256), 256, 0, e->stream>>>(
      s->d_desc, at<int32_t>(db, d_rank), W, at<double>(db, d_fit), at<int32_t>(db, d_wr), at<int32_t>(db, d_nodes),
      at<int32_t>(db, d_nc), at<int32_t>(db, d_cc), at<int32_t>(db, d_org), at<int64_t>(db, d_con));
  // every array in one pinned staging area, copied asynchronously, one sync
  Layout L;
  const size_t o_sum = L.take(8 * size_t(H)), o_hf = L.take(8 * size_t(H)), o_hw = L.take(4 * size_t(H)),
               o_hn = L.take(4 * size_t(H)), o_hnode = L.take(8 * size_t(H) * S), o_hc = L.take(8 * size_t(H) * S),
               o_hl = L.take(4 * size_t(H)), o_fit = L.take(8 * size_t(P)), o_wr = L.take(4 * size_t(P)),
               o_nodes = L.take(4 * size_t(P)), o_nc = L.take(4 * size_t(P)), o_cc = L.take(4 * size_t(P)),
               o_org = L.take(4 * size_t(P) * W), o_con = L.take(8 * size_t(P) * W), o_cnt = L.take(8 * 4);
  if (L.total > e->pinned_bytes) {
    if (e->pinned) cudaFreeHost(e->pinned);
    e->pinned = nullptr;
    e->pinned_bytes = 0;
    CUDA_TRY(cudaMallocHost(reinterpret_cast<void**>(&e->pinned), L.total));
    e->pinned_bytes = L.total;
  }
  char* hb = e->pinned;
  auto fetch = [&](size_t off, const void* src, size_t bytes) -> cudaError_t {
    e->d2h_bytes += bytes;
    return bytes ? cudaMemcpyAsync(hb + off, src, bytes, cudaMemcpyDeviceToHost, e->stream) : cudaSuccess;
  };
  CUDA_TRY(fetch(o_sum, d.hist_sum, 8 * size_t(H)));
  CUDA_TRY(fetch(o_hf, d.hist_fitness, 8 * size_t(H)));
  CUDA_TRY(fetch(o_hw, d.hist_wrong, 4 * size_t(H)));
  CUDA_TRY(fetch(o_hn, d.hist_nodes, 4 * size_t(H)));
  CUDA_TRY(fetch(o_hnode, d.hist_node, 8 * size_t(H) * S));
  CUDA_TRY(fetch(o_hc, d.hist_cval, 8 * size_t(H) * S));
  CUDA_TRY(fetch(o_hl, d.hist_len, 4 * size_t(H)));
  // the ranked population: only the rows the caller asked for
  const int n_out = std::min(P, out->population);
  CUDA_TRY(fetch(o_fit, db + d_fit, 8 * size_t(n_out)));
  CUDA_TRY(fetch(o_wr, db + d_wr, 4 * size_t(n_out)));
  CUDA_TRY(fetch(o_nodes, db + d_nodes, 4 * size_t(n_out)));
  CUDA_TRY(fetch(o_nc, db + d_nc, 4 * size_t(n_out)));
  CUDA_TRY(fetch(o_cc, db + d_cc, 4 * size_t(n_out)));
  CUDA_TRY(fetch(o_org, db + d_org, 4 * size_t(n_out) * W));
  CUDA_TRY(fetch(o_con, db + d_con, 8 * size_t(n_out) * W));
  CUDA_TRY(fetch(o_cnt, d.counters, 8 * 4));
  CUDA_TRY(cudaFreeAsync(db, e->stream));
  CUDA_TRY(cudaStreamSynchronize(e->stream));
  const int64_t* sum = reinterpret_cast<const int64_t*>(hb + o_sum);
  const double* hf = reinterpret_cast<const double*>(hb + o_hf);
  const uint32_t* hw = reinterpret_cast<const uint32_t*>(hb + o_hw);
  const uint32_t* hn = reinterpret_cast<const uint32_t*>(hb + o_hn);
  const uint64_t* hnode = reinterpret_cast<const uint64_t*>(hb + o_hnode);
  const int64_t* hc = reinterpret_cast<const int64_t*>(hb + o_hc);
  const int32_t* hl = reinterpret_cast<const int32_t*>(hb + o_hl);
  const uint64_t* counters = reinterpret_cast<const uint64_t*>(hb + o_cnt);
  auto put_row = [&](const gagp_rows& rows, int index, const uint64_t* node, const int64_t* cval, int32_t l) {
    const int n = l & 0xffff, nc = (l >> 16) & 0xffff;
    rows.node_counts[index] = n;
    rows.constant_counts[index] = nc;
    for (int i = 0; i < n && i < rows.stride; ++i) rows.origins[size_t(index) * rows.stride + i] = int32_t(node[i] & 0xffffu);
    for (int i = 0; i < nc && i < rows.stride; ++i) rows.constants[size_t(index) * rows.stride + i] = cval[i];
  };
  for (int h = 0; h < H; ++h) {
    out->history_best_fitness[h] = hf[h];
    // long double mean of member fitness, as the reference forms it (evolve.cpp:370-371)
    out->history_mean_fitness[h] = double((long double)sum[h] / (long double)P);
    out->history_best_wrong[h] = s->has_wrong ? int32_t(hw[h]) : -1;
    out->history_best_nodes[h] = int32_t(hn[h]);
    put_row(out->history_best, h, hnode + size_t(h) * S, hc + size_t(h) * S, hl[h]);
  }
  out->generations = H;
  std::memcpy(out->final_fitness, hb + o_fit, 8 * size_t(n_out));
  std::memcpy(out->final_wrong, hb + o_wr, 4 * size_t(n_out));
  std::memcpy(out->final_nodes, hb + o_nodes, 4 * size_t(n_out));
  const gagp_rows& fr = out->final_rows;
  std::memcpy(fr.node_counts, hb + o_nc, 4 * size_t(n_out));
  std::memcpy(fr.constant_counts, hb + o_cc, 4 * size_t(n_out));
  const int32_t* org = reinterpret_cast<const int32_t*>(hb + o_org);
  const int64_t* con = reinterpret_cast<const int64_t*>(hb + o_con);
  if (fr.stride == W) {
    std::memcpy(fr.origins, org, 4 * size_t(n_out) * W);
    std::memcpy(fr.constants, con, 8 * size_t(n_out) * W);
  } else {
    const int w = std::min(W, fr.stride);
    for (int r = 0; r < n_out; ++r) {
      std::memcpy(fr.origins + size_t(r) * fr.stride, org + size_t(r) * W, 4 * size_t(w));
      std::memcpy(fr.constants + size_t(r) * fr.stride, con + size_t(r) * W, 8 * size_t(w));
    }
  }
  out->population = n_out;
  out->evaluated_programs = counters[0];
  out->reused_programs = counters[1];
  out->program_cases = counters[2];
  return GAGP_OK;
}

}  // extern "C"

// ======================================================================= serving
namespace {

// A queued or running request: owned copies of the caller's blobs, then the
// finished search's result read back to host memory.
struct Request {
  int64_t ticket = 0;
  int32_t state = GAGP_REQUEST_QUEUED;
  std::string error;
  std::vector<gagp_expression> ex;
  std::vector<gagp_production> prods;
  std::vector<gagp_nonterminal> nts;
  std::vector<gagp_domain> doms;
  std::vector<gagp_value> vals;
  std::vector<uint32_t> minimum;
  std::vector<gagp_region> regions;
  std::vector<int64_t> inputs, expected, lists;
  std::vector<int32_t> tags;
  gagp_grammar grammar{};
  gagp_cases cases{};
  gagp_search_config config{};
  uint64_t bytes = 0;
  int32_t search = -1;
  int32_t rounds_done = 0;  // rounds the server has run for this search
  double submitted = -1, admitted = -1, finished = -1;
  // result (gagp_search_result layout)
  int32_t generations = 0, population = 0, stride = 0;
  std::vector<double> hbf, hmf, ff;
  std::vector<int32_t> hbw, hbn, fw, fn;
  std::vector<int32_t> h_nodes, h_orig, h_ncon, f_nodes, f_orig, f_ncon;
  std::vector<int64_t> h_con, f_con;
  uint64_t evaluated = 0, reused = 0, program_cases = 0;
};

template <class T>
std::vector<T> copy_of(const T* p, int32_t n) {
  return p && n > 0 ? std::vector<T>(p, p + n) : std::vector<T>();
}

}  // namespace

struct gagp_server {
  gagp_engine* e = nullptr;
  uint64_t budget = 0;
  int32_t max_active = 0;
  int64_t next_ticket = 1;
  std::deque<int64_t> queue;
  std::vector<int64_t> active;
  std::map<int64_t, std::unique_ptr<Request>> requests;
  int32_t* d_status = nullptr;
  size_t status_capacity = 0;
  // rounds each step runs before the server reads the searches' states
  int32_t rounds_per_step = 1;
  std::chrono::steady_clock::time_point epoch = std::chrono::steady_clock::now();
  double now() const {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - epoch).count();
  }
};

namespace {

// Reads a finished search's result into the request, then frees the search.
gagp_status retire(gagp_server* sv, Request& r) {
  gagp_engine* e = sv->e;
  Search* s = e->searches.at(r.search).get();
  const int H = r.config.generations + 1, P = s->P, S = s->stride;
  r.generations = H;
  r.population = P;
  r.stride = S;
  r.hbf.assign(H, 0); r.hmf.assign(H, 0); r.hbw.assign(H, 0); r.hbn.assign(H, 0);
  r.h_nodes.assign(H, 0); r.h_ncon.assign(H, 0); r.h_orig.assign(size_t(H) * S, -1); r.h_con.assign(size_t(H) * S, 0);
  r.ff.assign(P, 0); r.fw.assign(P, 0); r.fn.assign(P, 0);
  r.f_nodes.assign(P, 0); r.f_ncon.assign(P, 0); r.f_orig.assign(size_t(P) * S, -1); r.f_con.assign(size_t(P) * S, 0);
  gagp_search_result out{};
  out.generations = H;
  out.history_best_fitness = r.hbf.data();
  out.history_mean_fitness = r.hmf.data();
  out.history_best_wrong = r.hbw.data();
  out.history_best_nodes = r.hbn.data();
  out.history_best = gagp_rows{H, S, r.h_nodes.data(), r.h_orig.data(), r.h_ncon.data(), r.h_con.data()};
  out.population = P;
  out.final_fitness = r.ff.data();
  out.final_wrong = r.fw.data();
  out.final_nodes = r.fn.data();
  out.final_rows = gagp_rows{P, S, r.f_nodes.data(), r.f_orig.data(), r.f_ncon.data(), r.f_con.data()};
  const gagp_status st = gagp_b200_search_result(e, r.search, &out);
  if (st == GAGP_OK) {
    r.generations = out.generations;
    r.population = out.population;
    r.evaluated = out.evaluated_programs;
    r.reused = out.reused_programs;
    r.program_cases = out.program_cases;
    r.state = GAGP_REQUEST_DONE;
  } else {
    r.state = GAGP_REQUEST_FAILED;
    r.error = gagp_b200_last_error();
  }
  gagp_b200_search_destroy(e, r.search);
  r.search = -1;
  r.finished = sv->now();
  return st == GAGP_DEVICE_ERROR ? st : GAGP_OK;
}

}  // namespace

extern "C" {

gagp_status gagp_b200_server_set_rounds_per_step(gagp_server* sv, int32_t rounds) {
  if (!sv || rounds < 1 || rounds > 4096) return fail(GAGP_INVALID_ARGUMENT, "rounds per step must be in 1..4096");
  sv->rounds_per_step = rounds;
  return GAGP_OK;
}

gagp_status gagp_b200_server_create(gagp_engine* e, uint64_t memory_budget, int32_t max_active, gagp_server** out) {
  if (!e || !out || max_active < 0) return fail(GAGP_INVALID_ARGUMENT, "bad argument");
  auto sv = std::make_unique<gagp_server>();
  sv->e = e;
  sv->budget = memory_budget ? std::min<uint64_t>(memory_budget, e->arena_limit) : e->arena_limit;
  sv->max_active = max_active;
  *out = sv.release();
  return GAGP_OK;
}

void gagp_b200_server_destroy(gagp_server* sv) {
  if (!sv) return;
  for (int64_t t : sv->active) {
    Request& r = *sv->requests.at(t);
    if (r.search >= 0) gagp_b200_search_destroy(sv->e, r.search);
  }
  if (sv->d_status) {
    cudaSetDevice(sv->e->device);
    cudaFree(sv->d_status);
  }
  delete sv;
}

gagp_status gagp_b200_server_submit(gagp_server* sv, const gagp_grammar* g, const gagp_cases* c,
                                    const gagp_search_config* cfg, int64_t* ticket) {
  if (!sv || !g || !c || !cfg || !ticket) return fail(GAGP_INVALID_ARGUMENT, "null argument");
  if (!cfg->steady_state) return fail(GAGP_DECLINED, "the server batches steady-state searches");
  gagp_status st = admit(g, c, cfg);
  if (st != GAGP_OK) return st;
  const Plan p = plan_search(g, c, cfg);
  if (p.L.total > sv->budget) return fail(GAGP_OUT_OF_MEMORY, "request larger than the server's memory budget");
  auto r = std::make_unique<Request>();
  r->ticket = sv->next_ticket++;
  r->ex = copy_of(g->expressions, g->expression_count);
  r->prods = copy_of(g->productions, g->production_count);
  r->nts = copy_of(g->nonterminals, g->nonterminal_count);
  r->doms = copy_of(g->domains, g->domain_count);
  r->vals = copy_of(g->values, g->value_count);
  r->minimum = copy_of(g->minimum, g->expression_count * g->depth_count * g->logical_depth_count);
  r->regions = copy_of(g->regions, g->region_count);
  r->grammar = *g;
  r->grammar.expressions = r->ex.data();
  r->grammar.productions = r->prods.data();
  r->grammar.nonterminals = r->nts.data();
  r->grammar.domains = r->doms.data();
  r->grammar.values = r->vals.data();
  r->grammar.minimum = r->minimum.data();
  r->grammar.regions = r->regions.empty() ? nullptr : r->regions.data();
  r->inputs = copy_of(c->inputs, c->case_count * c->input_count);
  r->lists = copy_of(c->list_values, c->list_values ? int(c->list_value_count) : 0);
  r->expected = copy_of(c->expected, c->case_count);
  r->tags = copy_of(c->input_tags, c->input_count);
  r->cases = *c;
  r->cases.inputs = r->inputs.data();
  r->cases.expected = r->expected.data();
  r->cases.input_tags = r->tags.empty() ? nullptr : r->tags.data();
  r->cases.list_values = r->lists.empty() ? nullptr : r->lists.data();
  r->config = *cfg;
  r->bytes = p.L.total;
  r->submitted = sv->now();
  *ticket = r->ticket;
  sv->queue.push_back(r->ticket);
  sv->requests[r->ticket] = std::move(r);
  return GAGP_OK;
}

gagp_status gagp_b200_server_step(gagp_server* sv, int32_t* running, int32_t* queued, int32_t* finished_now) {
  if (!sv) return fail(GAGP_INVALID_ARGUMENT, "null server");
  gagp_engine* e = sv->e;
  if (e->poisoned) return fail(GAGP_DEVICE_ERROR, "engine is poisoned by an earlier device error");
  CUDA_TRY(cudaSetDevice(e->device));
  // admission in arrival order while the head request fits
  while (!sv->queue.empty() && (sv->max_active == 0 || int32_t(sv->active.size()) < sv->max_active)) {
    Request& r = *sv->requests.at(sv->queue.front());
    if (e->arena_used + r.bytes > sv->budget) break;
    int32_t id = -1;
    const gagp_status st = gagp_b200_search_create(e, &r.grammar, &r.cases, &r.config, nullptr, &id);
    if (st == GAGP_OUT_OF_MEMORY) break;
    sv->queue.pop_front();
    if (st != GAGP_OK) {
      r.state = GAGP_REQUEST_FAILED;
      r.error = gagp_b200_last_error();
      r.finished = sv->now();
      if (st == GAGP_DEVICE_ERROR) return st;
      continue;
    }
    r.search = id;
    r.state = GAGP_REQUEST_RUNNING;
    r.admitted = sv->now();
    sv->active.push_back(r.ticket);
  }
  int32_t done = 0;
  if (!sv->active.empty()) {
    std::vector<Search*> list, fresh;
    for (int64_t t : sv->active) list.push_back(e->searches.at(sv->requests.at(t)->search).get());
    for (Search* s : list) if (!s->started) fresh.push_back(s);
    BatchView v;
    gagp_status st;
    if (!fresh.empty()) {
      if ((st = make_batch_view(e, fresh, &v)) != GAGP_OK) return st;
      if ((st = launch_start(e, v)) != GAGP_OK) return st;
      for (Search* s : fresh) s->started = true;
    }
    if ((st = make_batch_view(e, list, &v)) != GAGP_OK) return st;
    // up to rounds_per_step rounds (graph replays after the first), no more
    // than the longest remaining search needs; a search that finishes within
    // them idles (its kernels skip finished searches) until the states are
    // read after the last
    int rounds = 1;
    for (int64_t t : sv->active) {
      const Request& r = *sv->requests.at(t);
      rounds = std::max(rounds, e->searches.at(r.search)->total_rounds - r.rounds_done);
    }
    rounds = std::max(1, std::min(rounds, sv->rounds_per_step));
    if ((st = launch_rounds(e, v, rounds)) != GAGP_OK) return st;
    for (int64_t t : sv->active) sv->requests.at(t)->rounds_done += rounds;
    const size_t n = list.size();
    if (n > sv->status_capacity) {
      const size_t cap = std::max(n, 2 * sv->status_capacity);
      cudaFree(sv->d_status);
      CUDA_TRY(cudaMalloc(&sv->d_status, cap * sizeof(int32_t)));
      sv->status_capacity = cap;
    }
    gb::k_status<<<blocks_for(int(n), 256), 256, 0, e->stream>>>(v.d_desc, int(n), sv->d_status);
    std::vector<int32_t> status(n);
    CUDA_TRY(cudaMemcpyAsync(status.data(), sv->d_status, n * sizeof(int32_t), cudaMemcpyDeviceToHost, e->stream));
    CUDA_TRY(cudaStreamSynchronize(e->stream));
    e->d2h_bytes += n * sizeof(int32_t);
    harvest(e);
    std::vector<int64_t> still;
    for (size_t i = 0; i < n; ++i) {
      Request& r = *sv->requests.at(sv->active[i]);
      if (status[i] & 2) {
        r.state = GAGP_REQUEST_FAILED;
        r.error = "search failed on the device";
        gagp_b200_search_destroy(e, r.search);
        r.search = -1;
        r.finished = sv->now();
        ++done;
      } else if (status[i] & 1) {
        if ((st = retire(sv, r)) != GAGP_OK) return st;
        ++done;
      } else {
        still.push_back(r.ticket);
      }
    }
    sv->active.swap(still);
  }
  if (running) *running = int32_t(sv->active.size());
  if (queued) *queued = int32_t(sv->queue.size());
  if (finished_now) *finished_now = done;
  return GAGP_OK;
}

gagp_status gagp_b200_server_poll(gagp_server* sv, int64_t ticket, int32_t* state) {
  if (!sv || !state) return fail(GAGP_INVALID_ARGUMENT, "null argument");
  auto it = sv->requests.find(ticket);
  if (it == sv->requests.end()) return fail(GAGP_INVALID_ARGUMENT, "unknown ticket");
  *state = it->second->state;
  if (it->second->state == GAGP_REQUEST_FAILED) return fail(GAGP_OK, it->second->error);
  return GAGP_OK;
}

gagp_status gagp_b200_server_times(gagp_server* sv, int64_t ticket, double* submitted, double* admitted,
                                   double* finished) {
  if (!sv) return fail(GAGP_INVALID_ARGUMENT, "null server");
  auto it = sv->requests.find(ticket);
  if (it == sv->requests.end()) return fail(GAGP_INVALID_ARGUMENT, "unknown ticket");
  if (submitted) *submitted = it->second->submitted;
  if (admitted) *admitted = it->second->admitted;
  if (finished) *finished = it->second->finished;
  return GAGP_OK;
}

gagp_status gagp_b200_server_result(gagp_server* sv, int64_t ticket, gagp_search_result* out) {
  if (!sv || !out) return fail(GAGP_INVALID_ARGUMENT, "null argument");
  auto it = sv->requests.find(ticket);
  if (it == sv->requests.end()) return fail(GAGP_INVALID_ARGUMENT, "unknown ticket");
  Request& r = *it->second;
  if (r.state == GAGP_REQUEST_FAILED) return fail(GAGP_DEVICE_ERROR, r.error);
  if (r.state != GAGP_REQUEST_DONE) return fail(GAGP_NOT_READY, "request has not finished");
  const int H = std::min(r.generations, out->generations), P = std::min(r.population, out->population);
  auto rows = [&](const gagp_rows& to, int count, const std::vector<int32_t>& nodes, const std::vector<int32_t>& orig,
                  const std::vector<int32_t>& ncon, const std::vector<int64_t>& con) {
    for (int i = 0; i < count; ++i) {
      to.node_counts[i] = nodes[i];
      to.constant_counts[i] = ncon[i];
      for (int k = 0; k < std::min(to.stride, r.stride); ++k) {
        to.origins[size_t(i) * to.stride + k] = orig[size_t(i) * r.stride + k];
        to.constants[size_t(i) * to.stride + k] = con[size_t(i) * r.stride + k];
      }
    }
  };
  for (int h = 0; h < H; ++h) {
    out->history_best_fitness[h] = r.hbf[h];
    out->history_mean_fitness[h] = r.hmf[h];
    out->history_best_wrong[h] = r.hbw[h];
    out->history_best_nodes[h] = r.hbn[h];
  }
  rows(out->history_best, H, r.h_nodes, r.h_orig, r.h_ncon, r.h_con);
  for (int i = 0; i < P; ++i) {
    out->final_fitness[i] = r.ff[i];
    out->final_wrong[i] = r.fw[i];
    out->final_nodes[i] = r.fn[i];
  }
  rows(out->final_rows, P, r.f_nodes, r.f_orig, r.f_ncon, r.f_con);
  out->generations = H;
  out->population = P;
  out->evaluated_programs = r.evaluated;
  out->reused_programs = r.reused;
  out->program_cases = r.program_cases;
  sv->requests.erase(it);
  return GAGP_OK;
}

gagp_status gagp_b200_server_cancel(gagp_server* sv, int64_t ticket) {
  if (!sv) return fail(GAGP_INVALID_ARGUMENT, "null server");
  auto it = sv->requests.find(ticket);
  if (it == sv->requests.end()) return fail(GAGP_INVALID_ARGUMENT, "unknown ticket");
  Request& r = *it->second;
  if (r.search >= 0) gagp_b200_search_destroy(sv->e, r.search);
  sv->queue.erase(std::remove(sv->queue.begin(), sv->queue.end(), ticket), sv->queue.end());
  sv->active.erase(std::remove(sv->active.begin(), sv->active.end(), ticket), sv->active.end());
  sv->requests.erase(it);
  return GAGP_OK;
}

}  // extern "C"
