// On-device lowering of a phase row.
//
// Two outputs per program:
//  * the reference bytecode -- compile_phase_tree for value phases
//    (cpp/src/evolution/repro/gpu/device/phase_compile.cuh:207-895) plus the
//    RETURN that patch_whole_program appends (phase_layout.hpp:476-500) --
//    executed by the exact general VM (fuel, errors, per-lane control flow);
//  * an accumulator program for the fast VM, when the program is provably
//    free of runtime errors and of fuel exhaustion: every operation is total
//    (no unprotected division or modulo) and the bytecode length, an upper
//    bound of any executed path, fits the fuel.  Value ifs, and/or become
//    selects, which cannot change the result of an error-free, side-effect-
//    free expression.  Operands are evaluated in Sethi-Ullman order so that at
//    most kMaxTemps values are ever spilled.
#pragma once
#include "device_ops.cuh"

namespace gb {

// Opcode (cpp/include/gagp/core/opcode.hpp:8-37) and BuiltinId
// (cpp/include/gagp/core/builtin.hpp:13-45) numbers.
enum {
  OP_PUSH_CONST = 0, OP_LOAD = 1, OP_STORE = 2, OP_NEG = 3, OP_NOT = 4, OP_ADD = 5, OP_SUB = 6, OP_MUL = 7,
  OP_DIV = 8, OP_MOD = 9, OP_LT = 10, OP_LE = 11, OP_GT = 12, OP_GE = 13, OP_EQ = 14, OP_NE = 15, OP_JMP = 16,
  OP_JMP_IF_FALSE = 17, OP_JMP_IF_TRUE = 18, OP_CALL_BUILTIN = 19, OP_RETURN = 20, OP_CHECK_INT = 22,
  OP_BOUNDED_REGION = 28
};
enum {
  B_ABS = 0, B_MIN = 1, B_MAX = 2, B_LEN = 4, B_INDEX = 7, B_IS_INT = 12, B_IDIV0 = 13, B_IMOD0 = 14, B_TRUNC_DIV0 = 28,
  B_TRUNC_MOD0 = 29
};

// Accumulator VM operations.
enum : uint32_t {
  A_MOV = 0, A_SPILL, A_ADD, A_SUB, A_MUL, A_NEG, A_NOT, A_ABS, A_LT, A_LE, A_GT, A_GE, A_EQ, A_NE, A_AND, A_OR,
  A_MIN, A_MAX, A_IDIV0, A_IMOD0, A_TDIV0, A_TMOD0, A_SELECT, A_COUNT
};
// Operand kinds.
enum : uint32_t { K_ACC = 0, K_TEMP = 1, K_INPUT = 2, K_CONST = 3 };
// x: op | swap<<8 | k1<<9 | k2<<11 | k3<<13 | i3<<16 ; y: i1 | i2<<16
__device__ __forceinline__ uint2 a_instr(uint32_t op, bool swap, uint32_t k1, uint32_t i1, uint32_t k2 = 0,
                                         uint32_t i2 = 0, uint32_t k3 = 0, uint32_t i3 = 0) {
  return make_uint2(op | (uint32_t(swap) << 8) | (k1 << 9) | (k2 << 11) | (k3 << 13) | (i3 << 16), i1 | (i2 << 16));
}

constexpr int kMaxLowerNodes = 256;

// A row to lower: node words and prefix-ordered constants.
struct LRow {
  const uint64_t* node;
  const int64_t* cval;
  int n, nc;
};

// What lowering reads of an admitted search: the expression table, the
// traversal table, the evaluator inputs (the preset locals), the phase's
// result type and the fuel of the appended RETURN.
struct LowerView {
  const gagp_expression* ex;
  const RegionInfo* regions;
  int n_ex, n_regions;
  int local_count;
  const int32_t* local_types;
  int slot_type;
  uint32_t return_fuel;
};
__host__ __device__ inline LowerView lower_view(const SearchDesc& s) {
  return LowerView{s.ex, s.regions, s.n_ex, s.n_regions, s.local_count, s.local_types, s.slot_type, s.return_fuel};
}

// Shape of a lowered program.
struct LowerResult {
  int code;         // instructions: the main code, its appended RETURN, then any region records and phase code
  int constants;    // constant pool entries
  int locals;       // inputs + temporaries
  int stack_bound;  // deepest value stack
  int main;         // instructions of the main code with its RETURN (the records start here)
  int main_constants;  // constants of the main code (the phases' follow)
};

// Bounded regions of one program, in completion order (the reference's
// RegionRecord, phase_compile.cuh:236-238): the table entry, the caller
// slot of each capture, the node range of each phase subtree and the row
// constant index where each phase's constants start.
constexpr int kMaxRegions = 4;   // kPhaseMaxRegions
constexpr int kRegionRecord = 0xFF;
struct RegionRecords {
  int count;
  struct {
    int info, captures[8], bounds[5], consts[4];
  } r[kMaxRegions];
};

constexpr int kMaxStack = 64;     // MAX_STACK (cpp/include/gagp/runtime/gpu/constants_gpu.hpp:9)
constexpr int kLowerLocals = 64;  // phase compiler local capacity
constexpr int kLowerWalks = 8;    // open traversals on one lowering path (kPhaseWalks)
constexpr int kLowerBinders = 16; // lexical binder numbers (kPhaseBinders)
constexpr int kLowerLets = 16;     // open lets (kPhaseLets)
constexpr int kLowerLoops = 16;    // open for_range loops (kPhaseLoops)
// instruction flags (DINSTR_HAS_A / DINSTR_HAS_B); bit 2 marks a Bool
// constant, whose tag the reference keeps in its constant Value
constexpr int kHasA = 1, kHasB = 2, kBoolConst = 4;

// Reference bytecode of a whole-program value phase: compile_phase_tree
// (cpp/src/evolution/repro/gpu/device/phase_compile.cuh:207-895) for the
// node kinds this engine admits -- constants, inputs, operations, value
// ifs, and/or, lets, bound reads and forward or reverse traversals without a
// fuel profile -- followed by the RETURN that patch_whole_program appends
// (phase_layout.hpp:476-500).  Instructions are 5 ints (op, flags, a, b,
// fuel) and the constants int64 payloads (flags bit 2: a Bool).  The
// emitted code, constant numbering, temporaries and their LIFO reuse
// follow the reference step by step, so the program consumes the same fuel
// and fails the same way on every case.  Returns the instruction count, or
// -1 when the compiler rejects the row (or it exceeds a capacity).
//
// Without a fuel profile none of the traversal's operands is aliased and no
// event is uncharged, so the reference's binder facts and analysed ifs
// (which only decide aliases and uncharged checks) never change the output
// and are not kept here.
//
// `regions` null: a bounded region's phase (Regions=false in the
// reference): the value is left on the stack with no RETURN, and no region
// may occur.  Otherwise the main code, whose bounded regions are recorded
// there (the operands lowered in place, the phase subtrees set aside).
__host__ __device__ __noinline__ int lower_code(const LowerView& v, const uint64_t* node, const int64_t* cval, int n, int nc,
                                          int32_t* code, int code_cap, int64_t* consts, int const_cap,
                                          LowerResult* result, RegionRecords* regions) {
  struct Frame {
    int node, base_stack, first_jump, second_jump, seen;
    int8_t args[3];
  };
  // one open traversal: its table entry, the first live temporary it owns,
  // its storage slots, the loop head and the exit jump to patch, and the
  // binder slots its body shadows
  struct Walk {
    int info, live_begin, xs, start, begin, limit, length, counter, element, index, state, loop_head, done_jump;
    int8_t saved_slot[3], saved_type[3];
  };
  // one open let (phase_compile.cuh:263): its binder, its slot, the first
  // live temporary it owns and the binder slot its body shadows
  struct Let {
    int binder, slot, live_begin;
    int8_t saved_slot, saved_type;
  };
  Frame frames[64];
  Walk walks[kLowerWalks];
  Let lets[kLowerLets];
  int let_depth = 0;
  // one open for_range (phase_compile.cuh:251-252): its bound and counter
  // slots, the loop head, the exit jump to patch, the constant 1's index
  // and the first live temporary it owns
  struct Loop {
    int bound, counter, head, end_jump, one, live_begin;
  };
  Loop loops[kLowerLoops];
  int loop_depth = 0;
  // grammar locals get a slot on first use, after the inputs, and keep it
  unsigned named_mask = 0;
  int8_t named[kNamedLocals];
  int8_t env_slot[kLowerBinders], env_type[kLowerBinders];
  int8_t live[kLowerLocals], freed[kLowerLocals] = {};
  for (int i = 0; i < kLowerBinders; ++i) { env_slot[i] = -1; env_type[i] = GAGP_TAG_INVALID; }
  int depth = 0, walk_depth = 0, cursor = 0, count = 0, nconst = 0, stack = 0, stack_bound = 0, row_const = 0;
  int total_locals = v.local_count, live_count = 0, free_count = 0;
  int completed = GAGP_TAG_INVALID;
  bool have_value = false;
  const bool statements = is_statement_tag(v.slot_type);
  if (n <= 0 || n > kCapacity || v.local_count < 0 || v.local_count > kLowerLocals) return -1;
  // a statement program reads only definitely assigned grammar locals
  if (statements && !locals_defined(n, [&](int i) {
        const int o = w_origin(node[i]);
        if (o < 0 || o >= v.n_ex) return StatementNode{-1, 0, w_arity(node[i]), 0};
        const gagp_expression& x = v.ex[o];
        return StatementNode{x.kind == EK_OPERATION ? x.node_kind : -1, x.operand, w_arity(node[i]), x.type};
      }))
    return -1;
  auto emit = [&](int op, unsigned fuel, int a, int b, int flags) -> bool {
    if (count >= code_cap) return false;
    int32_t* x = code + 5 * count++;
    x[0] = op; x[1] = flags; x[2] = a; x[3] = b; x[4] = int32_t(fuel);
    return true;
  };
  auto grow = [&](int by) { stack += by; if (stack > stack_bound) stack_bound = stack; };
  auto add_const = [&](int64_t value) -> int {
    if (nconst >= const_cap) return -1;
    consts[nconst] = value;
    return nconst++;
  };
  // a traversal's own instructions, grouped by source fuel event: with a
  // fuel profile the first instruction of an event carries its charge and
  // the rest none, without one each costs 1 (phase_compile.cuh:422-432)
  bool event_profile = false;
  unsigned event_first = 1;
  int event_count = 0;
  auto event = [&](const RegionInfo& info, int which) {
    event_profile = info.fuel_profile != 0;
    event_first = event_profile ? info.event_cost[which] : 1u;
    event_count = 0;
  };
  auto put = [&](int op, int a, int b, int flags, int delta) -> bool {
    const unsigned fuel = event_profile ? (event_count++ ? 0u : event_first) : 1u;
    if (!emit(op, fuel, a, b, flags)) return false;
    if (delta > 0) grow(delta); else stack += delta;
    return true;
  };
  auto put_load = [&](int slot) { return put(OP_LOAD, slot, 0, kHasA, 1); };
  auto put_store = [&](int slot) { return put(OP_STORE, slot, 0, kHasA, -1); };
  auto put_int = [&](int64_t value) {
    const int index = add_const(value);
    return index >= 0 && put(OP_PUSH_CONST, index, 0, kHasA, 1);
  };
  auto temporary = [&]() -> int {
    int slot;
    if (free_count) slot = freed[--free_count];
    else if (total_locals >= kLowerLocals) return -1;
    else slot = total_locals++;
    live[live_count++] = int8_t(slot);
    return slot;
  };
  // the slot of an assignment target or local read: an input (-1 - its
  // evaluator position) or a grammar local, numbered on first use
  auto variable_slot = [&](int operand) -> int {
    if (operand < 0) return -1 - operand < v.local_count ? -1 - operand : -1;
    if (operand >= kNamedLocals) return -1;
    if (!((named_mask >> operand) & 1u)) {
      if (total_locals >= kLowerLocals) return -1;
      named[operand] = int8_t(total_locals++);
      named_mask |= 1u << operand;
    }
    return named[operand];
  };
  // the operands are on the stack: resolve the captures, set the phase
  // subtrees aside and emit BOUNDED_REGION (finish_region,
  // phase_compile.cuh:289-319)
  auto finish_region = [&](const gagp_expression& e) -> bool {
    if (!regions || regions->count == kMaxRegions) return false;
    const RegionInfo& info = v.regions[e.operand];
    auto& rec = regions->r[regions->count];
    rec.info = e.operand;
    for (int c = 0; c < info.captures; ++c) {
      const int target = info.capture_target[c];
      int slot = -1;
      if (info.capture_kind[c] == 0) slot = target >= 0 ? variable_slot(-1 - target) : -1;
      else if (info.capture_kind[c] == 1) slot = variable_slot(target);
      else if (target >= 0 && target < kLowerBinders) slot = env_slot[target];
      if (slot < 0) return false;
      rec.captures[c] = slot;
    }
    for (int p = 0; p < info.phases; ++p) {
      rec.bounds[p] = cursor;
      rec.consts[p] = row_const;
      int pending = 1;
      while (pending) {
        if (cursor >= n) return false;
        const uint64_t w = node[cursor++];
        row_const += w_const(w);
        pending += w_arity(w) - 1;
      }
    }
    rec.bounds[info.phases] = cursor;
    if (!emit(OP_BOUNDED_REGION, e.fuel, regions->count, 0, kHasA)) return false;
    stack -= info.operands;
    grow(1);
    ++regions->count;
    completed = e.type;
    return true;
  };
  auto subtree_end = [&](int i) -> int {
    int pending = 1;
    while (pending) {
      if (i < 0 || i >= n) return -1;
      pending += w_arity(node[i++]) - 1;
    }
    return i;
  };
  // compile_region_prefix of a traversal after its child `c` completed
  // (phase_compile.cuh:409-516, every event charged and nothing aliased)
  auto walk_after = [&](Walk& w, int c) -> bool {
    const RegionInfo& info = v.regions[w.info];
    const bool reverse = info.traversal == 2;
    const int arity = info.arity;
    if (c == 0) {
      event(info, 4);                                                      // StoreSequence
      if (!put_store(w.xs)) return false;
    }
    if (c == 1) {
      event(info, 5);                                                      // StoreStart
      if (!put_store(w.start)) return false;
      event(info, 8);                                                      // CheckStart
      if (!put_load(w.start) || !put(OP_CHECK_INT, 0, 0, 0, 0) || !put_store(w.start)) return false;
      event(info, 11);                                                     // ObserveSequence
      if (!put_load(w.xs) || !put(OP_CALL_BUILTIN, B_LEN, 1, kHasA | kHasB, 0) || !put_store(w.length))
        return false;
      event(info, 14);                                                     // SetBegin
      if (!put_int(0) || !put_store(w.begin)) return false;
      event(info, 15);                                                     // SetEnd
      if (!put_load(w.length) || !put_store(w.limit)) return false;
    }
    if (c == arity - 2) {
      event(info, 16);                                                     // InitializeState
      if (!put_store(w.state)) return false;
      event(info, 17);                                                     // InitializeCursor
      if (!(reverse ? put_load(w.limit) : put_load(w.begin))) return false;
      if (reverse && (!put_int(1) || !put(OP_SUB, 0, 0, 0, -1))) return false;
      if (!put_store(w.counter)) return false;
      w.loop_head = count;
      event(info, 18);                                                     // TestCursor
      if (!put_load(w.counter) || !(reverse ? put_load(w.begin) : put_load(w.limit)) ||
          !put(reverse ? OP_GE : OP_LT, 0, 0, 0, -1))
        return false;
      w.done_jump = count;
      if (!put(OP_JMP_IF_FALSE, 0, 0, kHasA, -1)) return false;
      event(info, 19);                                                     // ReadElement
      if (!put_load(w.xs) || !put_load(w.counter) || !put(OP_CALL_BUILTIN, B_INDEX, 2, kHasA | kHasB, -1))
        return false;
      event(info, 20);                                                     // BindElement
      if (!put_store(w.element)) return false;
      event(info, 21);                                                     // ComputeIndex
      if (!put_load(w.start) || !put_load(w.counter) || !put(OP_ADD, 0, 0, 0, -1) || !put_store(w.index))
        return false;
      const int slots[3] = {w.element, w.index, w.state};
      for (int k = 0; k < 3; ++k) {
        const int b = info.binders[k];
        w.saved_slot[k] = env_slot[b];
        w.saved_type[k] = env_type[b];
        env_slot[b] = int8_t(slots[k]);
        env_type[b] = info.binding_types[k];
      }
    }
    if (c == arity - 1) {
      for (int k = 2; k >= 0; --k) {
        const int b = info.binders[k];
        env_slot[b] = w.saved_slot[k];
        env_type[b] = w.saved_type[k];
      }
      event(info, 22);                                                     // UpdateState
      if (!put_store(w.state)) return false;
      event(info, 23);                                                     // AdvanceCursor
      if (!put_load(w.counter) || !put_int(1) || !put(reverse ? OP_SUB : OP_ADD, 0, 0, 0, -1) ||
          !put_store(w.counter))
        return false;
      event(info, 24);                                                     // Repeat
      if (!put(OP_JMP, w.loop_head, 0, kHasA, 0)) return false;
      code[5 * w.done_jump + 2] = count;
      event(info, 25);                                                     // Result
      if (!put_load(w.state)) return false;
    }
    event_profile = false;
    return true;
  };
  for (;;) {
    if (!have_value) {
      if (cursor >= n) return -1;
      const int index = cursor++;
      const int origin = w_origin(node[index]);
      if (origin < 0 || origin >= v.n_ex) return -1;
      const gagp_expression& e = v.ex[origin];
      if (e.node_kind == TK_CONSTANT) {
        // constants are Int payloads in prefix order, the order the cursor
        // visits the constant nodes in
        if (row_const >= nc) return -1;
        const int k = add_const(cval[row_const++]);
        if (k < 0 || !emit(OP_PUSH_CONST, e.fuel, k, 0, kHasA)) return -1;
        grow(1);
        completed = GAGP_TAG_INT;
        have_value = true;
      } else if (e.node_kind == TK_BOUND && e.operand >= 0 && e.operand < kLowerBinders && env_slot[e.operand] >= 0) {
        completed = env_type[e.operand];
        if (e.type != GAGP_TAG_INVALID && e.type != completed) return -1;
        if (!emit(OP_LOAD, e.fuel, env_slot[e.operand], 0, kHasA)) return -1;
        grow(1);
        have_value = true;
      } else if (e.node_kind == TK_LOCAL || e.node_kind == TK_BOUND) {
        if (e.operand < 0 || e.operand >= v.local_count) return -1;
        if (!emit(OP_LOAD, e.fuel, e.operand, 0, kHasA)) return -1;
        grow(1);
        completed = v.local_types[e.operand];
        have_value = true;
      } else if (e.node_kind == TK_NIL) {
        if (e.arity != 0) return -1;
        completed = kStatementTag;
        have_value = true;
      } else if (e.node_kind == TK_VAR) {
        // a grammar local's read
        if (e.arity != 0 || e.operand < 0 || e.type == GAGP_TAG_INVALID || is_statement_tag(e.type)) return -1;
        const int slot = variable_slot(e.operand);
        if (slot < 0 || !emit(OP_LOAD, e.fuel, slot, 0, kHasA)) return -1;
        grow(1);
        completed = e.type;
        have_value = true;
      } else if (e.node_kind == TK_REGION) {
        // a bounded region (phase_compile.cuh:652-666): operands first, its
        // phases set aside when the last operand completes
        if (!regions || e.operand < 0 || e.operand >= v.n_regions) return -1;
        const RegionInfo& info = v.regions[e.operand];
        if (info.traversal != 0 || info.phases < 1 || e.arity != info.operands + info.phases || e.arity > 8) return -1;
        if (info.operands == 0) {
          if (!finish_region(e)) return -1;
          have_value = true;
        } else {
          if (depth == 64) return -1;
          frames[depth++] = Frame{index, stack, -1, -1, 0, {0, 0, 0}};
          continue;
        }
      } else if (e.node_kind == TK_TRAVERSE) {
        if (e.operand < 0 || e.operand >= v.n_regions) return -1;
        const RegionInfo& info = v.regions[e.operand];
        if ((info.traversal != 1 && info.traversal != 2) || info.ranged || e.arity != info.arity) return -1;
        for (int k = 0; k < 3; ++k)
          if (info.binders[k] < 0 || info.binders[k] >= kLowerBinders) return -1;
        if (depth == 64 || walk_depth == kLowerWalks) return -1;
        if (subtree_end(index) < 0) return -1;
        Walk& w = walks[walk_depth++];
        w.info = e.operand;
        w.live_begin = live_count;
        // the native temporary order
        w.xs = temporary();
        w.start = temporary();
        w.begin = temporary();
        w.limit = temporary();
        w.length = temporary();
        w.counter = temporary();
        w.element = temporary();
        w.index = temporary();
        w.state = temporary();
        if (w.xs < 0 || w.start < 0 || w.begin < 0 || w.limit < 0 || w.length < 0 || w.counter < 0 ||
            w.element < 0 || w.index < 0 || w.state < 0)
          return -1;
        frames[depth++] = Frame{index, stack, -1, -1, 0, {0, 0, 0}};
        continue;
      } else if (e.node_kind == TK_LET) {
        // the value's slot is taken before the value's own temporaries
        if (e.arity != 2 || depth == 64 || e.operand < 0 || e.operand >= kLowerBinders) return -1;
        if (let_depth == kLowerLets) return -1;
        Let& l = lets[let_depth++];
        l.binder = e.operand;
        l.live_begin = live_count;
        l.slot = temporary();
        if (l.slot < 0) return -1;
        frames[depth++] = Frame{index, stack, -1, -1, 0, {0, 0, 0}};
        continue;
      } else {
        if (e.arity < 1 || e.arity > 3 || depth == 64) return -1;
        if (e.node_kind == TK_IF && e.arity != 3) return -1;
        if ((e.node_kind == TK_AND || e.node_kind == TK_OR) && e.arity != 2) return -1;
        if ((e.node_kind == TK_PROGRAM || e.node_kind == TK_ASSIGN || e.node_kind == TK_RETURN) && e.arity != 1)
          return -1;
        if ((e.node_kind == TK_BLOCK || e.node_kind == TK_FOR_RANGE) && e.arity != 2) return -1;
        if (e.node_kind != TK_OPERATION && e.node_kind != TK_IF && e.node_kind != TK_AND && e.node_kind != TK_OR &&
            e.node_kind != TK_PROGRAM && e.node_kind != TK_BLOCK && e.node_kind != TK_ASSIGN &&
            e.node_kind != TK_RETURN && e.node_kind != TK_FOR_RANGE)
          return -1;
        if (e.node_kind == TK_FOR_RANGE) {
          // the bound's slot precedes the bound expression's own temporaries
          if (loop_depth == kLowerLoops) return -1;
          Loop& l = loops[loop_depth++];
          l.live_begin = live_count;
          l.bound = temporary();
          if (l.bound < 0) return -1;
        }
        frames[depth++] = Frame{index, stack, -1, -1, 0, {0, 0, 0}};
        continue;
      }
    }
    if (depth == 0) {
      // a value phase leaves its value for the appended RETURN; a statement
      // program returns by its own RETURNs and has no terminator
      // (patch_whole_program, phase_layout.hpp:494-496)
      if (cursor != n || stack != (statements ? 0 : 1) || completed != v.slot_type || stack_bound > kMaxStack)
        return -1;
      if (regions && !statements && (stack_bound < 1 || !emit(OP_RETURN, v.return_fuel, 0, 0, 0))) return -1;
      result->code = count;
      result->main = count;
      result->constants = nconst;
      result->locals = total_locals;
      result->stack_bound = stack_bound;
      return count;
    }
    Frame& f = frames[depth - 1];
    const gagp_expression& e = v.ex[w_origin(node[f.node])];
    if (f.seen < 3) f.args[f.seen] = int8_t(completed);
    ++f.seen;
    if (e.node_kind == TK_TRAVERSE) {
      Walk& w = walks[walk_depth - 1];
      const RegionInfo& info = v.regions[w.info];
      if (completed != info.operand_types[f.seen - 1] || !walk_after(w, f.seen - 1)) return -1;
      if (f.seen < e.arity) { have_value = false; continue; }
      while (live_count > w.live_begin) freed[free_count++] = live[--live_count];
      --walk_depth;
      completed = info.result_type;
      --depth;
      continue;
    }
    if (e.node_kind == TK_LET) {
      Let& l = lets[let_depth - 1];
      if (f.seen == 1) {
        // store the value and bind it for the body
        if (!emit(OP_STORE, e.fuel, l.slot, 0, kHasA)) return -1;
        stack = f.base_stack;
        l.saved_slot = env_slot[l.binder];
        l.saved_type = env_type[l.binder];
        env_slot[l.binder] = int8_t(l.slot);
        env_type[l.binder] = int8_t(completed);
        have_value = false;
        continue;
      }
      // the body's value is the let's
      if (e.type != GAGP_TAG_INVALID && e.type != completed) return -1;
      env_slot[l.binder] = l.saved_slot;
      env_type[l.binder] = l.saved_type;
      while (live_count > l.live_begin) freed[free_count++] = live[--live_count];
      --let_depth;
      --depth;
      continue;
    }
    if (e.node_kind == TK_REGION) {
      const RegionInfo& info = v.regions[e.operand];
      if (completed != info.operand_types[f.seen - 1]) return -1;
      if (f.seen < info.operands) { have_value = false; continue; }
      if (!finish_region(e)) return -1;
      --depth;
      continue;
    }
    const bool branch = e.node_kind == TK_IF || e.node_kind == TK_AND || e.node_kind == TK_OR;
    if (branch && f.seen == 1) {
      if (completed != GAGP_TAG_BOOL) return -1;
      f.first_jump = count;
      if (!emit(e.node_kind == TK_OR ? OP_JMP_IF_TRUE : OP_JMP_IF_FALSE, e.fuel, 0, 0, kHasA)) return -1;
      --stack;
    } else if (e.node_kind == TK_IF && f.seen == 2) {
      f.second_jump = count;
      if (!emit(OP_JMP, e.merge_fuel, 0, 0, kHasA)) return -1;
      code[5 * f.first_jump + 2] = count;
      stack = f.base_stack;
    }
    if (e.node_kind == TK_FOR_RANGE && f.seen == 1) {
      // for_range (phase_compile.cuh:767-807): store the bound, fail on a
      // bound that is not an Int or is negative (NEG of true, a type
      // error), then count from zero, copying the counter into the named
      // target at the top of every pass
      Loop& l = loops[loop_depth - 1];
      if (is_statement_tag(completed)) return -1;
      if (!emit(OP_STORE, 1, l.bound, 0, kHasA)) return -1;
      stack = f.base_stack;
      if (!emit(OP_LOAD, 1, l.bound, 0, kHasA)) return -1;
      grow(1);
      if (!emit(OP_CALL_BUILTIN, 1, B_IS_INT, 1, kHasA | kHasB)) return -1;
      const int bad = count;
      if (!emit(OP_JMP_IF_FALSE, 1, 0, 0, kHasA)) return -1;
      stack = f.base_stack;
      if (!emit(OP_LOAD, 1, l.bound, 0, kHasA)) return -1;
      grow(1);
      const int zero_test = add_const(0);
      if (zero_test < 0 || !emit(OP_PUSH_CONST, 1, zero_test, 0, kHasA)) return -1;
      grow(1);
      if (!emit(OP_LT, 1, 0, 0, 0)) return -1;
      const int valid = count;
      if (!emit(OP_JMP_IF_FALSE, 1, 0, 0, kHasA)) return -1;
      stack = f.base_stack;
      code[5 * bad + 2] = count;
      const int truth = add_const(1);
      if (truth < 0 || !emit(OP_PUSH_CONST, 1, truth, 0, kHasA | kBoolConst)) return -1;
      grow(1);
      if (!emit(OP_NEG, 1, 0, 0, 0)) return -1;
      code[5 * valid + 2] = count;
      stack = f.base_stack;
      const int zero = add_const(0);
      l.one = add_const(1);
      if (zero < 0 || l.one < 0) return -1;
      l.counter = temporary();
      const int user = variable_slot(e.operand);
      if (l.counter < 0 || user < 0) return -1;
      if (!emit(OP_PUSH_CONST, 1, zero, 0, kHasA)) return -1;
      grow(1);
      if (!emit(OP_STORE, 1, l.counter, 0, kHasA)) return -1;
      stack = f.base_stack;
      l.head = count;
      if (!emit(OP_LOAD, 1, l.counter, 0, kHasA) || !emit(OP_LOAD, 1, l.bound, 0, kHasA)) return -1;
      grow(2);
      if (!emit(OP_LT, 1, 0, 0, 0)) return -1;
      l.end_jump = count;
      if (!emit(OP_JMP_IF_FALSE, 1, 0, 0, kHasA)) return -1;
      stack = f.base_stack;
      if (!emit(OP_LOAD, 1, l.counter, 0, kHasA)) return -1;
      grow(1);
      if (!emit(OP_STORE, 1, user, 0, kHasA)) return -1;
      stack = f.base_stack;
    }
    if (f.seen < e.arity) { have_value = false; continue; }
    if (e.node_kind == TK_IF) {
      if (f.args[1] != f.args[2]) return -1;
      code[5 * f.second_jump + 2] = count;
    } else if (e.node_kind == TK_PROGRAM) {
      if (!is_statement_tag(completed)) return -1;
    } else if (e.node_kind == TK_BLOCK) {
      if (!is_statement_tag(f.args[0]) || !is_statement_tag(f.args[1])) return -1;
    } else if (e.node_kind == TK_ASSIGN || e.node_kind == TK_RETURN) {
      // the grammar fixes the stored or returned type; an assigned grammar
      // local gets its slot after its value's temporaries
      if (completed != e.type || is_statement_tag(completed)) return -1;
      if (e.node_kind == TK_ASSIGN) {
        const int slot = variable_slot(e.operand);
        if (slot < 0 || !emit(OP_STORE, e.fuel, slot, 0, kHasA)) return -1;
      } else if (!emit(OP_RETURN, e.fuel, 0, 0, 0)) {
        return -1;
      }
      stack = f.base_stack;
      completed = kStatementTag;
    } else if (e.node_kind == TK_FOR_RANGE) {
      if (!is_statement_tag(completed)) return -1;
      const Loop l = loops[--loop_depth];
      if (!emit(OP_LOAD, 1, l.counter, 0, kHasA) || !emit(OP_PUSH_CONST, 1, l.one, 0, kHasA)) return -1;
      grow(2);
      if (!emit(OP_ADD, 1, 0, 0, 0) || !emit(OP_STORE, 1, l.counter, 0, kHasA) || !emit(OP_JMP, 1, l.head, 0, kHasA))
        return -1;
      code[5 * l.end_jump + 2] = count;
      stack = f.base_stack;
      while (live_count > l.live_begin) freed[free_count++] = live[--live_count];
    } else if (e.node_kind == TK_AND || e.node_kind == TK_OR) {
      if (completed != GAGP_TAG_BOOL) return -1;
      if (!emit(OP_NOT, e.fuel, 0, 0, 0) || !emit(OP_NOT, e.fuel, 0, 0, 0)) return -1;
      const int finish = count;
      if (!emit(OP_JMP, e.fuel, 0, 0, kHasA)) return -1;
      code[5 * f.first_jump + 2] = count;
      stack = f.base_stack;
      const int k = add_const(e.node_kind == TK_OR ? 1 : 0);
      if (k < 0 || !emit(OP_PUSH_CONST, e.fuel, k, 0, kHasA | kBoolConst)) return -1;
      grow(1);
      code[5 * finish + 2] = count;
      completed = GAGP_TAG_BOOL;
    } else {
      // the typed grammar fixes an operation's result type
      completed = e.type;
      if (e.opcode == OP_CALL_BUILTIN) {
        if (!emit(e.opcode, e.fuel, e.operand, e.arity, kHasA | kHasB)) return -1;
      } else if (!emit(e.opcode, e.fuel, 0, 0, 0)) {
        return -1;
      }
      stack -= e.arity - 1;
    }
    --depth;
  }
}

// Reference bytecode of a whole program: the main code (lower_code) with
// its RETURN, then, for each bounded region in completion order, the
// reference's records (phase_compile.cuh:889-912): a header (fuel: the
// capture count, a: the table entry, b: the phase count), one record per
// capture (a: its caller slot), and per phase a header (a: its
// instructions, b: its constants, fuel: its locals, bit 16 when it reads a
// binder or a let) followed by the phase's own code, lowered with its
// bindings as its first locals.  Phase constants follow the main ones in
// the pool.  Returns the instruction count or -1.
__host__ __device__ inline int lower_program(const LowerView& v, const uint64_t* node, const int64_t* cval, int n,
                                             int nc, int32_t* code, int code_cap, int64_t* consts, int const_cap,
                                             LowerResult* result) {
  RegionRecords rec;
  rec.count = 0;
  int count = lower_code(v, node, cval, n, nc, code, code_cap, consts, const_cap, result, &rec);
  if (count >= 0) result->main_constants = result->constants;
  if (count < 0 || !rec.count) return count;
  int nconst = result->constants;
  auto emit = [&](int fuel, int a, int b) -> bool {
    if (count >= code_cap) return false;
    int32_t* x = code + 5 * count++;
    x[0] = kRegionRecord; x[1] = 0; x[2] = a; x[3] = b; x[4] = fuel;
    return true;
  };
  for (int r = 0; r < rec.count; ++r) {
    const RegionInfo& info = v.regions[rec.r[r].info];
    if (!emit(info.captures, rec.r[r].info, info.phases)) return -1;
    for (int c = 0; c < info.captures; ++c)
      if (!emit(0, rec.r[r].captures[c], 0)) return -1;
    for (int p = 0; p < info.phases; ++p) {
      const int header = count;
      if (!emit(0, 0, 0)) return -1;
      int32_t types[8];
      for (int b = 0; b < info.phase_bindings[p]; ++b) types[b] = info.phase_binding_types[p][b];
      LowerView pv = v;
      pv.local_count = info.phase_bindings[p];
      pv.local_types = types;
      pv.slot_type = info.phase_type[p];
      const int begin = rec.r[r].bounds[p], end = rec.r[r].bounds[p + 1];
      LowerResult pr{};
      const int pc = lower_code(pv, node + begin, cval + rec.r[r].consts[p], end - begin, nc - rec.r[r].consts[p],
                                code + 5 * count, code_cap - count, consts + nconst, const_cap - nconst, &pr, nullptr);
      if (pc < 0) return -1;
      // a phase that reads a binding or binds a let keeps its fuel table
      bool general = false;
      for (int i = begin; i < end; ++i) {
        const int nk = v.ex[w_origin(node[i])].node_kind;
        general |= nk == TK_BOUND || nk == TK_LET;
      }
      code[5 * header + 2] = pc;
      code[5 * header + 3] = pr.constants;
      code[5 * header + 4] = pr.locals | (general ? 1 << 16 : 0);
      count += pc;
      nconst += pr.constants;
      if (pr.stack_bound > result->stack_bound) result->stack_bound = pr.stack_bound;
    }
  }
  result->code = count;
  result->constants = nconst;
  return count;
}

// Per-warp shared memory of the accumulator lowering: per-node tables
// filled and read by the whole warp.
constexpr uint8_t kLeafOp = 0xff;
struct LowerScratch {
  uint8_t aop[kMaxLowerNodes];    // accumulator op (A_COUNT: not total), kLeafOp for leaves
  uint8_t arity[kMaxLowerNodes];
  int8_t need[kMaxLowerNodes];    // Sethi-Ullman temporaries of the subtree (-1: not yet known)
  uint8_t order[kMaxLowerNodes];  // evaluation order of the non-leaf children: 3 x 2 bits | count << 6
  int16_t end[kMaxLowerNodes];    // one past the subtree
  int16_t size[kMaxLowerNodes];   // code words of the subtree
  int16_t start[kMaxLowerNodes];  // open slots before the node, then the subtree's first code word
  int16_t temp_base[kMaxLowerNodes];
  int16_t depth[kMaxLowerNodes];  // non-leaf depth (root 1)
  int16_t anc[kMaxLowerNodes];    // pointer jumping: the ancestor the sums reach (-1: the root)
  uint32_t leaf[kMaxLowerNodes];  // leaves: operand kind << 16 | index
};

// Warp-parallel Sethi-Ullman code generation for lower_accumulator_warp.
// Same code, failure conditions and temporaries as evaluating the tree with
// an explicit stack (children in decreasing need, every non-leaf child but
// the last spilled; a spill past kMaxTemps, code past code_cap or non-leaf
// nesting past 64 frames fails), but computed with warp scans and
// level-synchronous sweeps: subtree ends from the open-slot prefix sums,
// needs and code sizes bottom-up, code positions and temporaries top-down,
// and every node writing its own instructions.  All lanes return the same.
__device__ inline int lower_accumulator_emit(LowerScratch& m, int n, uint2* code, int code_cap, int* temps_out) {
  const int lane = threadIdx.x & 31;
  // open slots before node i: 1 + sum over earlier nodes of (arity - 1)
  int carry = 1;
  for (int base = 0; base < n; base += 32) {
    const int i = base + lane;
    const int v = i < n ? int(m.arity[i]) - 1 : 0;
    int incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    if (i < n) m.start[i] = int16_t(carry + incl - v);
    carry += __shfl_sync(kFull, incl, 31);
  }
  __syncwarp();
  // a subtree ends at the first later node with fewer open slots: for 32
  // nodes at a time, every lane holds one later node's slot count and each
  // node's question is answered by one ballot per chunk
  for (int base = 0; base < n; base += 32) {
    const int i = base + lane;
    const int r = i < n ? m.start[i] : 0;
    int e = n;
    bool found = i >= n;
    for (int cb = base; cb < n && __any_sync(kFull, !found); cb += 32) {
      const int j = cb + lane;
      const int slots = j < n ? m.start[j] : 0x7fffffff;
      for (int q = 0; q < 32; ++q) {
        const int rq = __shfl_sync(kFull, r, q);
        const unsigned hit = __ballot_sync(kFull, j > base + q && slots < rq);
        if (lane == q && !found && hit) {
          e = cb + __ffs(hit) - 1;
          found = true;
        }
      }
    }
    if (i < n) m.end[i] = int16_t(e);
  }
  __syncwarp();
  if (carry != 0 || m.end[0] != n) return -1;
  // ---- bottom-up: need, size, evaluation order
  uint32_t pend = 0;  // bit k: node lane + 32 k not yet computed
  for (int k = 0; lane + 32 * k < n; ++k) {
    const int i = lane + 32 * k;
    m.anc[i] = -2;  // no parent yet
    if (m.arity[i] == 0) { m.need[i] = 0; m.size[i] = 0; }
    else { m.need[i] = -1; pend |= 1u << k; }
  }
  __syncwarp();
  bool fail = false;
  while (__any_sync(kFull, pend != 0)) {
    uint32_t ready = 0;
    for (uint32_t b = pend; b; b &= b - 1) {
      const int k = __ffs(b) - 1, i = lane + 32 * k, a = m.arity[i];
      bool ok = true;
      for (int x = 0, c = i + 1; x < a; ++x) {
        if (c >= n) { ok = false; fail = true; break; }
        ok &= m.need[c] >= 0;
        c = m.end[c];
      }
      if (ok) ready |= 1u << k;
    }
    __syncwarp();
    if (!__any_sync(kFull, ready != 0) || __any_sync(kFull, fail)) { fail = true; break; }
    for (uint32_t b = ready; b; b &= b - 1) {
      const int k = __ffs(b) - 1, i = lane + 32 * k, a = m.arity[i];
      // the non-leaf children as (need << 2 | position), in child order, in
      // registers (arity <= 3)
      const int c0 = i + 1, c1 = a > 1 ? m.end[c0] : 0, c2 = a > 2 ? m.end[c1] : 0;
      int e0 = 0, e1 = 0, e2 = 0, nonleaf = 0, sz = 0;
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        const int c = x == 0 ? c0 : x == 1 ? c1 : c2;
        if (x < a && m.end[c] - c > 1) {
          const int v = (int(m.need[c]) << 2) | x;
          if (nonleaf == 0) e0 = v; else if (nonleaf == 1) e1 = v; else e2 = v;
          ++nonleaf;
          sz += m.size[c];
        }
      }
      // the explicit-stack evaluator's exchange sort by decreasing need:
      // pairs (0,1), (0,2), (1,2), swapping when the later need is larger
      auto exchange = [](int& p, int& q) {
        if ((q >> 2) > (p >> 2)) { const int t = p; p = q; q = t; }
      };
      if (nonleaf > 1) exchange(e0, e1);
      if (nonleaf > 2) { exchange(e0, e2); exchange(e1, e2); }
      int mx = 0;
      if (nonleaf > 0) mx = max(mx, e0 >> 2);
      if (nonleaf > 1) mx = max(mx, (e1 >> 2) + 1);
      if (nonleaf > 2) mx = max(mx, (e2 >> 2) + 2);
      // own words: unary MOV + op when its child is a leaf; binary MOV + op
      // when both children are leaves; otherwise one word
      const bool leaf0 = m.end[c0] - c0 == 1;
      const int own = a == 1 ? (leaf0 ? 2 : 1) : a == 2 ? (nonleaf == 0 ? 2 : 1) : 1;
      m.size[i] = int16_t(min(sz + max(nonleaf - 1, 0) + own, 32767));
      m.order[i] = uint8_t((nonleaf << 6) | (nonleaf > 0 ? e0 & 3 : 0) | (nonleaf > 1 ? (e1 & 3) << 2 : 0) |
                           (nonleaf > 2 ? (e2 & 3) << 4 : 0));
      m.need[i] = int8_t(min(mx, 127));
    }
    pend &= ~ready;
    __syncwarp();
  }
  if (__any_sync(kFull, fail)) return -1;
  if (m.need[0] > kMaxTemps) return -1;
  *temps_out = m.need[0];
  if (m.end[0] == 1) {  // a leaf root
    if (code_cap < 1) return -1;
    if (lane == 0) code[0] = a_instr(A_MOV, false, m.leaf[0] >> 16, m.leaf[0] & 0xffffu);
    __syncwarp();
    return 1;
  }
  const int total = m.size[0];
  if (total > code_cap) return -1;
  // ---- top-down: code positions, temporaries and depth.  Each is a sum
  // along the path from the root (a child's code starts after its earlier
  // evaluated siblings' code and spills, its temporaries after its
  // position's, one level deeper), so every non-leaf node first records its
  // children's offsets from itself, then pointer jumping adds up the paths
  // in about log2(depth) rounds instead of one sweep per level.
  if (lane == 0) { m.start[0] = 0; m.temp_base[0] = 0; m.depth[0] = 1; m.anc[0] = -1; }
  for (int i = lane; i < n; i += 32) {
    const int a = m.arity[i];
    if (!a) continue;
    const int ob = m.order[i], count = ob >> 6;
    const int o0 = ob & 3, o1 = (ob >> 2) & 3, o2 = (ob >> 4) & 3;
    const int c0 = i + 1, c1 = a > 1 ? m.end[c0] : 0, c2 = a > 2 ? m.end[c1] : 0;
    int rel = 0;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      if (q < count) {
        const int x = q == 0 ? o0 : q == 1 ? o1 : o2;
        const int c = x == 0 ? c0 : x == 1 ? c1 : c2;
        rel += q > 0;  // the spill before every child but the first
        m.start[c] = int16_t(rel);
        m.temp_base[c] = int16_t(q);
        m.depth[c] = 1;
        m.anc[c] = int16_t(i);
        rel += m.size[c];
      }
    }
  }
  __syncwarp();
  for (int i = lane; i < n; i += 32)
    if (m.arity[i] && m.anc[i] == -2) fail = true;  // unreachable from the root
  if (__any_sync(kFull, fail)) return -1;
  // pointer jumping: node += ancestor, ancestor = ancestor's ancestor; a read
  // and a write step per node slot, so every read sees a consistent pair
  for (int round = 0; round < 10; ++round) {
    bool more = false;
    for (int base = 0; base < n; base += 32) {
      const int i = base + lane;
      const bool live = i < n && m.arity[i] && m.anc[i] >= 0;
      int s2 = 0, t2 = 0, d2 = 0, a2 = -1;
      if (live) {
        const int a = m.anc[i];
        s2 = m.start[a];
        t2 = m.temp_base[a];
        d2 = m.depth[a];
        a2 = m.anc[a];
      }
      __syncwarp();
      if (live) {
        m.start[i] = int16_t(m.start[i] + s2);
        m.temp_base[i] = int16_t(min(m.temp_base[i] + t2, 32767));
        m.depth[i] = int16_t(min(m.depth[i] + d2, 32767));
        m.anc[i] = int16_t(a2);
        more |= a2 >= 0;
      }
      __syncwarp();
    }
    if (!__any_sync(kFull, more)) break;
  }
  for (int i = lane; i < n; i += 32)
    if (m.arity[i] && m.anc[i] >= 0) fail = true;  // deeper than 2^10 levels: impossible for admitted rows
  // ---- every non-leaf node writes its spills and its own words
  for (int i = lane; i < n; i += 32) {
    const int a = m.arity[i];
    if (!a) continue;
    if (m.depth[i] >= 65) fail = true;  // the 65th nested frame overflows the 64-frame stack
    const int ob = m.order[i], count = ob >> 6, tb = m.temp_base[i];
    const int o0 = ob & 3, o1 = (ob >> 2) & 3, o2 = (ob >> 4) & 3;
    const int c0 = i + 1, c1 = a > 1 ? m.end[c0] : 0, c2 = a > 2 ? m.end[c1] : 0;
    auto child_at = [&](int x) { return x == 0 ? c0 : x == 1 ? c1 : c2; };
    int pos = m.start[i];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      if (q < count) {
        const int c = child_at(q == 0 ? o0 : q == 1 ? o1 : o2);
        if (q > 0) {
          const int temp = tb + q - 1;
          if (temp >= kMaxTemps) fail = true;
          else code[pos] = a_instr(A_SPILL, false, K_TEMP, uint32_t(temp));
          ++pos;
        }
        pos += m.size[c];
      }
    }
    const uint32_t op = m.aop[i];
    const int last = count == 1 ? o0 : count == 2 ? o1 : count == 3 ? o2 : -1;
    uint32_t kind0 = K_ACC, kind1 = K_ACC, kind2 = K_ACC, id0 = 0, id1 = 0, id2 = 0;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      if (x < a) {
        const int c = child_at(x);
        uint32_t kind = K_ACC, id = 0;
        if (m.end[c] - c == 1) {
          const uint32_t leaf = m.leaf[c];
          kind = leaf >> 16;
          id = leaf & 0xffffu;
        } else if (x != last) {
          // a spilled non-leaf child: the temporary of its evaluation slot
          kind = K_TEMP;
          if (count > 1 && o0 == x) id = uint32_t(tb);
          else if (count > 2 && o1 == x) id = uint32_t(tb + 1);
        }
        if (x == 0) { kind0 = kind; id0 = id; }
        else if (x == 1) { kind1 = kind; id1 = id; }
        else { kind2 = kind; id2 = id; }
      }
    }
    if (a == 1) {
      if (kind0 != K_ACC) code[pos++] = a_instr(A_MOV, false, kind0, id0);
      code[pos] = a_instr(op, false, K_ACC, 0);
    } else if (a == 2) {
      if (kind0 != K_ACC && kind1 != K_ACC) {
        code[pos++] = a_instr(A_MOV, false, kind0, id0);
        code[pos] = a_instr(op, false, kind1, id1);
      } else if (kind0 == K_ACC) {
        code[pos] = a_instr(op, false, kind1, id1);
      } else {
        code[pos] = a_instr(op, true, kind0, id0);  // acc = op(first, acc)
      }
    } else {
      code[pos] = a_instr(A_SELECT, false, kind0, id0, kind1, id1, kind2, id2);
    }
  }
  __syncwarp();
  if (__any_sync(kFull, fail)) return -1;
  return total;
}

__host__ __device__ __forceinline__ uint32_t accumulator_op_of(int node_kind, int opcode, int operand) {
  if (node_kind == TK_AND) return A_AND;
  if (node_kind == TK_OR) return A_OR;
  if (node_kind == TK_IF) return A_SELECT;
  if (node_kind != TK_OPERATION) return A_COUNT;
  switch (opcode) {
    case OP_ADD: return A_ADD;
    case OP_SUB: return A_SUB;
    case OP_MUL: return A_MUL;
    case OP_NEG: return A_NEG;
    case OP_NOT: return A_NOT;
    case OP_LT: return A_LT;
    case OP_LE: return A_LE;
    case OP_GT: return A_GT;
    case OP_GE: return A_GE;
    case OP_EQ: return A_EQ;
    case OP_NE: return A_NE;
    case OP_CALL_BUILTIN:
      switch (operand) {
        case B_ABS: return A_ABS;
        case B_MIN: return A_MIN;
        case B_MAX: return A_MAX;
        case B_IDIV0: return A_IDIV0;
        case B_IMOD0: return A_IMOD0;
        case B_TRUNC_DIV0: return A_TDIV0;
        case B_TRUNC_MOD0: return A_TMOD0;
        default: return A_COUNT;
      }
    default: return A_COUNT;  // DIV (Float result), MOD (ZeroDiv error)
  }
}

// Accumulator program of a row, by one warp; returns the instruction count
// (the same on every lane), or -1 when the row needs the general VM.
// *temps_out: temporaries used.  The lanes classify the nodes, number the
// constants, copy the constant pool and bound the bytecode length in
// parallel, then emit the code together (lower_accumulator_emit).
__device__ inline int lower_accumulator_warp(const SearchDesc& s, const uint64_t* node, int n, const int64_t* cval,
                                             int nc, uint2* code, int code_cap, int64_t* kpool, LowerScratch& m,
                                             int* temps_out) {
  const int lane = threadIdx.x & 31;
  if (n <= 0 || n > kMaxLowerNodes || !s.unit_fuel) return -1;
  const ExprInfo* __restrict__ info = s.info;
  bool total = true;
  int bytecode = 0, constants = 0;
  for (int base = 0; base < n; base += 32) {
    const int i = base + lane;
    const uint64_t w = i < n ? node[i] : 0;
    const bool is_const = i < n && w_const(w);
    const unsigned const_mask = __ballot_sync(kFull, is_const);
    if (i < n) {
      const int o = w_origin(w);
      const int arity = __ldg(&info[o].arity), nk = __ldg(&info[o].node_kind);
      m.arity[i] = uint8_t(arity);
      if (arity == 0) {
        m.aop[i] = kLeafOp;
        // the accumulator VM reads constants and Int/Bool inputs; a bound
        // read (a traversal binder) needs the general VM
        total &= nk == TK_CONSTANT || nk == TK_LOCAL;
      } else {
        const uint32_t op = accumulator_op_of(nk, __ldg(&info[o].opcode), __ldg(&info[o].operand));
        m.aop[i] = uint8_t(op);
        total &= op != A_COUNT && arity <= 3;
      }
      bytecode += nk == TK_IF ? 2 : (nk == TK_AND || nk == TK_OR) ? 5 : 1;
      // leaves: the row constants in prefix order, or the input operand
      m.leaf[i] = is_const ? (K_CONST << 16) | uint32_t(constants + __popc(const_mask & ((1u << lane) - 1)))
                           : (K_INPUT << 16) | uint32_t(__ldg(&info[o].operand) & 0xffff);
    }
    constants += __popc(const_mask);
  }
  for (int k = lane; k < nc; k += 32) kpool[k] = cval[k];
  total = __all_sync(kFull, total);
  for (int o = 16; o; o >>= 1) bytecode += __shfl_xor_sync(kFull, bytecode, o);
  bytecode += 1;
  __syncwarp();
  // the exact bytecode length (a bound of every executed path) must fit the fuel
  if (!total || bytecode > s.fuel) return -1;
  return lower_accumulator_emit(m, n, code, code_cap, temps_out);
}

}  // namespace gb
