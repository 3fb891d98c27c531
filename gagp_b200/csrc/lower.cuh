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

enum {
  OP_PUSH_CONST = 0, OP_LOAD = 1, OP_NEG = 3, OP_NOT = 4, OP_ADD = 5, OP_SUB = 6, OP_MUL = 7, OP_DIV = 8,
  OP_MOD = 9, OP_LT = 10, OP_LE = 11, OP_GT = 12, OP_GE = 13, OP_EQ = 14, OP_NE = 15, OP_JMP = 16,
  OP_JMP_IF_FALSE = 17, OP_JMP_IF_TRUE = 18, OP_CALL_BUILTIN = 19, OP_RETURN = 20
};
enum { B_ABS = 0, B_MIN = 1, B_MAX = 2, B_IDIV0 = 13, B_IMOD0 = 14, B_TRUNC_DIV0 = 28, B_TRUNC_MOD0 = 29 };

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

// Reference bytecode of a value phase.  Returns the instruction count
// (including the appended RETURN) or -1 when the compiler rejects the row.
// Code: 5 ints per instruction (op, flags, a, b, fuel).
__device__ inline int lower_reference(const SearchDesc& s, const LRow& t, int32_t* code, int code_cap,
                                      int64_t* consts, int* n_consts, int* stack_bound_out) {
  struct Frame { int node, base_stack, first_jump, second_jump, seen; int8_t args[3]; };
  Frame frames[64];
  int depth = 0, cursor = 0, count = 0, nconst = 0, stack = 0, stack_bound = 0, row_const = 0;
  int completed = GAGP_TAG_INVALID;
  bool have_value = false;
  auto emit = [&](int op, unsigned fuel, int a, int b, int flags) -> bool {
    if (count >= code_cap) return false;
    int32_t* x = code + 5 * count++;
    x[0] = op; x[1] = flags; x[2] = a; x[3] = b; x[4] = int32_t(fuel);
    return true;
  };
  auto grow = [&](int by) { stack += by; if (stack > stack_bound) stack_bound = stack; };
  if (t.n <= 0 || t.n > kCapacity) return -1;
  for (;;) {
    if (!have_value) {
      if (cursor >= t.n) return -1;
      const int index = cursor++;
      const gagp_expression& e = s.ex[w_origin(t.node[index])];
      if (e.node_kind == TK_CONSTANT) {
        // constants are Int payloads in prefix order
        if (nconst >= kCapacity) return -1;
        // the cursor visits nodes in prefix order, the order of row constants
        if (row_const >= t.nc) return -1;
        consts[nconst] = t.cval[row_const++];
        if (!emit(OP_PUSH_CONST, e.fuel, nconst, 0, 1)) return -1;
        ++nconst;
        grow(1);
        completed = GAGP_TAG_INT;
        have_value = true;
      } else if (e.node_kind == TK_LOCAL) {
        if (e.operand < 0 || e.operand >= s.local_count) return -1;
        if (!emit(OP_LOAD, e.fuel, e.operand, 0, 1)) return -1;
        grow(1);
        completed = e.type;
        have_value = true;
      } else {
        if (e.arity < 1 || e.arity > 3 || depth == 64) return -1;
        frames[depth++] = Frame{index, stack, -1, -1, 0, {0, 0, 0}};
        continue;
      }
    }
    if (depth == 0) {
      if (cursor != t.n || stack != 1 || completed != s.slot_type || stack_bound > 64) return -1;
      if (!emit(OP_RETURN, s.return_fuel, 0, 0, 0)) return -1;
      *n_consts = nconst;
      *stack_bound_out = stack_bound;
      return count;
    }
    Frame& f = frames[depth - 1];
    const gagp_expression& e = s.ex[w_origin(t.node[f.node])];
    if (f.seen < 3) f.args[f.seen] = int8_t(completed);
    ++f.seen;
    const bool branch = e.node_kind == TK_IF || e.node_kind == TK_AND || e.node_kind == TK_OR;
    if (branch && f.seen == 1) {
      f.first_jump = count;
      if (!emit(e.node_kind == TK_OR ? OP_JMP_IF_TRUE : OP_JMP_IF_FALSE, e.fuel, 0, 0, 1)) return -1;
      --stack;
    } else if (e.node_kind == TK_IF && f.seen == 2) {
      f.second_jump = count;
      if (!emit(OP_JMP, e.merge_fuel, 0, 0, 1)) return -1;
      code[5 * f.first_jump + 2] = count;
      stack = f.base_stack;
    }
    if (f.seen < e.arity) { have_value = false; continue; }
    if (e.node_kind == TK_IF) {
      code[5 * f.second_jump + 2] = count;
    } else if (e.node_kind == TK_AND || e.node_kind == TK_OR) {
      if (!emit(OP_NOT, e.fuel, 0, 0, 0) || !emit(OP_NOT, e.fuel, 0, 0, 0)) return -1;
      const int finish = count;
      if (!emit(OP_JMP, e.fuel, 0, 0, 1)) return -1;
      code[5 * f.first_jump + 2] = count;
      stack = f.base_stack;
      consts[nconst] = e.node_kind == TK_OR ? 1 : 0;
      // flag 4 marks a Bool constant for the general VM (the reference keeps
      // the tag in its constant Value); the low two bits are the reference's
      if (!emit(OP_PUSH_CONST, e.fuel, nconst, 0, 5)) return -1;
      ++nconst;
      grow(1);
      code[5 * finish + 2] = count;
      completed = GAGP_TAG_BOOL;
    } else {
      completed = e.type;
      if (e.opcode == OP_CALL_BUILTIN) {
        if (!emit(e.opcode, e.fuel, e.operand, e.arity, 3)) return -1;
      } else if (!emit(e.opcode, e.fuel, 0, 0, 0)) {
        return -1;
      }
      stack -= e.arity - 1;
    }
    --depth;
  }
}

// Accumulator op of a total operation node; A_COUNT when the node may raise
// a runtime error (then the program runs on the general VM).
__device__ __forceinline__ uint32_t accumulator_op(const gagp_expression& e) {
  if (e.node_kind == TK_AND) return A_AND;
  if (e.node_kind == TK_OR) return A_OR;
  if (e.node_kind == TK_IF) return A_SELECT;
  if (e.node_kind != TK_OPERATION) return A_COUNT;
  switch (e.opcode) {
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
      switch (e.operand) {
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

// Accumulator program of a row; returns the instruction count, or -1 when the
// row needs the general VM.  *temps_out: temporaries used.  MAXN bounds the
// row length (the per-thread working arrays).
template <int MAXN>
__device__ inline int lower_accumulator(const SearchDesc& s, const LRow& t, uint2* code, int code_cap,
                                        int64_t* kpool, int* kpool_len, int* temps_out) {
  (void)kpool_len;
  const int n = t.n;
  if (n <= 0 || n > MAXN) return -1;
  // child positions and Sethi-Ullman temporaries, children after parents
  int16_t end[MAXN];
  int8_t need[MAXN];
  int16_t constant_index[MAXN];
  {
    int k = 0;
    for (int i = 0; i < n; ++i) constant_index[i] = w_const(t.node[i]) ? int16_t(k++) : int16_t(-1);
  }
  for (int i = n - 1; i >= 0; --i) {
    const gagp_expression& e = s.ex[w_origin(t.node[i])];
    const int a = e.arity;
    if (a == 0) { end[i] = int16_t(i + 1); need[i] = 0; continue; }
    if (accumulator_op(e) == A_COUNT) return -1;
    int c = i + 1, needs[3], nonleaf = 0;
    for (int k = 0; k < a; ++k) {
      if (c >= n) return -1;
      if (end[c] - c > 1) needs[nonleaf++] = need[c];
      c = end[c];
    }
    end[i] = int16_t(c);
    // temporaries: non-leaf children by decreasing need, all but the last spilled
    for (int x = 0; x < nonleaf; ++x)
      for (int y = x + 1; y < nonleaf; ++y)
        if (needs[y] > needs[x]) { const int tmp = needs[x]; needs[x] = needs[y]; needs[y] = tmp; }
    int m = 0;
    for (int x = 0; x < nonleaf; ++x) m = max(m, needs[x] + x);
    need[i] = int8_t(min(m, 127));
  }
  if (end[0] != n) return -1;
  if (need[0] > kMaxTemps) return -1;
  *temps_out = need[0];
  // constant pool: the row constants in prefix order
  for (int k = 0; k < t.nc; ++k) kpool[k] = t.cval[k];
  *kpool_len = t.nc;
  auto leaf_kind = [&](int i) -> uint32_t {
    return constant_index[i] >= 0 ? K_CONST : K_INPUT;
  };
  auto leaf_index = [&](int i) -> uint32_t {
    return constant_index[i] >= 0 ? uint32_t(constant_index[i]) : uint32_t(s.ex[w_origin(t.node[i])].operand);
  };
  // explicit-stack post order emission
  struct Frame { int16_t node; int8_t stage, count, order[3], spilled[3]; int8_t temp_base; };
  Frame st[64];
  int sp = 0, len = 0, temp_top = 0;
  auto put = [&](uint2 x) -> bool { if (len >= code_cap) return false; code[len++] = x; return true; };
  // a leaf root
  if (end[0] - 0 == 1) {
    if (!put(a_instr(A_MOV, false, leaf_kind(0), leaf_index(0)))) return -1;
    return len;
  }
  auto push = [&](int node) -> bool {
    if (sp >= 64) return false;
    Frame& f = st[sp++];
    f.node = int16_t(node);
    f.stage = 0;
    f.temp_base = int8_t(temp_top);
    // non-leaf children in evaluation order (decreasing need, stable)
    const int a = s.ex[w_origin(t.node[node])].arity;
    int c = node + 1, k = 0;
    int8_t kids[3];
    for (int x = 0; x < a; ++x) { kids[x] = int8_t(c - node); c = end[c]; }
    f.count = 0;
    for (int x = 0; x < a; ++x) {
      const int ch = node + kids[x];
      if (end[ch] - ch > 1) f.order[f.count++] = int8_t(x);
    }
    for (int x = 0; x < f.count; ++x)
      for (int y = x + 1; y < f.count; ++y) {
        const int cx = node + kids[f.order[x]], cy = node + kids[f.order[y]];
        if (need[cy] > need[cx]) { const int8_t tmp = f.order[x]; f.order[x] = f.order[y]; f.order[y] = tmp; }
      }
    for (int x = 0; x < 3; ++x) f.spilled[x] = -1;
    (void)k;
    return true;
  };
  auto child_at = [&](int node, int x) -> int {
    int c = node + 1;
    for (int k = 0; k < x; ++k) c = end[c];
    return c;
  };
  if (!push(0)) return -1;
  while (sp) {
    Frame& f = st[sp - 1];
    const int node = f.node;
    if (f.stage < f.count) {
      // before evaluating the next non-leaf child, spill the previous one
      if (f.stage > 0) {
        const int prev = f.order[f.stage - 1];
        if (temp_top >= kMaxTemps) return -1;
        f.spilled[prev] = int8_t(temp_top);
        if (!put(a_instr(A_SPILL, false, K_TEMP, uint32_t(temp_top)))) return -1;
        ++temp_top;
      }
      const int child = child_at(node, f.order[f.stage]);
      ++f.stage;
      if (!push(child)) return -1;
      continue;
    }
    // all non-leaf children evaluated: the last one (if any) is in ACC
    const gagp_expression& e = s.ex[w_origin(t.node[node])];
    const uint32_t op = accumulator_op(e);
    const int a = e.arity;
    uint32_t kind[3] = {K_ACC, K_ACC, K_ACC}, idx[3] = {0, 0, 0};
    const int last = f.count ? f.order[f.count - 1] : -1;
    for (int x = 0; x < a; ++x) {
      const int ch = child_at(node, x);
      if (end[ch] - ch == 1) { kind[x] = leaf_kind(ch); idx[x] = leaf_index(ch); }
      else if (x == last) { kind[x] = K_ACC; }
      else { kind[x] = K_TEMP; idx[x] = uint32_t(f.spilled[x]); }
    }
    bool ok = true;
    if (a == 1) {
      if (kind[0] != K_ACC) ok = put(a_instr(A_MOV, false, kind[0], idx[0]));
      ok = ok && put(a_instr(op, false, K_ACC, 0));
    } else if (a == 2) {
      if (kind[0] != K_ACC && kind[1] != K_ACC) {
        ok = put(a_instr(A_MOV, false, kind[0], idx[0])) && put(a_instr(op, false, kind[1], idx[1]));
      } else if (kind[0] == K_ACC) {
        ok = put(a_instr(op, false, kind[1], idx[1]));
      } else {
        ok = put(a_instr(op, true, kind[0], idx[0]));  // acc = op(first, acc)
      }
    } else {
      ok = put(a_instr(A_SELECT, false, kind[0], idx[0], kind[1], idx[1], kind[2], idx[2]));
    }
    if (!ok) return -1;
    temp_top = f.temp_base;
    --sp;
  }
  return len;
}

}  // namespace gb
