// Fitness evaluation of lowered programs over the case set.
//
// Semantics: run_code_impl (cpp/src/runtime/cpu/execute_bytecode_cpu.cpp:152-626)
// with the value semantics of cpp/include/gagp/core/value_semantics.hpp:91-190
// and builtins_cpu.cpp:131-218, scored by fitness_case_score
// (cpp/include/gagp/core/fitness_policy.hpp:28-58) and summed as
// eval_fitness_cpu does (cpp/src/runtime/cpu/fitness_cpu.cpp:57-176).
//
// Exactness of the reduction: with an integral |penalty| every per-case
// score is an integer (a capped integer gap, 0/1, or the ceiling), so every
// partial sum is an integer below 2^48 in magnitude (admission checks
// cases * |penalty| < 2^48).  The reference's 48-bit canonicalisation is
// then the identity and its ordered 512-lane reduction equals any integer
// sum: lanes accumulate int64 losses and the warp reduces with shuffles.
#pragma once
#include "lower.cuh"

namespace gb {

__host__ __device__ __forceinline__ int64_t wrap_add(int64_t a, int64_t b) { return int64_t(uint64_t(a) + uint64_t(b)); }
__host__ __device__ __forceinline__ int64_t wrap_sub(int64_t a, int64_t b) { return int64_t(uint64_t(a) - uint64_t(b)); }
__host__ __device__ __forceinline__ int64_t wrap_mul(int64_t a, int64_t b) { return int64_t(uint64_t(a) * uint64_t(b)); }
__host__ __device__ __forceinline__ int64_t wrap_neg(int64_t a) { return int64_t(0ULL - uint64_t(a)); }
// Truncating quotient and remainder of int64 operands (b != 0, and not
// INT64_MIN / -1).  When both operands fit in 32 bits the 32-bit division
// gives the same results at a fraction of the 64-bit division's cost
// (program values are mostly small); b == -1 takes the 64-bit path, so the
// 32-bit one never sees INT32_MIN / -1.
__host__ __device__ __forceinline__ bool fits32(int64_t v) { return v == int64_t(int32_t(v)); }
__host__ __device__ __forceinline__ int64_t tquot(int64_t a, int64_t b) {
  return (fits32(a) && fits32(b) && b != -1) ? int64_t(int32_t(a) / int32_t(b)) : a / b;
}
__host__ __device__ __forceinline__ int64_t trem(int64_t a, int64_t b) {
  return (fits32(a) && fits32(b) && b != -1) ? int64_t(int32_t(a) % int32_t(b)) : a % b;
}
// Python-sign modulo (vm_semantics::py_int_mod); b != 0.
__host__ __device__ __forceinline__ int64_t py_mod(int64_t a, int64_t b) {
  if (b == -1) return 0;
  int64_t r = trem(a, b);
  if (r != 0 && ((r < 0) != (b < 0))) r += b;
  return r;
}
__host__ __device__ __forceinline__ int64_t idiv0(int64_t a, int64_t b) { return b == 0 ? 0 : b == -1 ? wrap_neg(a) : tquot(a, b); }
__host__ __device__ __forceinline__ int64_t imod0(int64_t a, int64_t b) { return b == 0 ? 0 : py_mod(a, b); }
__host__ __device__ __forceinline__ int64_t tdiv0(int64_t a, int64_t b) {
  return b == 0 || (a == INT64_MIN && b == -1) ? 0 : tquot(a, b);
}
__host__ __device__ __forceinline__ int64_t tmod0(int64_t a, int64_t b) {
  return b == 0 || (a == INT64_MIN && b == -1) ? 0 : trem(a, b);
}

// Loss (= -score) of one case and whether it is wrong.  `tag` is the
// program's static result type; values are Int payloads or 0/1 Bools.
__device__ __forceinline__ int64_t case_loss(const SearchDesc& s, int tag, int64_t value, int64_t expected,
                                             uint32_t& wrong) {
  const bool same = tag == s.expected_tag && value == expected;
  wrong += !same;
  if (s.metric == GAGP_METRIC_EXACT) return same ? 0 : 1;
  if (tag != GAGP_TAG_INT || s.expected_tag != GAGP_TAG_INT) return s.penalty_int;  // not numeric: ceiling
  const uint64_t gap = value >= expected ? uint64_t(value) - uint64_t(expected) : uint64_t(expected) - uint64_t(value);
  return gap < uint64_t(s.penalty_int) ? int64_t(gap) : s.penalty_int;
}
__device__ __forceinline__ int64_t error_loss(const SearchDesc& s) {
  return s.metric == GAGP_METRIC_EXACT ? 1 : s.penalty_int;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ------------------------------------------------------------ fast VM
// One warp runs one accumulator program; lane l holds cases
// tile*32K + k*32 + l for k < K (coalesced input loads).  The program's code
// and constants are staged in shared memory; with NIN (1 or 2) inputs the
// tile's input values live in registers, otherwise (NIN == 0) they are read
// through L1.  Temporaries live in shared memory [temp][k][lane].
struct VmWarpSmem {
  int64_t* temps;
  uint2* code;
  int64_t* consts;
};

// Staged form of an accumulator instruction: one handler per (operation,
// operand class), chosen once when a warp stages a program, so that running
// an instruction costs one dispatch.  Swapped operands are normalised away
// (a swapped comparison is the mirrored one; subtraction and the divisions
// have reversed handlers).  Staged word: x = handler | kinds << 8 | i3 << 16
// (kinds: the three 2-bit operand kinds, read by SELECT), y = i1 | i2 << 16.
enum : uint32_t {
  H_MOV_T = 0, H_MOV_I, H_MOV_C, H_SPILL, H_NEG, H_NOT, H_ABS, H_SELECT,
  H_BINARY  // first binary handler: H_BINARY + 3 * binary op + class (T, I, C)
};
enum : uint32_t {
  HB_ADD = 0, HB_SUB, HB_RSUB, HB_MUL, HB_LT, HB_LE, HB_GT, HB_GE, HB_EQ, HB_NE, HB_AND, HB_OR, HB_MIN, HB_MAX,
  HB_IDIV0, HB_RIDIV0, HB_IMOD0, HB_RIMOD0, HB_TDIV0, HB_RTDIV0, HB_TMOD0, HB_RTMOD0, HB_COUNT
};
__device__ __forceinline__ uint2 stage_accumulator(uint2 w) {
  const uint32_t op = w.x & 0xffu;
  const bool swap = (w.x >> 8) & 1u;
  const uint32_t k1 = (w.x >> 9) & 3u;
  const uint32_t kinds = (w.x >> 9) & 0x3fu;
  const uint32_t cls = k1 == K_TEMP ? 0u : k1 == K_INPUT ? 1u : 2u;  // binary and MOV operands are never the accumulator
  uint32_t h;
  switch (op) {
    case A_MOV: h = H_MOV_T + cls; break;
    case A_SPILL: h = H_SPILL; break;
    case A_NEG: h = H_NEG; break;
    case A_NOT: h = H_NOT; break;
    case A_ABS: h = H_ABS; break;
    case A_SELECT: h = H_SELECT; break;
    default: {
      uint32_t b;
      switch (op) {
        case A_ADD: b = HB_ADD; break;
        case A_SUB: b = swap ? HB_RSUB : HB_SUB; break;
        case A_MUL: b = HB_MUL; break;
        case A_LT: b = swap ? HB_GT : HB_LT; break;
        case A_LE: b = swap ? HB_GE : HB_LE; break;
        case A_GT: b = swap ? HB_LT : HB_GT; break;
        case A_GE: b = swap ? HB_LE : HB_GE; break;
        case A_EQ: b = HB_EQ; break;
        case A_NE: b = HB_NE; break;
        case A_AND: b = HB_AND; break;
        case A_OR: b = HB_OR; break;
        case A_MIN: b = HB_MIN; break;
        case A_MAX: b = HB_MAX; break;
        case A_IDIV0: b = swap ? HB_RIDIV0 : HB_IDIV0; break;
        case A_IMOD0: b = swap ? HB_RIMOD0 : HB_IMOD0; break;
        case A_TDIV0: b = swap ? HB_RTDIV0 : HB_TDIV0; break;
        default: b = swap ? HB_RTMOD0 : HB_TMOD0; break;
      }
      h = H_BINARY + 3 * b + cls;
    }
  }
  return make_uint2(h | (kinds << 8) | (w.x & 0xffff0000u), w.y);
}

// Runs cases [case_begin, case_end) (tiles of 32 K from case_begin).
template <int K, int NIN>
__device__ inline void run_accumulator(const SearchDesc& s, int slot, const VmWarpSmem& w, int case_begin,
                                       int case_end, int64_t& loss_out, uint32_t& wrong_out, uint64_t& ops_out) {
  const int lane = threadIdx.x & 31;
  const int C = s.C;  // input-major stride
  const int64_t* __restrict__ inputs = s.inputs;
  const int64_t* __restrict__ expected = s.expected;
  // a tile's inputs and expected values, loaded before they are needed: the
  // first tile's ahead of the code staging, each next tile's ahead of the
  // current tile's instructions, so that their latency overlaps other work
  int64_t in0[K], in1[K], want[K];
  auto fetch = [&](int tile) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int c = tile + k * 32 + lane;
      const bool live = c < case_end;
      in0[k] = (NIN >= 1 && live) ? __ldg(&inputs[c]) : 0;
      in1[k] = (NIN >= 2 && live) ? __ldg(&inputs[size_t(C) + c]) : 0;
      want[k] = live ? __ldg(&expected[c]) : 0;
    }
  };
  fetch(case_begin);
  const int len = s.code_len[slot];
  {
    const uint2* code = s.code + size_t(slot) * s.code_stride;
    const int64_t* kpool = s.kpool + size_t(slot) * s.stride;
    for (int i = lane; i < len; i += 32) w.code[i] = stage_accumulator(code[i]);
    for (int i = lane; i < s.stride; i += 32) w.consts[i] = kpool[i];
    __syncwarp();
  }
  int64_t* __restrict__ temps = w.temps;
  const int64_t* __restrict__ consts = w.consts;
  int64_t loss = 0;
  uint32_t wrong = 0;
  for (int tile = case_begin; tile < case_end; tile += 32 * K) {
    int64_t acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0;
    // this tile's operands, and the next tile's loads in flight
    int64_t cur0[K], cur1[K], cur_want[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      cur0[k] = in0[k];
      cur1[k] = in1[k];
      cur_want[k] = want[k];
    }
    if (tile + 32 * K < case_end) fetch(tile + 32 * K);
    // operand vector of kind `kind` (SELECT's operands)
    auto load = [&](uint32_t kind, uint32_t index, int64_t* v) {
      switch (kind) {
        case K_ACC:
#pragma unroll
          for (int k = 0; k < K; ++k) v[k] = acc[k];
          break;
        case K_TEMP:
#pragma unroll
          for (int k = 0; k < K; ++k) v[k] = temps[(index * K + k) * 32 + lane];
          break;
        case K_INPUT:
#pragma unroll
          for (int k = 0; k < K; ++k) {
            if (NIN == 1 || (NIN == 2 && index == 0)) v[k] = cur0[k];
            else if (NIN == 2) v[k] = cur1[k];
            else {
              const int c = tile + k * 32 + lane;
              v[k] = c < case_end ? __ldg(&inputs[size_t(index) * C + c]) : 0;
            }
          }
          break;
        default: {
          const int64_t x = consts[index];
#pragma unroll
          for (int k = 0; k < K; ++k) v[k] = x;
        }
      }
    };
    // the input operand of case k (I-class handlers)
    auto input = [&](uint32_t index, int k) -> int64_t {
      if (NIN == 1) return cur0[k];
      if (NIN == 2) return index == 0 ? cur0[k] : cur1[k];
      const int c = tile + k * 32 + lane;
      return c < case_end ? __ldg(&inputs[size_t(index) * C + c]) : 0;
    };
// One binary handler per operand class: a = the accumulator, b = the operand.
#define GB_ACC_BINARY(NAME, EXPR)                                        \
  case H_BINARY + 3 * NAME: {                                            \
    const int64_t* t = temps + i1 * (K * 32) + lane;                     \
    _Pragma("unroll") for (int k = 0; k < K; ++k) {                      \
      const int64_t a = acc[k], b = t[k * 32];                           \
      acc[k] = (EXPR);                                                   \
    }                                                                    \
    break;                                                               \
  }                                                                      \
  case H_BINARY + 3 * NAME + 1: {                                        \
    _Pragma("unroll") for (int k = 0; k < K; ++k) {                      \
      const int64_t a = acc[k], b = input(i1, k);                        \
      acc[k] = (EXPR);                                                   \
    }                                                                    \
    break;                                                               \
  }                                                                      \
  case H_BINARY + 3 * NAME + 2: {                                        \
    const int64_t b = consts[i1];                                        \
    _Pragma("unroll") for (int k = 0; k < K; ++k) {                      \
      const int64_t a = acc[k];                                          \
      acc[k] = (EXPR);                                                   \
    }                                                                    \
    break;                                                               \
  }
    uint2 ins = len ? w.code[0] : make_uint2(0, 0);
    for (int ip = 0; ip < len; ++ip) {
      const uint2 cur = ins;
      if (ip + 1 < len) ins = w.code[ip + 1];
      const uint32_t i1 = cur.y & 0xffffu;
      switch (cur.x & 0xffu) {
        case H_MOV_T: {
          const int64_t* t = temps + i1 * (K * 32) + lane;
#pragma unroll
          for (int k = 0; k < K; ++k) acc[k] = t[k * 32];
          break;
        }
        case H_MOV_I:
#pragma unroll
          for (int k = 0; k < K; ++k) acc[k] = input(i1, k);
          break;
        case H_MOV_C: {
          const int64_t x = consts[i1];
#pragma unroll
          for (int k = 0; k < K; ++k) acc[k] = x;
          break;
        }
        case H_SPILL: {
          int64_t* t = temps + i1 * (K * 32) + lane;
#pragma unroll
          for (int k = 0; k < K; ++k) t[k * 32] = acc[k];
          break;
        }
        case H_NEG:
#pragma unroll
          for (int k = 0; k < K; ++k) acc[k] = wrap_neg(acc[k]);
          break;
        case H_NOT:
#pragma unroll
          for (int k = 0; k < K; ++k) acc[k] ^= 1;
          break;
        case H_ABS:
#pragma unroll
          for (int k = 0; k < K; ++k) acc[k] = acc[k] < 0 ? wrap_neg(acc[k]) : acc[k];
          break;
        case H_SELECT: {
          const uint32_t kinds = (cur.x >> 8) & 0x3fu;
          int64_t b[K], t[K], e[K];
          load(kinds & 3u, i1, b);
          load((kinds >> 2) & 3u, cur.y >> 16, t);
          load((kinds >> 4) & 3u, cur.x >> 16, e);
#pragma unroll
          for (int k = 0; k < K; ++k) acc[k] = b[k] ? t[k] : e[k];
          break;
        }
        GB_ACC_BINARY(HB_ADD, wrap_add(a, b))
        GB_ACC_BINARY(HB_SUB, wrap_sub(a, b))
        GB_ACC_BINARY(HB_RSUB, wrap_sub(b, a))
        GB_ACC_BINARY(HB_MUL, wrap_mul(a, b))
        GB_ACC_BINARY(HB_LT, int64_t(a < b))
        GB_ACC_BINARY(HB_LE, int64_t(a <= b))
        GB_ACC_BINARY(HB_GT, int64_t(a > b))
        GB_ACC_BINARY(HB_GE, int64_t(a >= b))
        GB_ACC_BINARY(HB_EQ, int64_t(a == b))
        GB_ACC_BINARY(HB_NE, int64_t(a != b))
        GB_ACC_BINARY(HB_AND, a & b)
        GB_ACC_BINARY(HB_OR, a | b)
        GB_ACC_BINARY(HB_MIN, a < b ? a : b)
        GB_ACC_BINARY(HB_MAX, a > b ? a : b)
        GB_ACC_BINARY(HB_IDIV0, idiv0(a, b))
        GB_ACC_BINARY(HB_RIDIV0, idiv0(b, a))
        GB_ACC_BINARY(HB_IMOD0, imod0(a, b))
        GB_ACC_BINARY(HB_RIMOD0, imod0(b, a))
        GB_ACC_BINARY(HB_TDIV0, tdiv0(a, b))
        GB_ACC_BINARY(HB_RTDIV0, tdiv0(b, a))
        GB_ACC_BINARY(HB_TMOD0, tmod0(a, b))
        GB_ACC_BINARY(HB_RTMOD0, tmod0(b, a))
        default: break;
      }
    }
#undef GB_ACC_BINARY
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int c = tile + k * 32 + lane;
      if (c < case_end) loss += case_loss(s, s.result_type, acc[k], cur_want[k], wrong);
    }
  }
  __syncwarp();
  loss_out = loss;
  wrong_out = wrong;
  ops_out = uint64_t(len) * uint64_t(case_end - case_begin);
}

// ------------------------------------------------------------ general VM
// What the exact VM reads of a search: the case inputs (input-major), their
// tags, the IntList arena and the fuel.
struct VmView {
  const int64_t* inputs;
  const int32_t* local_types;
  const int64_t* lists;
  int64_t n_lists;
  int C, n_inputs, fuel;
};
__host__ __device__ inline VmView vm_view(const SearchDesc& s) {
  return VmView{s.inputs, s.local_types, s.lists, s.n_lists, s.C, s.n_inputs, s.fuel};
}

// Exact stack interpreter of the reference bytecode on case `c`: run_code_impl
// (cpp/src/runtime/cpu/execute_bytecode_cpu.cpp:152-626) for the opcodes the
// lowering emits, with the value semantics of value_semantics.hpp:91-190 and
// the len/index builtins of builtins_cpu.cpp:220-370.  Every instruction
// charges its fuel before it runs (Timeout when the fuel left is below the
// charge; a chain of more uncharged instructions than the program has is an
// error, as in the reference), so the loop is bounded by the fuel.  Values
// are an int64 payload and a tag: an Int, a Bool (0/1) or an IntList (the
// offset of its length word in the list arena).  `n_locals` is the
// program's inputs plus temporaries; the inputs are preset.  Returns false
// on any runtime error or timeout (every error scores the same), else the
// returned value and its tag.  `steps` counts executed instructions.
//
// A program with bounded regions runs through run_program_regions: its
// BOUNDED_REGION instructions execute the region (run_region) from the
// records and phase code that follow its main code.
struct RegionRun;
__host__ __device__ inline int region_operands(const RegionRun& rr, int ordinal);
__host__ __device__ inline bool run_region(const VmView& v, const RegionRun& rr, int ordinal, const int64_t* opv,
                                           const int8_t* opt, const int64_t* caller_lv, const int8_t* caller_lt,
                                           uint64_t caller_set, int& fuel, int64_t& value, int& tag, uint64_t& steps);

// The interpreter loop shared by a main program (Phase false: RETURN ends
// it, falling off the end is an error) and a bounded region's phase (Phase
// true: an expression segment whose value is the stack top at its end,
// run_code with require_return false).  lv/lt/set: the preset locals.
template <bool Phase>
__host__ __device__ inline bool run_code(const VmView& v, const int32_t* code, int n, const int64_t* consts,
                                         int n_locals, int64_t* lv, int8_t* lt, uint64_t set, int& fuel,
                                         const RegionRun* rr, int64_t& value, int& tag, uint64_t& steps) {
  int64_t sv[kMaxStack];
  int8_t st[kMaxStack];
  int sp = 0, ip = 0, uncharged = 0;
  while (ip < n) {
    const int32_t* x = code + 5 * ip++;
    const int op = x[0], flags = x[1], a = x[2], b = x[3];
    const int cost = x[4];
    if (cost < 0 || fuel < cost) return false;  // Timeout (or a charge beyond the signed fuel range)
    fuel -= cost;
    if (cost) uncharged = 0;
    else if (++uncharged > n) return false;     // zero-cost instruction cycle
    ++steps;
    switch (op) {
      case OP_PUSH_CONST:
        if (sp >= kMaxStack) return false;
        sv[sp] = consts[a];
        st[sp++] = int8_t((flags & kBoolConst) ? GAGP_TAG_BOOL : GAGP_TAG_INT);
        break;
      case OP_LOAD:
        if (sp >= kMaxStack || a < 0 || a >= n_locals || !((set >> a) & 1)) return false;  // Name error
        sv[sp] = lv[a];
        st[sp++] = lt[a];
        break;
      case OP_STORE:
        if (!sp || a < 0 || a >= n_locals) return false;
        --sp;
        lv[a] = sv[sp];
        lt[a] = st[sp];
        set |= 1ull << a;
        break;
      case OP_CHECK_INT:
        if (!sp || st[sp - 1] != GAGP_TAG_INT) return false;  // Type error
        break;
      case OP_NEG: case OP_NOT: {
        if (!sp) return false;
        const int64_t y = sv[sp - 1];
        const int t = st[sp - 1];
        if (op == OP_NEG) { if (t != GAGP_TAG_INT) return false; sv[sp - 1] = wrap_neg(y); }
        else { if (t != GAGP_TAG_BOOL) return false; sv[sp - 1] = y ^ 1; }
        break;
      }
      case OP_ADD: case OP_SUB: case OP_MUL: case OP_DIV: case OP_MOD: {
        if (sp < 2) return false;
        const int64_t y = sv[--sp], xv = sv[--sp];
        if (st[sp] != GAGP_TAG_INT || st[sp + 1] != GAGP_TAG_INT) return false;
        if ((op == OP_DIV || op == OP_MOD) && y == 0) return false;  // ZeroDiv
        if (op == OP_DIV) return false;                               // Float result: not admitted
        sv[sp] = op == OP_ADD ? wrap_add(xv, y) : op == OP_SUB ? wrap_sub(xv, y) : op == OP_MUL ? wrap_mul(xv, y)
                                                                                                 : py_mod(xv, y);
        st[sp++] = int8_t(GAGP_TAG_INT);
        break;
      }
      case OP_LT: case OP_LE: case OP_GT: case OP_GE: case OP_EQ: case OP_NE: {
        if (sp < 2) return false;
        const int64_t y = sv[--sp], xv = sv[--sp];
        const int ty = st[sp + 1], tx = st[sp];
        bool r;
        if (op == OP_EQ || op == OP_NE) {
          if (tx != ty || (tx != GAGP_TAG_INT && tx != GAGP_TAG_BOOL)) return false;
          r = (xv == y) == (op == OP_EQ);
        } else {
          if (tx != GAGP_TAG_INT || ty != GAGP_TAG_INT) return false;
          r = op == OP_LT ? xv < y : op == OP_LE ? xv <= y : op == OP_GT ? xv > y : xv >= y;
        }
        sv[sp] = r;
        st[sp++] = int8_t(GAGP_TAG_BOOL);
        break;
      }
      case OP_JMP:
        if (a < 0 || a > n) return false;
        ip = a;
        break;
      case OP_JMP_IF_FALSE: case OP_JMP_IF_TRUE: {
        if (!sp || a < 0 || a > n) return false;
        const int64_t y = sv[--sp];
        if (st[sp] != GAGP_TAG_BOOL) return false;
        if ((op == OP_JMP_IF_FALSE && !y) || (op == OP_JMP_IF_TRUE && y)) ip = a;
        break;
      }
      case OP_CALL_BUILTIN: {
        if (b < 0 || sp < b) return false;
        int64_t r;
        if (a == B_IS_INT) {
          // whether the value is an Int (builtins_cpu.cpp:493-499): a for_range's bound check
          if (b != 1) return false;
          sv[sp - 1] = st[sp - 1] == GAGP_TAG_INT;
          st[sp - 1] = int8_t(GAGP_TAG_BOOL);
          break;
        }
        if (a == B_LEN || a == B_INDEX) {
          // a read-only view of an input list: length word, then elements
          if (b != (a == B_LEN ? 1 : 2) || st[sp - b] != GAGP_TAG_INTLIST) return false;
          const int64_t at = sv[sp - b];
          if (at < 0 || at >= v.n_lists) return false;
          const int64_t len = v.lists[at];
          if (a == B_LEN) {
            r = len;
          } else {
            if (st[sp - 1] != GAGP_TAG_INT) return false;
            int64_t j = sv[sp - 1];
            if (j < 0) j += len;  // Python-style negative index
            if (j < 0 || j >= len) return false;  // index out of range
            r = v.lists[at + 1 + j];
          }
        } else {
          for (int k = sp - b; k < sp; ++k) if (st[k] != GAGP_TAG_INT) return false;
          if (a == B_ABS) { if (b != 1) return false; r = sv[sp - 1] < 0 ? wrap_neg(sv[sp - 1]) : sv[sp - 1]; }
          else {
            if (b != 2) return false;
            const int64_t p = sv[sp - 2], q = sv[sp - 1];
            switch (a) {
              case B_MIN: r = p < q ? p : q; break;
              case B_MAX: r = p > q ? p : q; break;
              case B_IDIV0: r = idiv0(p, q); break;
              case B_IMOD0: r = imod0(p, q); break;
              case B_TRUNC_DIV0: r = tdiv0(p, q); break;
              case B_TRUNC_MOD0: r = tmod0(p, q); break;
              default: return false;
            }
          }
        }
        sp -= b;
        sv[sp] = r;
        st[sp++] = int8_t(GAGP_TAG_INT);
        break;
      }
      case OP_RETURN:
        if (!sp) return false;
        value = sv[sp - 1];
        tag = st[sp - 1];
        return true;
      case OP_BOUNDED_REGION: {
        // the region's operands (initial states, bound operands) are popped
        // and its value pushed (execute_bytecode_cpu.cpp:482-570); a phase
        // holds no region
        if constexpr (Phase) {
          return false;
        } else {
          if (!rr || (flags & kHasA) == 0) return false;
          const int operands = region_operands(*rr, a);
          if (operands < 0 || sp < operands) return false;
          sp -= operands;
          int64_t r;
          int rt;
          if (!run_region(v, *rr, a, sv + sp, st + sp, lv, lt, set, fuel, r, rt, steps)) return false;
          sv[sp] = r;
          st[sp++] = int8_t(rt);
          break;
        }
      }
      default:
        return false;
    }
  }
  if (Phase && sp) {
    // an expression segment's value
    value = sv[sp - 1];
    tag = st[sp - 1];
    return true;
  }
  return false;  // finished without return
}

__host__ __device__ inline bool run_program(const VmView& v, const int32_t* code, int n, const int64_t* consts,
                                            int n_locals, int c, int64_t& value, int& tag, uint64_t& steps) {
  int64_t lv[kLowerLocals];
  int8_t lt[kLowerLocals];
  if (n_locals < v.n_inputs || n_locals > kLowerLocals) return false;
  uint64_t set = 0;  // bit k: local k holds a value
  for (int j = 0; j < v.n_inputs; ++j) {
    lv[j] = v.inputs[size_t(j) * v.C + c];
    lt[j] = int8_t(v.local_types[j]);
    set |= 1ull << j;
  }
  int fuel = v.fuel;
  return run_code<false>(v, code, n, consts, n_locals, lv, lt, set, fuel, nullptr, value, tag, steps);
}

// ------------------------------------------------------------ bounded regions
// A program's bounded regions at run time: the region table, the records
// and phase code after the main code (lower_program's layout), the phase
// constants after the main ones, and this lane's frame and memo workspace
// (region_lane_words int64 words).
struct RegionRun {
  const RegionInfo* regions;
  int n_regions;
  const int32_t* records;   // code + 5 * (main instructions)
  int n_records;            // instructions after the main code
  const int64_t* phase_consts;
  int64_t* ws;
  size_t ws_words;
};

// The records of region `ordinal`: its header's position, and its table
// entry; -1 when the records do not hold it.
__host__ __device__ inline int region_header(const RegionRun& rr, int ordinal, int* const_offset) {
  int at = 0, co = 0;
  for (int r = 0;; ++r) {
    if (at < 0 || at >= rr.n_records || rr.records[5 * at] != kRegionRecord) return -1;
    const int captures = rr.records[5 * at + 4], phases = rr.records[5 * at + 3];
    if (r == ordinal) {
      *const_offset = co;
      return at;
    }
    at += 1 + captures;
    for (int p = 0; p < phases; ++p) {
      if (at >= rr.n_records) return -1;
      co += rr.records[5 * at + 3];
      at += 1 + rr.records[5 * at + 2];
    }
  }
}
__host__ __device__ inline int region_operands(const RegionRun& rr, int ordinal) {
  int co = 0;
  const int at = region_header(rr, ordinal, &co);
  if (at < 0) return -1;
  const int info = rr.records[5 * at + 2];
  return info >= 0 && info < rr.n_regions ? rr.regions[info].operands : -1;
}

__host__ __device__ inline bool region_addable(int64_t a, int64_t b) {
  return b > 0 ? a <= INT64_MAX - b : b < 0 ? a >= INT64_MIN - b : true;
}

// One bounded region: the frame stack of d_run_bounded_region_impl
// (cpp/src/runtime/gpu/device/region_execution_device.cuh:328-510), whose
// results equal the reference CPU engine's execute_bounded_region with its
// region adapter (cpu/bounded_region.hpp:112-189, cpu/region_adapter.hpp:171-269).
// The coordinate bounds are resolved once and checked (lower <= upper;
// every request's offsets representable over a non-empty domain).  A frame
// entered is charged entry_fuel; a state outside the domain takes the
// boundary phase, else the base predicate decides between the base body
// and, after a memo miss, the requests in order -- each child state built
// by its transitions, a push past the frame limit a timeout -- and then
// the combine phase, whose value a memoized region stores (a store past
// the cell limit a timeout).  Phases run on the shared fuel with their
// bindings preset.  Coordinates are Int by the region's admission, so
// frames keep payloads only.
__host__ __device__ inline bool run_region(const VmView& v, const RegionRun& rr, int ordinal, const int64_t* opv,
                                           const int8_t* opt, const int64_t* caller_lv, const int8_t* caller_lt,
                                           uint64_t caller_set, int& fuel, int64_t& value, int& tag, uint64_t& steps) {
  int co = 0;
  const int at = region_header(rr, ordinal, &co);
  if (at < 0) return false;
  const int info_index = rr.records[5 * at + 2];
  if (info_index < 0 || info_index >= rr.n_regions) return false;
  const RegionInfo& R = rr.regions[info_index];
  const int S = R.state_count, Q = R.request_count;
  // phase code, constants and locals
  const int32_t* pcode[4];
  const int64_t* pconst[4];
  int plen[4], plocals[4];
  {
    int k = at + 1 + R.captures;
    for (int p = 0; p < 4; ++p) {
      if (k >= rr.n_records) return false;
      plen[p] = rr.records[5 * k + 2];
      plocals[p] = rr.records[5 * k + 4] & 0xffff;
      pcode[p] = rr.records + 5 * (k + 1);
      pconst[p] = rr.phase_consts + co;
      co += rr.records[5 * k + 3];
      k += 1 + plen[p];
      if (k > rr.n_records || plocals[p] > kLowerLocals) return false;
    }
  }
  int capture_slot[8];
  for (int c = 0; c < R.captures; ++c) capture_slot[c] = rr.records[5 * (at + 1 + c) + 2];
  for (int i = 0; i < R.operands; ++i)
    if (opt[i] != GAGP_TAG_INT) return false;  // states and bound operands are Int
  // the coordinate domain
  int64_t lower[4], upper[4];
  bool empty = false;
  for (int x = 0; x < R.axis_count; ++x) {
    lower[x] = R.lower_kind[x] ? opv[R.lower[x]] : R.lower[x];
    upper[x] = R.upper_kind[x] ? opv[R.upper[x]] : R.upper[x];
    if (lower[x] > upper[x]) return false;
    empty |= !R.inclusive && lower[x] == upper[x];
  }
  if (!empty)
    for (int x = 0; x < R.axis_count; ++x) {
      const int64_t top = R.inclusive ? upper[x] : upper[x] - 1;
      for (int q = 0; q < Q; ++q) {
        const int64_t off = R.transition_offset[q][R.axis_slot[x]];
        if (!region_addable(lower[x], off) || !region_addable(top, off)) return false;
      }
    }
  if (R.frames == 0) return false;  // Timeout
  if (!rr.ws || rr.ws_words < region_lane_words(R)) return false;
  // workspace: frames of (states, results, next request), then memo cells
  // of (states, value)
  const int fw = S + Q + 1;
  int64_t* frames = rr.ws;
  int64_t* memo = rr.ws + size_t(R.frames) * fw;
  uint32_t memo_count = 0;
  int depth = 1;
  for (int i = 0; i < S; ++i) frames[i] = opv[i];
  frames[S + Q] = -1;
  // one phase on frame f: bindings preset as its first locals
  auto phase = [&](int p, const int64_t* f, int64_t& out) -> bool {
    int64_t lv[kLowerLocals];
    int8_t lt[kLowerLocals];
    uint64_t set = 0;
    for (int b = 0; b < R.phase_bindings[p]; ++b) {
      const int bank = R.binding_bank[p][b], slot = R.binding_slot[p][b];
      if (bank == 0) {
        lv[b] = f[slot];
        lt[b] = int8_t(GAGP_TAG_INT);
      } else if (bank == 3) {
        lv[b] = f[S + slot];
        lt[b] = int8_t(R.result_type);
      } else {
        const int local = capture_slot[slot];
        if (local < 0 || local >= 64 || !((caller_set >> local) & 1)) continue;  // unset: not preset
        lv[b] = caller_lv[local];
        lt[b] = caller_lt[local];
      }
      set |= 1ull << b;
    }
    int t = 0;
    if (!run_code<true>(v, pcode[p], plen[p], pconst[p], plocals[p], lv, lt, set, fuel, nullptr, out, t, steps))
      return false;
    return t == R.phase_type[p];
  };
  int64_t result = 0;
  for (;;) {
    int64_t* f = frames + size_t(depth - 1) * fw;
    bool completed = false;
    if (f[S + Q] < 0) {
      if (fuel < 0 || R.entry_fuel > uint32_t(fuel)) return false;  // Timeout
      fuel -= int(R.entry_fuel);
      bool boundary = false, base = false;
      for (int x = 0; x < R.axis_count; ++x) {
        const int64_t c = f[R.axis_slot[x]];
        boundary |= c < lower[x] || (R.inclusive ? c > upper[x] : c >= upper[x]);
      }
      if (!boundary) {
        int64_t b;
        if (!phase(0, f, b)) return false;
        base = b != 0;
      }
      if (boundary || base) {
        if (!phase(boundary ? 3 : 1, f, result)) return false;
        completed = true;
      } else {
        if (R.memoized)
          for (uint32_t cell = 0; cell < memo_count; ++cell) {
            bool match = true;
            for (int i = 0; i < S; ++i) match &= memo[size_t(cell) * (S + 1) + i] == f[i];
            if (match) {
              result = memo[size_t(cell) * (S + 1) + S];
              completed = true;
              break;
            }
          }
        if (!completed) f[S + Q] = 0;
      }
    }
    if (!completed && f[S + Q] < Q) {
      const int q = int(f[S + Q]);
      int64_t next[4];
      for (int i = 0; i < S; ++i) {
        const int64_t src = f[R.transition_source[q][i]];
        if (R.transition_kind[q][i] == 0) {
          next[i] = src;
        } else {
          if (!region_addable(src, R.transition_offset[q][i])) return false;
          next[i] = src + R.transition_offset[q][i];
        }
      }
      if (uint32_t(depth) >= R.frames) return false;  // Timeout: frame capacity
      ++f[S + Q];
      int64_t* g = frames + size_t(depth) * fw;
      for (int i = 0; i < S; ++i) g[i] = next[i];
      g[S + Q] = -1;
      ++depth;
      continue;
    }
    if (!completed) {
      if (!phase(2, f, result)) return false;
      if (R.memoized) {
        if (memo_count >= R.cells) return false;  // Timeout: memo capacity
        for (int i = 0; i < S; ++i) memo[size_t(memo_count) * (S + 1) + i] = f[i];
        memo[size_t(memo_count) * (S + 1) + S] = result;
        ++memo_count;
      }
    }
    if (--depth == 0) break;
    int64_t* parent = frames + size_t(depth - 1) * fw;
    parent[S + parent[S + Q] - 1] = result;
  }
  value = result;
  tag = R.result_type;
  return true;
}

// A program with bounded regions on case `c`: n_main instructions of main
// code followed by n - n_main of records and phase code; the phase
// constants follow main_consts main constants.
__host__ __device__ inline bool run_program_regions(const VmView& v, const RegionInfo* regions, int n_regions,
                                                    const int32_t* code, int n, int n_main, const int64_t* consts,
                                                    int main_consts, int n_locals, int c, int64_t* ws,
                                                    size_t ws_words, int64_t& value, int& tag, uint64_t& steps) {
  int64_t lv[kLowerLocals];
  int8_t lt[kLowerLocals];
  if (n_locals < v.n_inputs || n_locals > kLowerLocals || n_main > n) return false;
  uint64_t set = 0;
  for (int j = 0; j < v.n_inputs; ++j) {
    lv[j] = v.inputs[size_t(j) * v.C + c];
    lt[j] = int8_t(v.local_types[j]);
    set |= 1ull << j;
  }
  const RegionRun rr{regions, n_regions, code + 5 * n_main, n - n_main, consts + main_consts, ws, ws_words};
  int fuel = v.fuel;
  return run_code<false>(v, code, n_main, consts, n_locals, lv, lt, set, fuel, &rr, value, tag, steps);
}

// ------------------------------------------------------------ warp-SIMD exact VM
// The exact VM for the 32 cases of one tile, executed by one warp with one
// decoded instruction at a time: every lane keeps its own instruction
// pointer, fuel and result, and at each step the lanes whose pointer is the
// smallest among the running lanes execute the instruction there together
// (a warp-uniform opcode, so no divergence inside the step).  Lanes that
// are ahead -- past a branch the others did not take, or out of a loop the
// others are still in -- wait until the others reach them, so branch joins
// and loop exits re-merge the warp.  The thread-per-case VM instead lets the
// lanes drift apart, after which every distinct opcode of a step runs
// serially.
//
// The stack and the locals live in shared memory as [slot][lane] columns of
// int64 payloads: locals first (inputs preset), then the stack.  Tags are
// not kept: the lowering's output is well typed (each operation's operands
// have the grammar's types, the stack depth and the definedness of every
// local are fixed per instruction), so none of the reference VM's type,
// underflow or uninitialised-local checks can fail on it and the result's
// tag is the phase's type; the checks that can fail on some case -- fuel,
// modulo by zero, index range -- are kept.  Results equal run_program's.
//
// Staged instruction (uint4): x = op (bits 0-6) | jump when true (bit 7) |
// instructions it stands for (bits 8-11) | binary operation (bits 12-15) |
// their summed fuel (bits 16-31); y, z, w: operands.  The kernel stages a
// program this way only when every cost is in 1..255 and its locals and
// stack fit kSimdSlots; otherwise it runs it on run_program.
//
// Superinstructions.  One thread of the block fuses, left to right, short
// straight-line runs that start anywhere but hold no jump target past their
// first instruction: LOAD a; LOAD b; op; STORE c (S_BIN_LL_ST), the same
// with PUSH_CONST k for the second load (S_BIN_LC_ST), LOAD a; LOAD b / PUSH
// k; comparison; JMP_IF_FALSE/TRUE t (S_JCMP_LL / S_JCMP_LC), LOAD a; LOAD b;
// CALL index; STORE c (S_INDEX_LL_ST), the three-instruction prefixes of the
// binary forms (S_BIN_LL, S_BIN_LC), op; STORE c (S_BIN_ST) and LOAD a;
// STORE c (S_MOVE).  A fused instruction charges the summed fuel before it
// runs (a timeout anywhere inside the run, or an error of one of its
// instructions, ends the case with an error in both forms, and otherwise
// every instruction runs) and counts as the instructions it stands for.  The
// skipped slots are never reached: jumps land only on run starts.
enum : int {
  S_MOVE = 64, S_BIN_LL, S_BIN_LC, S_BIN_LL_ST, S_BIN_LC_ST, S_JCMP_LL, S_JCMP_LC, S_INDEX_LL_ST, S_BIN_ST, S_FAIL
};
constexpr int kSimdSlots = 24;
constexpr int kSimdDone = 0x7fffffff;

__device__ __forceinline__ uint4 simd_plain(int op, int a, int cost) {
  return make_uint4(uint32_t(op & 0x7f) | (1u << 8) | (uint32_t(cost) << 16), uint32_t(a), 0u, 0u);
}
// The staged word of instruction k of `code` (5 ints per instruction).  The
// one type error the lowering emits on purpose -- NEG of the Bool constant
// that a for_range pushes for a bound that is not a non-negative Int --
// stages as S_FAIL, which charges the NEG's fuel and fails the case as the
// reference's NEG does; every other NEG has an Int operand.
__device__ __forceinline__ uint4 simd_stage(const int32_t* code, int k) {
  const int32_t* x = code + 5 * k;
  const bool bool_neg = x[0] == OP_NEG && k > 0 && code[5 * (k - 1)] == OP_PUSH_CONST &&
                        (code[5 * (k - 1) + 1] & kBoolConst);
  return simd_plain(bool_neg ? S_FAIL : x[0], x[2], x[4]);
}
__device__ __forceinline__ bool simd_binary_op(int op) {
  return op == OP_ADD || op == OP_SUB || op == OP_MUL || op == OP_MOD || (op >= OP_LT && op <= OP_NE);
}
__device__ __forceinline__ bool simd_compare_op(int op) { return op >= OP_LT && op <= OP_NE; }
// One binary operation of the reference VM on Int payloads (comparisons give
// 0/1); false on a modulo by zero (ZeroDiv).
__device__ __forceinline__ bool simd_binary(int op, int64_t x, int64_t y, int64_t& r) {
  switch (op) {
    case OP_ADD: r = wrap_add(x, y); return true;
    case OP_SUB: r = wrap_sub(x, y); return true;
    case OP_MUL: r = wrap_mul(x, y); return true;
    case OP_MOD:
      if (y == 0) return false;
      r = py_mod(x, y);
      return true;
    case OP_LT: r = x < y; return true;
    case OP_LE: r = x <= y; return true;
    case OP_GT: r = x > y; return true;
    case OP_GE: r = x >= y; return true;
    case OP_EQ: r = x == y; return true;
    default: r = x != y; return true;
  }
}

// The fusion pass over a staged program (code: 5 ints per instruction; words
// hold the plain staging; targets: n bits, zeroed).  One thread.
__device__ inline void simd_fuse(const int32_t* code, int n, uint4* words, unsigned long long* targets) {
  auto op_at = [&](int k) { return code[5 * k]; };
  auto a_at = [&](int k) { return code[5 * k + 2]; };
  auto cost_at = [&](int k) { return uint32_t(code[5 * k + 4]); };
  for (int k = 0; k < n; ++k) {
    const int op = op_at(k), t = a_at(k);
    if ((op == OP_JMP || op == OP_JMP_IF_FALSE || op == OP_JMP_IF_TRUE) && t >= 0 && t < n)
      targets[t >> 6] |= 1ull << (t & 63);
  }
  // instructions k+1 .. k+len-1 exist and none is a jump target
  auto free_run = [&](int k, int len) {
    if (k + len > n) return false;
    for (int j = 1; j < len; ++j)
      if (targets[(k + j) >> 6] >> ((k + j) & 63) & 1) return false;
    return true;
  };
  auto fused = [&](int k, int len, int op, int bop, bool jt, uint32_t y, uint32_t z, uint32_t w) {
    uint32_t cost = 0;
    for (int j = 0; j < len; ++j) cost += cost_at(k + j);
    words[k] = make_uint4(uint32_t(op) | (uint32_t(jt) << 7) | (uint32_t(len) << 8) | (uint32_t(bop - OP_ADD) << 12) |
                              (cost << 16),
                          y, z, w);
  };
  for (int k = 0; k < n;) {
    const int o0 = op_at(k), o1 = k + 1 < n ? op_at(k + 1) : -1, o2 = k + 2 < n ? op_at(k + 2) : -1,
              o3 = k + 3 < n ? op_at(k + 3) : -1;
    const bool second = o1 == OP_LOAD || o1 == OP_PUSH_CONST;
    int len = 1;
    if (o0 == OP_LOAD && second && simd_binary_op(o2) && o3 == OP_STORE && free_run(k, 4)) {
      fused(k, 4, o1 == OP_LOAD ? S_BIN_LL_ST : S_BIN_LC_ST, o2, false, a_at(k), a_at(k + 1), a_at(k + 3));
      len = 4;
    } else if (o0 == OP_LOAD && second && simd_compare_op(o2) && (o3 == OP_JMP_IF_FALSE || o3 == OP_JMP_IF_TRUE) &&
               free_run(k, 4)) {
      fused(k, 4, o1 == OP_LOAD ? S_JCMP_LL : S_JCMP_LC, o2, o3 == OP_JMP_IF_TRUE, a_at(k), a_at(k + 1), a_at(k + 3));
      len = 4;
    } else if (o0 == OP_LOAD && o1 == OP_LOAD && o2 == OP_CALL_BUILTIN && a_at(k + 2) == B_INDEX && o3 == OP_STORE &&
               free_run(k, 4)) {
      fused(k, 4, S_INDEX_LL_ST, OP_ADD, false, a_at(k), a_at(k + 1), a_at(k + 3));
      len = 4;
    } else if (o0 == OP_LOAD && second && simd_binary_op(o2) && free_run(k, 3)) {
      fused(k, 3, o1 == OP_LOAD ? S_BIN_LL : S_BIN_LC, o2, false, a_at(k), a_at(k + 1), 0);
      len = 3;
    } else if (simd_binary_op(o0) && o1 == OP_STORE && free_run(k, 2)) {
      fused(k, 2, S_BIN_ST, o0, false, a_at(k + 1), 0, 0);
      len = 2;
    } else if (o0 == OP_LOAD && o1 == OP_STORE && free_run(k, 2)) {
      fused(k, 2, S_MOVE, OP_ADD, false, a_at(k), a_at(k + 1), 0);
      len = 2;
    }
    k += len;
  }
}

struct SimdCase {
  int64_t value;
  bool ok;
  uint32_t steps;
};

__device__ inline SimdCase run_program_simd(const VmView& v, const uint4* code, int n, const int64_t* consts,
                                            int n_locals, int c, bool live, int64_t* slots) {
  const int lane = threadIdx.x & 31;
  SimdCase out{0, false, 0};
  // locals [0, n_locals): inputs preset; the stack follows
  for (int j = 0; j < v.n_inputs; ++j)
    if (live) slots[j * 32 + lane] = __ldg(&v.inputs[size_t(j) * v.C + c]);
  int ip = live ? 0 : kSimdDone, sp = n_locals, fuel = v.fuel;
  auto at = [&](int k) -> int64_t& { return slots[k * 32 + lane]; };
  for (;;) {
    const int ipm = __reduce_min_sync(kFull, ip);
    if (ipm == kSimdDone) break;
    if (ip != ipm) continue;
    const uint4 w = code[ipm];
    const int op = int(w.x & 0x7fu), len = int((w.x >> 8) & 0xfu), bop = OP_ADD + int((w.x >> 12) & 0xfu);
    const int cost = int(w.x >> 16), a = int(w.y);
    if (fuel < cost) { ip = kSimdDone; continue; }  // Timeout
    fuel -= cost;
    out.steps += len;
    ip += len;
    switch (op) {
      case OP_PUSH_CONST: at(sp++) = consts[a]; break;
      case OP_LOAD: { const int64_t x = at(a); at(sp++) = x; break; }
      case OP_STORE: at(a) = at(--sp); break;
      case OP_CHECK_INT: break;
      case OP_NEG: at(sp - 1) = wrap_neg(at(sp - 1)); break;
      case OP_NOT: at(sp - 1) ^= 1; break;
      case OP_ADD: case OP_SUB: case OP_MUL: case OP_MOD:
      case OP_LT: case OP_LE: case OP_GT: case OP_GE: case OP_EQ: case OP_NE: {
        const int64_t y = at(--sp), x = at(sp - 1);
        int64_t r;
        if (!simd_binary(op, x, y, r)) { ip = kSimdDone; break; }  // ZeroDiv
        at(sp - 1) = r;
        break;
      }
      case OP_JMP: ip = a; break;
      case OP_JMP_IF_FALSE: case OP_JMP_IF_TRUE: {
        const int64_t y = at(--sp);
        if ((op == OP_JMP_IF_FALSE) == (y == 0)) ip = a;
        break;
      }
      case OP_CALL_BUILTIN: {
        int64_t r = 0;
        if (a == B_IS_INT) {
          r = 1;  // a for_range bound: an Int in a well-typed program
        } else if (a == B_LEN) {
          r = __ldg(&v.lists[at(sp - 1)]);
        } else if (a == B_INDEX) {
          const int64_t j0 = at(--sp), h = at(sp - 1), len_h = __ldg(&v.lists[h]);
          const int64_t j = j0 < 0 ? j0 + len_h : j0;
          if (j < 0 || j >= len_h) { ip = kSimdDone; break; }  // index out of range
          r = __ldg(&v.lists[h + 1 + j]);
        } else if (a == B_ABS) {
          const int64_t x = at(sp - 1);
          r = x < 0 ? wrap_neg(x) : x;
        } else {
          const int64_t q = at(--sp), p = at(sp - 1);
          r = a == B_MIN ? (p < q ? p : q) : a == B_MAX ? (p > q ? p : q) : a == B_IDIV0 ? idiv0(p, q)
            : a == B_IMOD0 ? imod0(p, q) : a == B_TRUNC_DIV0 ? tdiv0(p, q) : tmod0(p, q);
        }
        at(sp - 1) = r;
        break;
      }
      case OP_RETURN:
        out.value = at(sp - 1);
        out.ok = true;
        ip = kSimdDone;
        break;
      case S_MOVE: at(int(w.z)) = at(a); break;
      case S_BIN_LL: case S_BIN_LC: case S_BIN_LL_ST: case S_BIN_LC_ST: {
        const int64_t x = at(a), y = (op == S_BIN_LL || op == S_BIN_LL_ST) ? at(int(w.z)) : consts[w.z];
        int64_t r;
        if (!simd_binary(bop, x, y, r)) { ip = kSimdDone; break; }  // ZeroDiv
        if (op == S_BIN_LL || op == S_BIN_LC) at(sp++) = r;
        else at(int(w.w)) = r;
        break;
      }
      case S_JCMP_LL: case S_JCMP_LC: {
        const int64_t x = at(a), y = op == S_JCMP_LL ? at(int(w.z)) : consts[w.z];
        int64_t r;
        simd_binary(bop, x, y, r);  // a comparison: never fails
        if ((r != 0) == bool(w.x & 0x80u)) ip = int(w.w);
        break;
      }
      case S_INDEX_LL_ST: {
        const int64_t h = at(a), j0 = at(int(w.z)), len_h = __ldg(&v.lists[h]);
        const int64_t j = j0 < 0 ? j0 + len_h : j0;
        if (j < 0 || j >= len_h) { ip = kSimdDone; break; }  // index out of range
        at(int(w.w)) = __ldg(&v.lists[h + 1 + j]);
        break;
      }
      case S_BIN_ST: {
        const int64_t y = at(--sp), x = at(--sp);
        int64_t r;
        if (!simd_binary(bop, x, y, r)) { ip = kSimdDone; break; }  // ZeroDiv
        at(a) = r;
        break;
      }
      case S_FAIL: ip = kSimdDone; break;  // NEG of a Bool: a type error
      default:
        ip = kSimdDone;  // not emitted by the lowering
    }
  }
  return out;
}

}  // namespace gb
