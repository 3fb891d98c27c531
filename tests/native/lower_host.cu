// Test harness only: the engine's lowering (lower_program) and exact VM
// (run_program) compiled for the host, so that CPU tests can compare them
// with the reference's own compiler output and CPU evaluator without a GPU.
// The product never loads this library; its kernels run the same functions
// on the device.
#include <algorithm>
#include <cstdint>
#include <vector>

#include "../../gagp_b200/csrc/vm.cuh"

namespace {
std::vector<gb::RegionInfo> regions_of(const gagp_region* regions, int count) {
  std::vector<gb::RegionInfo> out(count > 0 ? count : 1);
  for (int r = 0; r < count; ++r) out[r] = gb::region_info_of(regions[r]);
  return out;
}
}  // namespace

extern "C" {

// Lowers one row (construction expressions `origins`, Int constants in
// prefix order).  code: 5 ints per instruction; out[4]: instructions,
// constants, locals, stack bound.  Returns the instruction count or -1.
int host_lower(const gagp_grammar* g, const int32_t* origins, int n, const int64_t* constants, int nc,
               int32_t* code, int code_cap, int64_t* consts, int const_cap, int32_t* out) {
  std::vector<uint64_t> node(n);
  for (int i = 0; i < n; ++i) {
    const gagp_expression& x = g->expressions[origins[i]];
    node[i] = gb::w_make(origins[i], -1, 0, 0, x.arity, x.kind == gb::EK_CONSTANT, gb::kNoClass);
  }
  const std::vector<gb::RegionInfo> regions = regions_of(g->regions, g->region_count);
  const gb::LowerView v{g->expressions, regions.data(), g->expression_count, g->region_count, g->local_count,
                        g->local_types, g->slot_type, g->return_fuel};
  gb::LowerResult r{};
  const int len = gb::lower_program(v, node.data(), constants, n, nc, code, code_cap, consts, const_cap, &r);
  out[0] = r.code;
  out[1] = r.constants;
  out[2] = r.locals;
  out[3] = r.stack_bound;
  out[4] = r.main;
  out[5] = r.main_constants;
  return len;
}

// Runs a lowered program on case `c` of `cases` with `fuel`; returns 1 with
// the value and tag, 0 on a runtime error or timeout.  *steps: executed
// instructions.
int host_run(const gagp_cases* cases, const int32_t* local_types, int fuel, const int32_t* code, int n,
             const int64_t* consts, int n_locals, int c, int64_t* value, int32_t* tag, uint64_t* steps) {
  const int C = cases->case_count, NI = cases->input_count;
  std::vector<int64_t> inputs(size_t(NI > 0 ? NI : 1) * C);
  for (int j = 0; j < NI; ++j)
    for (int k = 0; k < C; ++k) inputs[size_t(j) * C + k] = cases->inputs[size_t(k) * NI + j];
  const gb::VmView v{inputs.data(), local_types, cases->list_values,
                     cases->list_values ? cases->list_value_count : 0, C, NI, fuel};
  int t = 0;
  uint64_t s = 0;
  const bool ok = gb::run_program(v, code, n, consts, n_locals, c, *value, t, s);
  *tag = t;
  *steps = s;
  return ok ? 1 : 0;
}

// Runs a lowered program with bounded regions (its main code the first
// n_main instructions, its main constants the first main_consts) on case
// `c`, with a host frame and memo workspace.
int host_run_regions(const gagp_grammar* g, const gagp_cases* cases, int fuel, const int32_t* code, int n, int n_main,
                     const int64_t* consts, int main_consts, int n_locals, int c, int64_t* value, int32_t* tag,
                     uint64_t* steps) {
  const int C = cases->case_count, NI = cases->input_count;
  std::vector<int64_t> inputs(size_t(NI > 0 ? NI : 1) * C);
  for (int j = 0; j < NI; ++j)
    for (int k = 0; k < C; ++k) inputs[size_t(j) * C + k] = cases->inputs[size_t(k) * NI + j];
  const gb::VmView v{inputs.data(), g->local_types, cases->list_values,
                     cases->list_values ? cases->list_value_count : 0, C, NI, fuel};
  const std::vector<gb::RegionInfo> regions = regions_of(g->regions, g->region_count);
  size_t words = 0;
  for (int r = 0; r < g->region_count; ++r) words = std::max(words, gb::region_lane_words(regions[r]));
  std::vector<int64_t> ws(words + 1);
  int t = 0;
  uint64_t s = 0;
  const bool ok = gb::run_program_regions(v, regions.data(), g->region_count, code, n, n_main, consts, main_consts,
                                          n_locals, c, ws.data(), words, *value, t, s);
  *tag = t;
  *steps = s;
  return ok ? 1 : 0;
}

}  // extern "C"
