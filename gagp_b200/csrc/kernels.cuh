// Kernels of one resident steady-state round and of search start-up.
//
// Every kernel works on a batch of searches: `descs` holds one SearchDesc per
// search and per-item kernels map a flat index to (search, item) with the
// offsets array (items of search i are [off[i], off[i+1])).  A single search
// is a batch of one.  Per round (run_phase_population_steady,
// cpp/src/evolution/evolve.cpp:388-427):
//   k_record (epoch start) -> k_vary -> k_lower -> k_vm_fast (exact-VM programs included)
//   -> k_child_results -> k_place -> k_commit
#pragma once
#include <cooperative_groups.h>

#include "operators.cuh"
#include "vm.cuh"

namespace gb {

namespace cg = cooperative_groups;

struct ProgramRef {
  int32_t search, slot;
};

__device__ __forceinline__ int find_search(const int32_t* off, int n, int item) {
  int lo = 0, hi = n;  // off[lo] <= item < off[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= item) lo = mid; else hi = mid;
  }
  return lo;
}
__device__ __forceinline__ bool search_live(const SearchDesc& s) { return !s.round[2] && !s.round[3]; }
__device__ __forceinline__ void raise_error(const SearchDesc& s, int code) { atomicCAS(&s.round[3], 0, code); }

// ----------------------------------------------------------- start-up
// generate_phase_initial_population for a one-phase whole program
// (cpp/src/evolution/repro/gpu/phase_population_cpu.cpp:54-113): member i is
// grown at site depth 2 + i mod (site_depth - 1), retried with fresh seeds
// and raised by one every fourth failure.
__global__ void k_init_population(const SearchDesc* descs, const int32_t* off, int n) {
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= off[n]) return;
  const int si = find_search(off, n, item);
  const SearchDesc& s = descs[si];
  if (s.imported) return;  // the caller's rows are the initial population
  const int i = item - off[si];
  const int site_limit = s.site_depth;
  const int ramp = site_limit < 2 ? site_limit : 2 + i % (site_limit - 1);
  uint64_t* node = s.node + size_t(i) * s.stride;
  int64_t* cval = s.cval + size_t(i) * s.stride;
  uint64_t pending[192];
  GenResult g{ST_INVALID, 0, 0, 0};
  for (int logical = ramp, attempt = 0; g.status != ST_OK; ++attempt) {
    const int room = s.maxv < kCapacity ? s.maxv : kCapacity;
    g = generate(s, s.gen_image, s.root_expression, 0, s.slot_max_depth, room,
                 mix64(s.seed ^ mix64((uint64_t(i) * 8 + 0) * 64 + uint64_t(attempt))), node, cval, logical, pending);
    // a statement program that reads a grammar local before assigning it
    // is retried with the next seed (phase_population_cpu.cpp:95-96)
    if (g.status == ST_OK && is_statement_tag(s.slot_type) && !row_locals_defined(s, node, g.nodes))
      g.status = ST_INVALID;
    if (g.status != ST_OK && attempt % 4 == 3 && logical < site_limit) ++logical;
    if (attempt >= 256 && g.status != ST_OK) {
      raise_error(s, 20);
      s.len[i] = make_len(1, 0);
      return;
    }
  }
  // site depths relative to the budget `logical` are absolute here: the root
  // phase starts with no site above it
  s.len[i] = make_len(g.nodes, g.constants);
}

// ----------------------------------------------------------- lowering
// mode 0: the members (initial evaluation); mode 1: this round's children
// that reuse no member's result; batch items [lo, hi).  One warp per row:
// the accumulator program when the row is total and fits the fuel (listed in
// fast_list, counted in list_count[0]), else the reference bytecode for the
// general VM (lane 0; listed in general_list, counted in *general_count).
constexpr int kLowerWarps = 4;
__global__ void __launch_bounds__(kLowerWarps * 32, 8) k_lower(const SearchDesc* descs, const int32_t* off, int n,
                                                            int mode, ProgramRef* fast_list, ProgramRef* general_list,
                                                            int32_t* list_count, int32_t* general_count, int lo,
                                                            int hi) {
  __shared__ LowerScratch scratch[kLowerWarps];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int total_items = min(off[n], hi);
  for (int item = lo + blockIdx.x * kLowerWarps + warp; item < total_items; item += gridDim.x * kLowerWarps) {
    const int si = find_search(off, n, item);
    const SearchDesc& s = descs[si];
    if (!search_live(s)) continue;
    const int slot = item - off[si];
    LRow t;
    if (mode == 0) {
      const int32_t l = s.len[slot];
      t = LRow{s.node + size_t(slot) * s.stride, s.cval + size_t(slot) * s.stride, len_nodes(l), len_consts(l)};
    } else {
      if (!s.c_eval[slot]) continue;
      const int32_t l = s.clen[slot];
      t = LRow{s.cnode + size_t(slot) * s.stride, s.ccval + size_t(slot) * s.stride, len_nodes(l), len_consts(l)};
      // a child its parent does not cover reuses an identical current
      // member's result when there is one (make_batch's member_hashes
      // lookup, phase_population_cpu.cpp:336-339) and is neither lowered
      // nor evaluated
      if (s.mtab) {
        const int m = warp_find_member(s, SRow{const_cast<uint64_t*>(t.node), const_cast<int64_t*>(t.cval), t.n, t.nc});
        if (m >= 0) {
          if (lane == 0) {
            s.c_reuse[slot] = m;
            s.c_eval[slot] = 0;
          }
          continue;
        }
      }
    }
    int temps = 0;
    const int len = lower_accumulator_warp(s, t.node, t.n, t.cval, t.nc, s.code + size_t(slot) * s.code_stride,
                                           s.code_stride, s.kpool + size_t(slot) * s.stride, scratch[warp], &temps);
    // row and its length read; code words, constants, length, temps and list entry written
    const uint64_t row_bytes = 8ull * (t.n + t.nc) + 4;
    if (len >= 0) {
      if (lane == 0) {
        s.code_len[slot] = len;
        s.code_temps[slot] = temps;
        s.vm_acc[2 * size_t(slot)] = 0;
        s.vm_acc[2 * size_t(slot) + 1] = 0;
        fast_list[atomicAdd(&list_count[0], 1)] = ProgramRef{si, slot};
        atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[9]),
                  (unsigned long long)(row_bytes + 8ull * (len + t.nc) + 16));
      }
      continue;
    }
    if (lane == 0) {
      LowerResult r{};
      const int bl = lower_program(lower_view(s), t.node, t.cval, t.n, t.nc, s.bc + size_t(slot) * 5 * s.bc_stride,
                                   s.bc_stride, s.bc_consts + size_t(slot) * s.bc_stride, s.bc_stride, &r);
      if (bl < 0) {
        raise_error(s, 30);  // the phase compiler rejected a constructed program
      } else {
        s.bc_len[slot] = bl;
        // the main code's length marks a program with bounded regions (its
        // records and phase code follow); an exact-VM program keeps its
        // main constant count where an accumulator program keeps its
        // temporaries
        s.bc_locals[slot] = r.locals | (r.stack_bound << 8) | (r.main << 16);
        s.code_temps[slot] = r.main_constants;
        general_list[atomicAdd(general_count, 1)] = ProgramRef{si, slot};
        atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[9]),
                  (unsigned long long)(row_bytes + 20ull * bl + 8ull * r.constants + 16));
      }
    }
    __syncwarp();
  }
}

__device__ __forceinline__ void store_result(const SearchDesc& s, int mode, int slot, int64_t loss, uint32_t wrong,
                                             uint32_t errors) {
  const double f = -double(loss);
  if (mode == 0) {
    s.fitness[slot] = f;
    s.wrong[slot] = s.has_wrong ? wrong : 0;
    if (s.errors) s.errors[slot] = errors;
  } else {
    s.c_fitness[slot] = f;
    s.c_wrong[slot] = s.has_wrong ? wrong : 0;
  }
}

// General VM: the programs the accumulator VM cannot run (list programs,
// possible runtime errors or fuel exhaustion) on the exact interpreter.
// Persistent blocks of 8 warps take one program of the list at a time and
// stage its bytecode and constants in shared memory.  A program whose costs
// are all 1..255 and whose locals and stack fit kSimdSlots runs on the
// warp-SIMD VM (run_program_simd): the block's warps take its tiles of 32
// cases; any other runs on run_program, a case per thread.  The block
// reduces the losses in order-free integer sums.  A separate kernel from the
// fast VM, so that the interpreters' registers and local arrays do not
// lower the fast VM's occupancy.
//
// Dynamic shared memory: constants (bc_stride_max int64), the staged SIMD
// words (bc_stride_max uint4), the 5-int code (bc_stride_max instructions),
// a jump-target bit per instruction and per warp kSimdSlots x 32 int64 slots.
constexpr int kGeneralWarps = 8;
__host__ __device__ __forceinline__ size_t general_smem_bytes(int bc_stride_max) {
  return size_t(bc_stride_max) * (8 + 16 + 20) + 8 * ((size_t(bc_stride_max) + 63) / 64) + 16 +
         size_t(kGeneralWarps) * kSimdSlots * 32 * 8;
}
__global__ void __launch_bounds__(kGeneralWarps * 32) k_vm_general(const SearchDesc* descs, int mode,
                                                                   const ProgramRef* list, const int32_t* list_count,
                                                                   int bc_stride_max, ProgramRef* deferred,
                                                                   int32_t* deferred_count) {
  extern __shared__ __align__(16) int64_t smem_general[];
  __shared__ int64_t red_loss[kGeneralWarps];
  __shared__ uint32_t red_wrong[kGeneralWarps], red_errors[kGeneralWarps];
  __shared__ unsigned long long red_steps[kGeneralWarps];
  int64_t* consts = smem_general;
  uint4* words = reinterpret_cast<uint4*>(smem_general + bc_stride_max);
  int32_t* code = reinterpret_cast<int32_t*>(smem_general + 3 * size_t(bc_stride_max));
  unsigned long long* targets =
      reinterpret_cast<unsigned long long*>(smem_general + 3 * size_t(bc_stride_max) + (5 * size_t(bc_stride_max) + 1) / 2);
  int64_t* slots_all = reinterpret_cast<int64_t*>(targets + (size_t(bc_stride_max) + 63) / 64);
  const int count = *list_count;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int64_t* slots = slots_all + size_t(warp) * kSimdSlots * 32;
  for (int i = blockIdx.x; i < count; i += gridDim.x) {
    const ProgramRef p = list[i];
    const SearchDesc& s = descs[p.search];
    const int n = s.bc_len[p.slot], shape = s.bc_locals[p.slot];
    const int n_locals = shape & 0xff, stack_bound = (shape >> 8) & 0xff;
    if (((shape >> 16) & 0xffff) < n) {
      // a program with bounded regions: k_vm_region runs it with a frame
      // and memo workspace per lane
      if (threadIdx.x == 0) deferred[atomicAdd(deferred_count, 1)] = p;
      continue;
    }
    bool simd_ok = n_locals + stack_bound <= kSimdSlots;
    {
      const int32_t* gcode = s.bc + size_t(p.slot) * 5 * s.bc_stride;
      const int64_t* gconsts = s.bc_consts + size_t(p.slot) * s.bc_stride;
      for (int k = threadIdx.x; k < 5 * n; k += blockDim.x) code[k] = gcode[k];
      for (int k = threadIdx.x; k < n; k += blockDim.x) {
        consts[k] = gconsts[k];  // at most one constant per instruction
        const int32_t* x = gcode + 5 * k;
        const int cost = x[4];
        simd_ok &= cost >= 1 && cost <= 255 && x[0] >= 0 && x[0] < 64;
        words[k] = simd_stage(gcode, k);
      }
      for (int k = threadIdx.x; k < (n + 63) / 64; k += blockDim.x) targets[k] = 0;
    }
    simd_ok = __syncthreads_and(simd_ok);
    if (simd_ok && threadIdx.x == 0) simd_fuse(code, n, words, targets);
    __syncthreads();
    const VmView view = vm_view(s);
    int64_t loss = 0;
    uint32_t wrong = 0, errors = 0;
    uint64_t steps = 0;
    if (simd_ok) {
      for (int c0 = warp * 32; c0 < s.C; c0 += kGeneralWarps * 32) {
        const int c = c0 + lane;
        const bool live = c < s.C;
        const SimdCase r = run_program_simd(view, words, n, consts, n_locals, c, live, slots);
        if (live) {
          if (r.ok) loss += case_loss(s, s.result_type, r.value, s.expected[c], wrong);
          else { loss += error_loss(s); ++wrong; ++errors; }
        }
        steps += r.steps;
      }
    } else {
      for (int c = threadIdx.x; c < s.C; c += blockDim.x) {
        int64_t value = 0;
        int tag = 0;
        if (run_program(view, code, n, consts, n_locals, c, value, tag, steps)) {
          loss += case_loss(s, tag, value, s.expected[c], wrong);
        } else {
          loss += error_loss(s);
          ++wrong;
          ++errors;
        }
      }
    }
    loss = warp_sum(loss);
    wrong = warp_sum(wrong);
    errors = warp_sum(errors);
    steps = warp_sum(steps);
    if (lane == 0) {
      red_loss[warp] = loss;
      red_wrong[warp] = wrong;
      red_errors[warp] = errors;
      red_steps[warp] = steps;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t tl = 0;
      uint32_t tw = 0, te = 0;
      unsigned long long ts = 0;
      for (int w = 0; w < kGeneralWarps; ++w) {
        tl += red_loss[w];
        tw += red_wrong[w];
        te += red_errors[w];
        ts += red_steps[w];
      }
      store_result(s, mode, p.slot, tl, tw, te);
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[24]), ts);
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[0]), 1ULL);
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[2]), (unsigned long long)s.C);
    }
    __syncthreads();
  }
}

// Programs with bounded regions (deferred by k_vm_general): a fixed grid of
// blocks of kRegionThreads, one program per block at a time and one case
// per thread at a time on the per-thread interpreter
// (run_program_regions), each thread with its own `ws_words` words of
// frames and memo cells in `ws` (gridDim x kRegionThreads lanes).
constexpr int kRegionThreads = 128;
__global__ void __launch_bounds__(kRegionThreads) k_vm_region(const SearchDesc* descs, int mode, const ProgramRef* list,
                                                              const int32_t* list_count, int64_t* ws,
                                                              size_t ws_words) {
  __shared__ int64_t red_loss[kRegionThreads / 32];
  __shared__ uint32_t red_wrong[kRegionThreads / 32], red_errors[kRegionThreads / 32];
  __shared__ unsigned long long red_steps[kRegionThreads / 32];
  const int count = *list_count;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int64_t* mine = ws + (size_t(blockIdx.x) * kRegionThreads + threadIdx.x) * ws_words;
  for (int i = blockIdx.x; i < count; i += gridDim.x) {
    const ProgramRef p = list[i];
    const SearchDesc& s = descs[p.search];
    const int n = s.bc_len[p.slot], shape = s.bc_locals[p.slot];
    const int n_locals = shape & 0xff, n_main = (shape >> 16) & 0xffff;
    const int32_t* code = s.bc + size_t(p.slot) * 5 * s.bc_stride;
    const int64_t* consts = s.bc_consts + size_t(p.slot) * s.bc_stride;
    const int main_consts = s.code_temps[p.slot];
    const VmView view = vm_view(s);
    int64_t loss = 0;
    uint32_t wrong = 0, errors = 0;
    uint64_t steps = 0;
    for (int c = threadIdx.x; c < s.C; c += kRegionThreads) {
      int64_t value = 0;
      int tag = 0;
      if (run_program_regions(view, s.regions, s.n_regions, code, n, n_main, consts, main_consts, n_locals, c, mine,
                              ws_words, value, tag, steps)) {
        loss += case_loss(s, tag, value, s.expected[c], wrong);
      } else {
        loss += error_loss(s);
        ++wrong;
        ++errors;
      }
    }
    loss = warp_sum(loss);
    wrong = warp_sum(wrong);
    errors = warp_sum(errors);
    steps = warp_sum(steps);
    if (lane == 0) {
      red_loss[warp] = loss;
      red_wrong[warp] = wrong;
      red_errors[warp] = errors;
      red_steps[warp] = steps;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t tl = 0;
      uint32_t tw = 0, te = 0;
      unsigned long long ts = 0;
      for (int w = 0; w < kRegionThreads / 32; ++w) {
        tl += red_loss[w];
        tw += red_wrong[w];
        te += red_errors[w];
        ts += red_steps[w];
      }
      store_result(s, mode, p.slot, tl, tw, te);
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[24]), ts);
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[0]), 1ULL);
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[2]), (unsigned long long)s.C);
    }
    __syncthreads();
  }
}

// Fast VM: persistent warps over the fast list.  Per warp shared memory:
// temporaries (kMaxTemps x K x 32), the staged code (code_stride) and
// constants (stride).
template <int K>
__device__ __forceinline__ void run_k(const SearchDesc& s, int slot, const VmWarpSmem& w, int case_begin,
                                      int case_end, int64_t& loss, uint32_t& wrong, uint64_t& ops) {
  switch (s.n_inputs) {
    case 1: run_accumulator<K, 1>(s, slot, w, case_begin, case_end, loss, wrong, ops); break;
    case 2: run_accumulator<K, 2>(s, slot, w, case_begin, case_end, loss, wrong, ops); break;
    default: run_accumulator<K, 0>(s, slot, w, case_begin, case_end, loss, wrong, ops); break;
  }
}
// One instantiation per cases-per-lane K (each with its own register
// budget); the engine's autotuner picks K per batch shape.  Work items are
// (program, tile of 32 K cases), program-major, so that a round with fewer
// programs than resident warps still fills the GPU; each tile adds its loss
// and wrong count to the program's accumulators and the last tile to finish
// stores the program's result (integer sums: the order does not matter).
template <int K>
__global__ void __launch_bounds__(256, K == 4 ? 2 : 4) k_vm_fast(const SearchDesc* descs, int mode, const ProgramRef* list,
                                                 const int32_t* list_count, int temp_stride, int code_stride,
                                                 int const_stride, int tiles_max) {
  extern __shared__ __align__(16) int64_t smem_vm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  const size_t per_warp = size_t(temp_stride) + size_t(code_stride) + size_t(const_stride);  // int64 units
  int64_t* base = smem_vm + size_t(warp) * per_warp;
  const VmWarpSmem w{base, reinterpret_cast<uint2*>(base + temp_stride), base + temp_stride + code_stride};
  const long long items = (long long)(*list_count) * tiles_max;
  for (long long item = (long long)blockIdx.x * warps + warp; item < items; item += (long long)gridDim.x * warps) {
    const ProgramRef p = list[item / tiles_max];
    const int case0 = int(item % tiles_max) * 32 * K;
    const SearchDesc& s = descs[p.search];
    if (case0 >= s.C) continue;
    int64_t loss = 0;
    uint32_t wrong = 0;
    uint64_t ops = 0;
    run_k<K>(s, p.slot, w, case0, min(s.C, case0 + 32 * K), loss, wrong, ops);
    loss = warp_sum(loss);
    wrong = warp_sum(wrong);
    if (lane == 0) {
      unsigned long long* acc = s.vm_acc + 2 * size_t(p.slot);
      const unsigned tiles = unsigned((s.C + 32 * K - 1) / (32 * K));
      const uint64_t worst = s.metric == GAGP_METRIC_EXACT ? 1 : uint64_t(s.penalty_int);
      bool last;
      int64_t total;
      uint32_t total_wrong;
      if (tiles < 256 && s.C < 65536 && uint64_t(s.C) * worst < (1ULL << 40)) {
        // loss (40 bits), wrong count (16) and finished tiles (8) of the
        // program in one word: one atomic per tile and no fence
        const unsigned long long mine = (unsigned long long)loss | ((unsigned long long)wrong << 40) | (1ULL << 56);
        const unsigned long long sum = atomicAdd(&acc[0], mine) + mine;
        last = unsigned(sum >> 56) == tiles;
        total = int64_t(sum & ((1ULL << 40) - 1));
        total_wrong = uint32_t((sum >> 40) & 0xffffu);
      } else {
        atomicAdd(&acc[0], (unsigned long long)loss);
        __threadfence();
        const unsigned long long before = atomicAdd(&acc[1], (unsigned long long)wrong | (1ULL << 32));
        last = unsigned(before >> 32) == tiles - 1;
        total_wrong = uint32_t(before) + wrong;
        total = 0;
        if (last) {
          __threadfence();
          total = int64_t(atomicAdd(&acc[0], 0ULL));
        }
      }
      if (last) {  // the last tile of the program
        store_result(s, mode, p.slot, total, total_wrong, 0);  // accumulator programs never fail
        // the program's instructions over all its cases, counted once
        atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[3]),
                  (unsigned long long)s.code_len[p.slot] * (unsigned long long)s.C);
        atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[0]), 1ULL);
        atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[2]), (unsigned long long)s.C);
      }
    }
  }
}

// Packed ranking key: (-fitness, wrong, nodes); smaller is better.
__device__ __forceinline__ uint64_t pack_key(const SearchDesc& s, double fitness, uint32_t wrong, uint32_t nodes) {
  const uint64_t loss = uint64_t(-fitness);
  if (!s.has_wrong) return loss;
  return (loss << s.key_shift_wrong) | (uint64_t(wrong) << s.key_shift_nodes) | uint64_t(nodes);
}

// Member statistics after the initial evaluation.
__global__ void k_member_keys(const SearchDesc* descs, const int32_t* off, int n) {
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= off[n]) return;
  const int si = find_search(off, n, item);
  const SearchDesc& s = descs[si];
  const int m = item - off[si];
  const uint32_t nodes = s.has_wrong ? ranking_nodes(s, s.node + size_t(m) * s.stride, len_nodes(s.len[m])) : 0;
  s.nodes[m] = nodes;
  s.key[m] = pack_key(s, s.fitness[m], s.wrong[m], nodes);
}

// ----------------------------------------------------------- run generator
// MT19937-64 (std::mt19937_64, evolve.cpp:339): the published Matsumoto-
// Nishimura generator.  The block regenerates the 312-word state in two
// dependency phases (words below 156 read only old words; words from 156 read
// the new word 156 positions back), tempers and appends the block.
__device__ __forceinline__ uint64_t mt_temper(uint64_t x) {
  x ^= (x >> 29) & 0x5555555555555555ULL;
  x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
  x ^= (x << 37) & 0xFFF7EEE000000000ULL;
  x ^= x >> 43;
  return x;
}
__device__ __forceinline__ uint64_t mt_mix(uint64_t upper_src, uint64_t lower_src, uint64_t far) {
  const uint64_t x = (upper_src & 0xFFFFFFFF80000000ULL) | (lower_src & 0x7FFFFFFFULL);
  return far ^ (x >> 1) ^ ((x & 1) ? 0xB5026F5AA96619E9ULL : 0);
}
// x mod P from a multiply-high quotient estimate (Barrett): the estimate
// is at most two below floor(x / P), so at most two corrections follow.
__device__ __forceinline__ uint32_t mod_p(uint64_t x, uint64_t magic, uint32_t P) {
  const uint64_t q = __umul64hi(x, magic);
  uint64_t r = x - q * P;
  while (r >= P) r -= P;
  return uint32_t(r);
}
// Twists `mt` (smem, 312 words) using scratch `nw` (312 words) and appends
// the tempered block to the stream ring at stream position `wp`.
__device__ inline void mt_block(const SearchDesc& s, uint64_t* mt, uint64_t* nw, long long wp) {
  for (int i = threadIdx.x; i < 156; i += blockDim.x) nw[i] = mt_mix(mt[i], mt[i + 1], mt[i + 156]);
  __syncthreads();
  for (int i = 156 + threadIdx.x; i < 311; i += blockDim.x) nw[i] = mt_mix(mt[i], mt[i + 1], nw[i - 156]);
  __syncthreads();
  if (threadIdx.x == 0) nw[311] = mt_mix(mt[311], nw[0], nw[155]);
  __syncthreads();
  const int base = int(wp % s.stream_capacity);
  for (int i = threadIdx.x; i < 312; i += blockDim.x) {
    mt[i] = nw[i];
    const uint64_t out = mt_temper(nw[i]);
    int pos = base + i;
    if (pos >= s.stream_capacity) pos -= s.stream_capacity;
    s.stream[pos] = out;
    s.stream_mod[pos] = mod_p(out, s.mod_magic, uint32_t(s.P));
  }
  __syncthreads();
}
// Serial fallback of one block, for a consumer that ran ahead of the buffer.
__device__ inline void mt_block_serial(const SearchDesc& s, uint64_t* mt, long long wp) {
  for (int i = 0; i < 312; ++i) mt[i] = mt_mix(mt[i], mt[(i + 1) % 312], mt[(i + 156) % 312]);
  const int base = int(wp % s.stream_capacity);
  for (int i = 0; i < 312; ++i) {
    const uint64_t out = mt_temper(mt[i]);
    int pos = base + i;
    if (pos >= s.stream_capacity) pos -= s.stream_capacity;
    s.stream[pos] = out;
    s.stream_mod[pos] = mod_p(out, s.mod_magic, uint32_t(s.P));
  }
}

// stream_head as two 64-bit counters: [0] read, [1] written
__device__ __forceinline__ long long* stream_ptrs(const SearchDesc& s) { return s.stream_head; }

// Tops up each search's run-generator stream to the next placement's
// 2B+1 draws (as far as the ring allows).  Launched on a side stream so the
// generation overlaps the round's variation, lowering and evaluation; the
// placement kernel waits for it and only generates what redraws add.
__global__ void k_stream(const SearchDesc* descs, int n) {
  __shared__ uint64_t mt[312], nw[312];
  const SearchDesc& s = descs[blockIdx.x];
  if (!search_live(s)) return;
  for (int i = threadIdx.x; i < 312; i += blockDim.x) mt[i] = s.mt[i];
  __syncthreads();
  const long long rp = stream_ptrs(s)[0];
  long long wp = stream_ptrs(s)[1];
  const long long need = (long long)s.B * s.replacement_size + 1;
  while (wp - rp < need && wp - rp + 312 <= s.stream_capacity) {
    mt_block(s, mt, nw, wp);
    wp += 312;
  }
  for (int i = threadIdx.x; i < 312; i += blockDim.x) s.mt[i] = mt[i];
  if (threadIdx.x == 0) stream_ptrs(s)[1] = wp;
}

// The `count` best members in ranking order (smallest (key, member) first),
// written to out[0..count): pass j takes the smallest (key, member) above
// pass j-1's.  For the generational schedule's elites this is the order of
// reproduce's stable sort by completed fitness (phase_population_cpu.cpp:
// 283-288): rank values when wrong counts are kept, fitness with ties to the
// lower index otherwise.  The whole block calls it; out[0] is the best.
__device__ inline void block_best_members(const SearchDesc& s, int count, int32_t* out) {
  __shared__ uint64_t top_key[32];
  __shared__ int top_idx[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, warps = (blockDim.x + 31) >> 5;
  uint64_t prev_key = 0;
  int prev_idx = -1;
  for (int j = 0; j < count; ++j) {
    uint64_t bk = ~0ULL;
    int bi = 0x7fffffff;
    for (int m = threadIdx.x; m < s.P; m += blockDim.x) {
      const uint64_t k = s.key[m];
      const bool above = k > prev_key || (k == prev_key && m > prev_idx);
      if (above && (k < bk || (k == bk && m < bi))) { bk = k; bi = m; }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
      const uint64_t k2 = __shfl_xor_sync(kFull, bk, o);
      const int i2 = __shfl_xor_sync(kFull, bi, o);
      if (k2 < bk || (k2 == bk && i2 < bi)) { bk = k2; bi = i2; }
    }
    if (lane == 0) { top_key[warp] = bk; top_idx[warp] = bi; }
    __syncthreads();
    bk = top_key[0];
    bi = top_idx[0];
    for (int w = 1; w < warps; ++w)
      if (top_key[w] < bk || (top_key[w] == bk && top_idx[w] < bi)) { bk = top_key[w]; bi = top_idx[w]; }
    __syncthreads();
    if (threadIdx.x == 0) out[j] = bi;
    prev_key = bk;
    prev_idx = bi;
  }
}

// Seeds the generator, tops up the stream, finds the best member and draws
// the first round's variation seed.  One block per search.
__global__ void k_start(const SearchDesc* descs, int n) {
  __shared__ uint64_t mt[312], nw[312];
  __shared__ uint64_t best_key[256];
  __shared__ int best_idx[256];
  const SearchDesc& s = descs[blockIdx.x];
  if (s.round[3]) return;
  if (threadIdx.x == 0) {
    mt[0] = s.seed;
    for (int i = 1; i < 312; ++i) mt[i] = 6364136223846793005ULL * (mt[i - 1] ^ (mt[i - 1] >> 62)) + uint64_t(i);
    stream_ptrs(s)[0] = 0;
    stream_ptrs(s)[1] = 0;
  }
  __syncthreads();
  mt_block(s, mt, nw, 0);
  // best member: smallest key, ties to the lowest index
  uint64_t bk = ~0ULL;
  int bi = 0x7fffffff;
  for (int m = threadIdx.x; m < s.P; m += blockDim.x) {
    const uint64_t k = s.key[m];
    if (k < bk || (k == bk && m < bi)) { bk = k; bi = m; }
  }
  best_key[threadIdx.x] = bk;
  best_idx[threadIdx.x] = bi;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int t = 1; t < blockDim.x; ++t)
      if (best_key[t] < bk || (best_key[t] == bk && best_idx[t] < bi)) { bk = best_key[t]; bi = best_idx[t]; }
    s.best[0] = bi;
    s.round_seed[0] = s.stream[0];  // the first run-generator output seeds round 0
    stream_ptrs(s)[0] = 1;
    stream_ptrs(s)[1] = 312;
    s.round[0] = 0;
    s.round[1] = 0;
    s.round[2] = s.total_rounds == 0;
  }
  for (int i = threadIdx.x; i < 312; i += blockDim.x) s.mt[i] = mt[i];
  if (s.generational && s.elite_count > 0) block_best_members(s, s.elite_count, s.elites);
}

// ----------------------------------------------------------- one round
// History entry before every population/batch rounds (record(),
// evolve.cpp:360-371): the best member, its row, and the exact integer sum of
// member fitness (the host forms the long double mean).
__global__ void __launch_bounds__(1024) k_record(const SearchDesc* descs, int n, int only_epoch_start) {
  __shared__ long long partial[1024];
  const SearchDesc& s = descs[blockIdx.x];
  if (!search_live(s)) return;
  const int round = s.round[0];
  if (only_epoch_start && round % s.rounds_per_epoch) return;
  const int entry = s.round[1];
  if (entry >= s.generations) return;
  long long sum = 0;
#pragma unroll 4
  for (int m = threadIdx.x; m < s.P; m += blockDim.x) sum += (long long)s.fitness[m];
  partial[threadIdx.x] = sum;
  __syncthreads();
  for (int w = blockDim.x / 2; w; w >>= 1) {
    if (threadIdx.x < w) partial[threadIdx.x] += partial[threadIdx.x + w];
    __syncthreads();
  }
  const int b = s.best[0];
  const int32_t l = s.len[b];
  for (int i = threadIdx.x; i < len_nodes(l); i += blockDim.x)
    s.hist_node[size_t(entry) * s.stride + i] = s.node[size_t(b) * s.stride + i];
  for (int i = threadIdx.x; i < len_consts(l); i += blockDim.x)
    s.hist_cval[size_t(entry) * s.stride + i] = s.cval[size_t(b) * s.stride + i];
  if (threadIdx.x == 0) {
    s.hist_sum[entry] = partial[0];
    s.hist_fitness[entry] = s.fitness[b];
    s.hist_wrong[entry] = s.wrong[b];
    s.hist_nodes[entry] = uint32_t(s.fixed_nodes + len_nodes(l));
    s.hist_len[entry] = l;
    s.round[1] = entry + 1;
  }
}

// The round's member index (HostPhasePopulation's member_hashes, kept
// current by commit_batch, phase_population_cpu.cpp:318-321,382-394): a warp
// per member hashes its row and inserts it by linear probing unless an
// identical row is indexed already, so every distinct row has one entry and
// the probe runs stay short however many copies the population holds.  A
// slot word carries the hash's top bits with the member, so a warp that
// loses a slot to another compares tags and then rows (stable in memory
// all round) without waiting for any other write.  At most P entries in at
// least 2P slots: every probe sequence meets an empty slot.  k_commit clears
// the table for the next round.
__global__ void __launch_bounds__(256) k_member_index(const SearchDesc* descs, const int32_t* off, int n) {
  const int item = int((size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  if (item >= off[n]) return;
  const int si = find_search(off, n, item);
  const SearchDesc& s = descs[si];
  if (!search_live(s) || !s.mtab) return;
  const int m = item - off[si];
  const int32_t l = s.len[m];
  const uint64_t* node = s.node + size_t(m) * s.stride;
  const int64_t* cval = s.cval + size_t(m) * s.stride;
  const uint64_t h = warp_row_hash(node, cval, len_nodes(l), len_consts(l));
  const unsigned long long mine = index_word(h, m);
  const uint32_t mask = uint32_t(s.mtab_mask);
  uint32_t slot = uint32_t(h) & mask;
  for (uint32_t probe = 0; probe <= mask; ++probe) {
    unsigned long long cur = 0;
    if (lane == 0) cur = atomicCAS(&s.mtab[slot], 0ULL, mine);
    cur = __shfl_sync(kFull, cur, 0);
    if (!cur) return;  // indexed
    if (index_tag_matches(cur, h)) {
      const int other = index_member(cur);
      const int32_t lc = s.len[other];
      if (warp_rows_equal(s.node + size_t(other) * s.stride, s.cval + size_t(other) * s.stride, len_nodes(lc),
                          len_consts(lc), node, cval, len_nodes(l), len_consts(l)))
        return;  // an identical row is indexed already
    }
    slot = (slot + 1) & mask;
  }
}

// make_batch (phase_population_cpu.cpp:322-353): one warp per child, rows
// staged in dynamic shared memory (warp_rows_bytes(stride) per warp).
// Persistent warps over the batch items [lo, hi): each warp takes the next
// child from `next_item` (zeroed before the launch) until the range is
// varied, so warps that drew short children go on to the next one instead
// of idling.  When the range's children all belong to search `staged`, the
// block first copies that search's generator image (image_bytes) into
// shared memory after the rows: a generation step is a chain of dependent
// table lookups, each a shared-memory load instead of a global one.
__global__ void __launch_bounds__(128, 6) k_vary(const SearchDesc* descs, const int32_t* off, int n, int stride_max,
                                                 int32_t* next_item, int lo, int hi, int collect_stats, int staged,
                                                 int image_bytes) {
  extern __shared__ __align__(16) char smem_rows[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  char* base = smem_rows + size_t(warp) * warp_rows_bytes(stride_max);
  char* image = smem_rows + size_t(blockDim.x >> 5) * warp_rows_bytes(stride_max);
  if (staged >= 0) {
    const uint4* from = reinterpret_cast<const uint4*>(descs[staged].gen_image);
    uint4* to = reinterpret_cast<uint4*>(image);
    for (int i = threadIdx.x; i < image_bytes / 16; i += blockDim.x) to[i] = from[i];
    __syncthreads();
  }
  const int total = min(off[n], hi);
  for (;;) {
    int item = 0;
    if (lane == 0) item = lo + atomicAdd(next_item, 1);
    item = __shfl_sync(kFull, item, 0);
    if (item >= total) break;
    const int si = find_search(off, n, item);
    const SearchDesc& s = descs[si];
    if (!search_live(s)) continue;
    const int child = item - off[si];
    WarpRows rows = carve_rows(base, s.stride);
    int reuse = -1, parent = -1;
    long long stamp[5] = {0, 0, 0, 0, 0};
    const long long started = clock64();
    const int error = warp_vary_child(s, si == staged ? image : s.gen_image, child, s.round_seed[0], rows, &reuse,
                                      &parent, stamp);
    if (lane == 0 && collect_stats) {
      // per-phase SM cycles: selection, crossover, subtree generation, rest
      stamp[3] = clock64();
      long long prev = started;
      for (int k = 0; k < 4; ++k) {
        if (stamp[k] == 0) stamp[k] = prev;
        atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[10 + k]), (unsigned long long)(stamp[k] - prev));
        atomicMax(reinterpret_cast<unsigned long long*>(&s.counters[16 + k]), (unsigned long long)(stamp[k] - prev));
        prev = stamp[k];
      }
      atomicMax(reinterpret_cast<unsigned long long*>(&s.counters[15]), (unsigned long long)(stamp[3] - started));
      if (stamp[3] - started > 200000) atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[20]), 1ULL);
      if (stamp[4]) {
        atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[21]), (unsigned long long)(stamp[4] - 1));
        atomicMax(reinterpret_cast<unsigned long long*>(&s.counters[22]), (unsigned long long)(stamp[4] - 1));
        atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[23]), 1ULL);
      }
      // rows read (parent, donor) and written (child) with their lengths,
      // 2 x pressure tournament keys, four per-child outputs
      const uint64_t bytes = 8ull * (rows.parent.n + rows.parent.nc + rows.donor.n + rows.donor.nc + rows.child.n +
                                     rows.child.nc + 2 * s.pressure) + 12 + 16;
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[8]), (unsigned long long)bytes);
    }
    if (lane == 0) {
      s.c_parent[child] = parent;
      s.c_reuse[child] = reuse;
      s.c_error[child] = error;
      s.c_eval[child] = error == 0 && reuse < 0;
      if (error) raise_error(s, 100 + error);
    }
    __syncwarp();
  }
}

// State of every search of a batch in one array (bit 0: finished, bit 1:
// failed), so that a serving step reads them with one copy.
__global__ void k_status(const SearchDesc* descs, int n, int32_t* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const SearchDesc& s = descs[i];
  out[i] = (s.round[2] ? 1 : 0) | (s.round[3] ? 2 : 0);
}

// Cluster placement shape (k_place_levels, k_place_cluster): kPlaceCtas
// blocks of kClusterThreads threads, kClusterPer children per thread, for
// rounds of at least kClusterMinChildren children.
constexpr int kPlaceCtas = 8;
constexpr int kClusterThreads = 1024;
constexpr int kClusterPer = 2;
constexpr int kClusterMinChildren = 4096;

// A child's result and ranking key before any placement (evolve.cpp:403-413):
// an unchanged genotype takes its parent's.  Returns the key; reports a
// reuse through `reused`.
__device__ inline uint64_t child_result_of(const SearchDesc& s, int b, bool* reused) {
  const int source = s.c_reuse[b];
  double f;
  uint32_t w, nodes;
  *reused = source >= 0;
  if (source >= 0) {
    f = s.fitness[source];
    w = s.wrong[source];
    nodes = s.nodes[source];
  } else {
    f = s.c_fitness[b];
    w = s.c_wrong[b];
    nodes = s.has_wrong ? ranking_nodes(s, s.cnode + size_t(b) * s.stride, len_nodes(s.clen[b])) : 0;
  }
  s.c_fitness[b] = f;
  s.c_wrong[b] = w;
  s.c_nodes[b] = nodes;
  const uint64_t key = pack_key(s, f, w, nodes);
  s.c_key[b] = key;
  return key;
}
__device__ inline void child_result(const SearchDesc& s, int b) {
  bool reused;
  child_result_of(s, b, &reused);
  if (reused) {
    atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[1]), 1ULL);
    // the generational evaluate copies a reused member's case counts too
    // (HostPhasePopulation::evaluate, phase_population_cpu.cpp:252-253), so
    // its program-case total covers every member
    if (s.generational) atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[2]), (unsigned long long)s.C);
  }
}

// Results of all children before any placement, thread per child, for
// rounds that the single-block placement takes.
__global__ void k_child_results(const SearchDesc* descs, const int32_t* off, int n) {
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= off[n]) return;
  const int si = find_search(off, n, item);
  const SearchDesc& s = descs[si];
  if (!search_live(s)) return;
  if (s.B >= kClusterMinChildren && !s.generational) return;  // the cluster placement forms these
  const int b = item - off[si];
  child_result(s, b);
}


// Windowed placement step over lanes [seg_begin, seg_end) of a window whose
// children's draws do not overlap (every lane's members differ from every
// earlier active lane's): victims from the current keys equal the
// sequential ones, the best member before each lane is an exclusive prefix
// minimum of (key, member), and the lanes commit up to the first whose
// victim is the current best (a redraw).  Returns the committed count.
__device__ __forceinline__ int place_segment(uint64_t* keys, int32_t* placed, int b0, int seg_begin, int seg_end,
                                             int d0, int d1, uint64_t ck, int& best, uint64_t& best_key) {
  const int lane = threadIdx.x & 31;
  const bool live = lane >= seg_begin && lane < seg_end;
  const uint64_t k0 = live ? keys[d0] : 0, k1 = live ? keys[d1] : 0;
  // worst of the pair: the second replaces the first when the first is better
  const int v = (k0 < k1 || (k0 == k1 && d0 < d1)) ? d1 : d0;
  uint64_t pk = live ? ck : ~0ULL;
  int pv = live ? v : 0x7fffffff;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t uk = __shfl_up_sync(kFull, pk, o);
    const int uv = __shfl_up_sync(kFull, pv, o);
    if (lane >= o && (uk < pk || (uk == pk && uv < pv))) { pk = uk; pv = uv; }
  }
  uint64_t ek = __shfl_up_sync(kFull, pk, 1);
  int ev = __shfl_up_sync(kFull, pv, 1);
  if (lane == 0 || best_key < ek || (best_key == ek && best < ev)) { ek = best_key; ev = best; }
  const unsigned rmask = __ballot_sync(kFull, live && v == ev);
  const int stop = rmask ? __ffs(rmask) - 1 : seg_end;
  const int valid = stop - seg_begin;
  if (valid <= 0) return 0;
  if (live && lane < stop) {
    keys[v] = ck;
    placed[v] = b0 + lane;
  }
  uint64_t nk = __shfl_sync(kFull, pk, stop - 1);
  int nv = __shfl_sync(kFull, pv, stop - 1);
  if (best_key < nk || (best_key == nk && best < nv)) { nk = best_key; nv = best; }
  best_key = nk;
  best = nv;
  __syncwarp();
  return valid;
}

// Lanes of a 32-child window whose draws overlap an earlier lane's: bit j
// set when child j draws a member that some child i < j of the window drew.
__device__ __forceinline__ int latest_overlap(int d0, int d1) {
  const int lane = threadIdx.x & 31;
  int latest = -1;
#pragma unroll 8
  for (int o = 1; o < 32; ++o) {
    const int e0 = __shfl_up_sync(kFull, d0, o), e1 = __shfl_up_sync(kFull, d1, o);
    if (lane >= o && ((e0 == d0) | (e0 == d1) | (e1 == d0) | (e1 == d1))) latest = max(latest, lane - o);
  }
  return latest;
}

// Steady-state placement (evolve.cpp:414-427): children in order, each
// replacing the worst of replacement_size uniform draws (redrawn when it is
// the current best).  One block per search; `dyn_bytes`: dynamic shared
// memory of the launch (member keys, then the level owners or staged draws).
//
// Level-parallel path (replacement size 2): without a redraw child j draws
// stream positions 2j and 2j+1.  A child is ready once it is the earliest
// unplaced child drawing each of its members; the ready children of a level
// draw disjoint members, so they read exactly the keys the sequential loop
// would and place at once.  The best member before each child is then a
// prefix minimum of (key, member) in child order; a child whose victim is
// that best member would have redrawn (both its draws are the best member),
// and then the round is replayed on the exact windowed path.
//
// Windowed path (warp 0): 32 children per step, one per lane, over draws
// staged in shared memory; a step commits the lanes before the first lane
// drawing a member an earlier lane drew, or before the first redraw, which
// the sequential loop then takes.  Other replacement sizes and the end of
// the staged draws run the sequential loop.
// Finally the next round's seed is drawn.
constexpr int kPlaceThreads = 1024;
__device__ __forceinline__ bool key_before(uint64_t ka, int va, uint64_t kb, int vb) {
  return ka < kb || (ka == kb && va < vb);
}
// after_cluster: the cluster placement ran first; return if it placed the
// round (place_state 1), replay it on the exact windowed path if it found a
// redraw (2), or place it here if it did not take it (0).
__global__ void __launch_bounds__(kPlaceThreads, 1) k_place(const SearchDesc* descs, int n, int dyn_bytes,
                                                            int after_cluster) {
  extern __shared__ __align__(16) uint64_t keys[];
  __shared__ uint64_t mt[312], nw[312];
  __shared__ uint64_t ck_stage[1024];
  __shared__ uint64_t scan_key[32];
  __shared__ int scan_idx[32];
  __shared__ long long shared_pos, shared_wp;
  __shared__ int shared_best, shared_fail, ready_count[2], redraw_at;
  const SearchDesc& s = descs[blockIdx.x];
  if (!search_live(s)) return;
  const int cluster_state = after_cluster ? *s.place_state : 0;
  if (cluster_state == 1) return;
  const long long t0 = clock64();
  const int P = s.P, B = s.B, rs = s.replacement_size, cap = s.stream_capacity;
  const int tid = threadIdx.x;
  int32_t* __restrict__ placed = s.placed;
  for (int m = tid; m < P; m += blockDim.x) {
    keys[m] = s.key[m];
    placed[m] = -1;
  }
  for (int i = tid; i < 312; i += blockDim.x) mt[i] = s.mt[i];
  __syncthreads();
  const long long rp = stream_ptrs(s)[0];
  long long wp = stream_ptrs(s)[1];
  const long long need = (long long)B * rs + 1;
  while (wp - rp < need && wp - rp + 312 <= cap) {
    mt_block(s, mt, nw, wp);
    wp += 312;
  }
  const long long t1 = clock64();
  // ---------------------------------------------------- level-parallel path
  constexpr int kPerThread = 16;
  // owner area after the keys, 16-byte aligned, with 64 bytes of slack for
  // the per-thread 16-byte reads of the staged draws
  int32_t* owner = reinterpret_cast<int32_t*>(keys + P + (P & 1));
  const bool parallel_path = cluster_state == 0 && rs == 2 && blockDim.x == kPlaceThreads &&
                             B <= kPlaceThreads * kPerThread &&
                             wp - rp >= need &&
                             dyn_bytes >= int(sizeof(uint64_t)) * (P + 1) + int(sizeof(int32_t)) * P + 64;
  bool parallel_done = false;
  if (parallel_path) {
    // thread tid owns children [16 tid, 16 tid + 16): cand[t] holds child
    // begin + t's two draws, and once it is placed, its victim
    const int base = int(rp % cap);
    const int begin = tid * kPerThread;
    constexpr int kBatch = 4;  // child keys loaded together
    const uint64_t* __restrict__ ckey = s.c_key;
    // the 2B draws (residues < P <= 65536), staged as 16-bit values in the
    // owner area with coalesced loads, then read back per thread: child j's
    // pair is the 32-bit word j
    {
      uint16_t* stage = reinterpret_cast<uint16_t*>(owner);
      const uint32_t* __restrict__ smod = s.stream_mod;
      for (int i = tid; i < 2 * B; i += blockDim.x) {
        int pos = base + i;
        if (pos >= cap) pos -= cap;
        stage[i] = uint16_t(smod[pos]);
      }
    }
    __syncthreads();
    uint32_t cand[kPerThread];
    uint32_t pending = 0;
    {
      static_assert(kPerThread % 4 == 0, "draw pairs are read four at a time");
      const uint4* pairs = reinterpret_cast<const uint4*>(owner) + size_t(begin) / 4;
#pragma unroll
      for (int q = 0; q < kPerThread / 4; ++q) {
        const uint4 v = begin < B ? pairs[q] : make_uint4(0, 0, 0, 0);
        cand[4 * q] = v.x;
        cand[4 * q + 1] = v.y;
        cand[4 * q + 2] = v.z;
        cand[4 * q + 3] = v.w;
      }
#pragma unroll
      for (int t = 0; t < kPerThread; ++t) {
        if (begin + t < B) pending |= 1u << t;
        else cand[t] = 0;
      }
    }
    __syncthreads();  // the owner area is reset below
    // owner[m]: the earliest child of the current level that drew member m,
    // tagged with the level so that no per-level reset is needed (a later
    // level's tag is smaller than every earlier one's)
    for (int m = tid; m < P; m += blockDim.x) owner[m] = 0x7fffffff;
    if (tid == 0) {
      ready_count[0] = ready_count[1] = 0;
      redraw_at = 0x7fffffff;
    }
    __syncthreads();
    int levels_run = 0, left = B;
    const long long level_start = clock64();
    for (int level = 0; level <= B; ++level) {
      ++levels_run;
      const int tag = (0x7fff - level) << 16;
#pragma unroll
      for (int t = 0; t < kPerThread; ++t)
        if (pending >> t & 1) {
          atomicMin(&owner[cand[t] & 0xffff], tag | (begin + t));
          atomicMin(&owner[cand[t] >> 16], tag | (begin + t));
        }
      __syncthreads();
      // children owning both their members are placed at this level; they
      // touch disjoint members, so their order within the level is free
      uint32_t ready = 0;
#pragma unroll
      for (int t = 0; t < kPerThread; ++t)
        if ((pending >> t & 1) && owner[cand[t] & 0xffff] == (tag | (begin + t)) &&
            owner[cand[t] >> 16] == (tag | (begin + t)))
          ready |= 1u << t;
      if (ready) {
#pragma unroll
        for (int h = 0; h < kPerThread; h += kBatch) {
          uint64_t kv[kBatch];
#pragma unroll
          for (int u = 0; u < kBatch; ++u) kv[u] = (ready >> (h + u) & 1) ? ckey[begin + h + u] : 0;
#pragma unroll
          for (int u = 0; u < kBatch; ++u)
            if (ready >> (h + u) & 1) {
              const int d0 = int(cand[h + u] & 0xffff), d1 = int(cand[h + u] >> 16);
              const uint64_t k0 = keys[d0], k1 = keys[d1];
              // worst of the pair: the second replaces the first when the first is better
              const int v = (k0 < k1 || (k0 == k1 && d0 < d1)) ? d1 : d0;
              keys[v] = kv[u];
              placed[v] = begin + h + u;
              cand[h + u] = uint32_t(v);
            }
        }
        pending &= ~ready;
      }
      {
        // one shared-memory atomic per warp, not per thread
        int placed_here = __popc(ready);
        for (int o = 16; o; o >>= 1) placed_here += __shfl_xor_sync(kFull, placed_here, o);
        if ((tid & 31) == 0 && placed_here) atomicAdd(&ready_count[level & 1], placed_here);
      }
      if (tid == 0) ready_count[(level + 1) & 1] = 0;  // read by every thread before this level's first barrier
      __syncthreads();
      left -= ready_count[level & 1];
      if (left == 0) break;
    }
    const int level_left = left;
    if (tid == 0)
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[14]), (unsigned long long)(clock64() - level_start));
    // best member before each child (child order): each thread's minimum of
    // (key, victim) over its children, a warp-shuffle scan, then a scan of
    // the warp totals, gives each thread's incoming best
    const int lane = tid & 31, warp = tid >> 5;
    uint64_t mk = ~0ULL;
    int mv = 0x7fffffff;
#pragma unroll
    for (int h = 0; h < kPerThread; h += kBatch) {
      uint64_t kv[kBatch];
#pragma unroll
      for (int u = 0; u < kBatch; ++u) kv[u] = begin + h + u < B ? ckey[begin + h + u] : ~0ULL;
#pragma unroll
      for (int u = 0; u < kBatch; ++u)
        if (begin + h + u < B && key_before(kv[u], int(cand[h + u]), mk, mv)) {
          mk = kv[u];
          mv = int(cand[h + u]);
        }
    }
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t uk = __shfl_up_sync(kFull, mk, o);
      const int uv = __shfl_up_sync(kFull, mv, o);
      if (lane >= o && key_before(uk, uv, mk, mv)) { mk = uk; mv = uv; }
    }
    constexpr int kWarps = kPlaceThreads / 32;
    if (lane == 31) { scan_key[warp] = mk; scan_idx[warp] = mv; }
    __syncthreads();
    if (warp == 0) {
      uint64_t wk = lane < kWarps ? scan_key[lane] : ~0ULL;
      int wv = lane < kWarps ? scan_idx[lane] : 0x7fffffff;
      for (int o = 1; o < 32; o <<= 1) {
        const uint64_t uk = __shfl_up_sync(kFull, wk, o);
        const int uv = __shfl_up_sync(kFull, wv, o);
        if (lane >= o && key_before(uk, uv, wk, wv)) { wk = uk; wv = uv; }
      }
      scan_key[lane] = wk;
      scan_idx[lane] = wv;
    }
    __syncthreads();
    const int best0 = s.best[0];
    const uint64_t best0_key = s.key[best0];
    int bv = best0;
    uint64_t bk = best0_key;
    {
      const uint64_t lk = __shfl_up_sync(kFull, mk, 1);
      const int lv = __shfl_up_sync(kFull, mv, 1);
      if (lane > 0 && key_before(lk, lv, bk, bv)) { bk = lk; bv = lv; }
      if (warp > 0 && key_before(scan_key[warp - 1], scan_idx[warp - 1], bk, bv)) {
        bk = scan_key[warp - 1];
        bv = scan_idx[warp - 1];
      }
    }
    // a child whose victim is the best member before it would have redrawn
    bool hit = false;
#pragma unroll
    for (int h = 0; h < kPerThread; h += kBatch) {
      uint64_t kv[kBatch];
#pragma unroll
      for (int u = 0; u < kBatch; ++u) kv[u] = begin + h + u < B ? ckey[begin + h + u] : 0;
#pragma unroll
      for (int u = 0; u < kBatch; ++u)
        if (!hit && begin + h + u < B) {
          const int v = int(cand[h + u]);
          if (v == bv) {
            atomicMin(&redraw_at, begin + h + u);
            hit = true;
          } else if (key_before(kv[u], v, bk, bv)) {
            bk = kv[u];
            bv = v;
          }
        }
    }
    __syncthreads();
    parallel_done = redraw_at == 0x7fffffff;
    if (tid == 0)  // levels of the parallel path; a replay adds 2^20
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[7]),
                (unsigned long long)(B - level_left >= 0 ? levels_run : 0) + (parallel_done ? 0ULL : (1ULL << 20)));
    if (parallel_done) {
      if (tid == 0) {
        int fv = best0;
        uint64_t fk = best0_key;
        if (key_before(scan_key[kWarps - 1], scan_idx[kWarps - 1], fk, fv)) {
          fk = scan_key[kWarps - 1];
          fv = scan_idx[kWarps - 1];
        }
        shared_best = fv;
        shared_fail = 0;
        // the next round's seed: the raw output after the 2B placement draws
        const long long pos = rp + 2LL * B;
        s.round_seed[0] = s.stream[pos % cap];
        shared_pos = pos + 1;
        shared_wp = wp;
      }
    } else {
      // replay the round on the exact windowed path from the round's keys
      for (int m = tid; m < P; m += blockDim.x) {
        keys[m] = s.key[m];
        placed[m] = -1;
      }
    }
    __syncthreads();
  }
  // ---------------------------------------------------- windowed path
  uint16_t* draws = reinterpret_cast<uint16_t*>(keys + P);
  const int slots = (dyn_bytes - int(sizeof(uint64_t)) * P) / int(sizeof(uint16_t));
  const int avail = int(min((long long)slots, wp - rp));
  if (!parallel_done) {
    const int base = int(rp % cap);
    for (int i = tid; i < avail; i += blockDim.x) {
      int pos = base + i;
      if (pos >= cap) pos -= cap;
      draws[i] = uint16_t(s.stream_mod[pos]);
    }
  }
  __syncthreads();
  const long long t2 = clock64();
  if (!parallel_done && tid < 32) {
    const int lane = tid;
    const uint32_t* __restrict__ smod = s.stream_mod;
    const uint64_t* __restrict__ ckey = s.c_key;
    long long gen_wp = wp;
    int best = s.best[0];
    uint64_t best_key = keys[best];
    int di = 0, b = 0;
    int failed = 0;
    int stage_begin = 0, stage_end = 0;
    auto stage = [&]() {  // child keys [b, b + 1024) into shared memory
      __syncwarp();
      stage_begin = b;
      stage_end = min(B, b + 1024);
      for (int i = lane; i < stage_end - stage_begin; i += 32) ck_stage[i] = ckey[stage_begin + i];
      __syncwarp();
    };
    while (b < B && !failed) {
      while (rs == 2 && b < B && di + 64 <= avail) {
        if (b + 32 > stage_end) stage();
        const int cnt = min(32, B - b);
        const bool live = lane < cnt;
        const int d0 = live ? int(draws[di + 2 * lane]) : -1 - 2 * lane;
        const int d1 = live ? int(draws[di + 2 * lane + 1]) : -2 - 2 * lane;
        const int latest = latest_overlap(d0, d1);
        const unsigned omask = __ballot_sync(kFull, live && latest >= 0);
        const int first_overlap = omask ? __ffs(omask) - 1 : cnt;
        const uint64_t ck = live ? ck_stage[b - stage_begin + lane] : ~0ULL;
        const int valid = place_segment(keys, placed, b, 0, first_overlap, max(d0, 0), max(d1, 0), ck, best,
                                        best_key);
        if (valid == 0) break;  // lane 0's victim is the best: the sequential loop redraws
        b += valid;
        di += 2 * valid;
      }
      if (b >= B) break;
      // sequential placement (lane 0): one child after a window stop, or every
      // remaining child past the staged draws / with another replacement size
      __syncwarp();
      if (lane == 0) {
        auto draw = [&](int idx) -> int {
          if (idx < avail) return draws[idx];
          const long long pos = rp + idx;
          while (pos >= gen_wp) {  // ran ahead of the buffer: one serial block
            mt_block_serial(s, mt, gen_wp);
            gen_wp += 312;
          }
          return int(smod[pos % cap]);
        };
        const bool rest = rs != 2 || di + 64 > avail;
        do {
          const uint64_t ck = ckey[b];
          int v = -1;
          for (int guard = 0; guard < (1 << 20); ++guard) {
            int worst = draw(di++);
            uint64_t kw = keys[worst];
            for (int i = 1; i < rs; ++i) {
              const int c = draw(di++);
              const uint64_t kc = keys[c];
              if (kw < kc || (kw == kc && worst < c)) { worst = c; kw = kc; }
            }
            if (worst != best) { v = worst; break; }
          }
          if (v < 0) { failed = 1; break; }
          keys[v] = ck;
          placed[v] = b;
          if (ck < best_key || (ck == best_key && v < best)) { best = v; best_key = ck; }
          ++b;
        } while (rest && b < B);
      }
      __syncwarp();
      b = __shfl_sync(kFull, b, 0);
      di = __shfl_sync(kFull, di, 0);
      best = __shfl_sync(kFull, best, 0);
      best_key = __shfl_sync(kFull, best_key, 0);
      gen_wp = __shfl_sync(kFull, gen_wp, 0);
      failed = __shfl_sync(kFull, failed, 0);
    }
    __syncwarp();
    if (lane == 0) {
      // the next round's variation seed: the raw output at the next position
      const long long pos = rp + di;
      while (pos >= gen_wp) {
        mt_block_serial(s, mt, gen_wp);
        gen_wp += 312;
      }
      s.round_seed[0] = s.stream[pos % cap];
      shared_best = best;
      shared_pos = pos + 1;
      shared_wp = gen_wp;
      shared_fail = failed;
    }
  }
  __syncthreads();
  const long long t3 = clock64();
  if (tid == 0) {
    if (shared_fail) raise_error(s, 40);
    s.best[0] = shared_best;
    stream_ptrs(s)[0] = shared_pos;
    stream_ptrs(s)[1] = shared_wp;
  }
  for (int i = tid; i < 312; i += blockDim.x) s.mt[i] = mt[i];
  {
    // placed members take their child's statistics; four members' loads in flight at once
    const double* __restrict__ cfit = s.c_fitness;
    const uint32_t* __restrict__ cwrong = s.c_wrong;
    const uint32_t* __restrict__ cnodes = s.c_nodes;
    const int stride = blockDim.x;
    for (int m0 = tid; m0 < P; m0 += 4 * stride) {
      int c[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) c[u] = m0 + u * stride < P ? placed[m0 + u * stride] : -1;
      double f[4];
      uint32_t w[4], nd[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (c[u] >= 0) {
          f[u] = cfit[c[u]];
          w[u] = cwrong[c[u]];
          nd[u] = cnodes[c[u]];
        }
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (c[u] >= 0) {
          const int m = m0 + u * stride;
          s.key[m] = keys[m];
          s.fitness[m] = f[u];
          s.wrong[m] = w[u];
          s.nodes[m] = nd[u];
        }
    }
  }
  if (tid == 0) {
    const int r = s.round[0] + 1;
    s.round[0] = r;
    if (r >= s.total_rounds) s.round[2] = 1;
    // SM clock cycles of the placement phases: generation, parallel
    // placement (and draw staging), windowed placement
    atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[4]), (unsigned long long)(t1 - t0));
    atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[5]), (unsigned long long)(t2 - t1));
    atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[6]), (unsigned long long)(t3 - t2));
  }
}

// Cluster placement: the level-parallel placement above, spread over a
// cluster of kPlaceCtas blocks that share their shared memory.  Member m
// lives in block m % kPlaceCtas (its key and level owner); thread g of the
// cluster owns children [2g, 2g + 2), so the blocks hold the children in
// order.  Each level is two cluster barriers: level-tagged atomicMin on the
// owning block's owner word, then the ready children place (remote key
// reads and writes).  The running best before each child is a scan inside
// each block plus a prefix over the blocks' totals.  When a child would have
// redrawn, nothing is written back (place_state 2) and k_place replays the
// round on the exact path; a batch of fewer than kClusterMinChildren
// children, another replacement size or a stream short of draws is left to
// k_place (place_state 0), whose single block is then as fast.  On success
// this kernel finishes the round as k_place does (statistics, best member,
// stream position, next seed).
// Whether a round of search s is placed by the cluster (the same answer in
// every block and in both cluster kernels of the round).
__device__ __forceinline__ bool cluster_placement_applies(const SearchDesc& s, long long rp, long long wp) {
  return s.replacement_size == 2 && s.B >= kClusterMinChildren && s.B <= kPlaceCtas * kClusterThreads * kClusterPer &&
         wp - rp >= 2LL * s.B + 1;
}

// The children's two drawn members for this round, from the run generator's
// residues (draws 2j and 2j + 1 after the read position).
__device__ __forceinline__ uint32_t child_draws(const SearchDesc& s, int base, int j) {
  const int cap = s.stream_capacity;
  int p0 = base + 2 * j, p1 = p0 + 1;
  if (p0 >= cap) p0 -= cap;
  if (p1 >= cap) p1 -= cap;
  return s.stream_mod[p0] | (s.stream_mod[p1] << 16);
}

// Placement levels of a round, found before the children's keys exist.  A
// child can be placed once every earlier child that drew one of its members
// is placed: its level is one more than the largest level among those, which
// depends on the draws alone.  So this runs on the side stream, once the run
// generator has topped up the stream, while the children are still being
// varied and evaluated; k_place_cluster then only compares and writes keys,
// level by level.  Levels are found as the placement would find them: each
// level, every pending child claims both its members with a level-tagged
// atomicMin on the owning block's owner word (member m lives in block
// m % kPlaceCtas), and a child that owns both is at this level.  The owner
// words alternate between two arrays by level parity: a thread that has
// moved on to level L + 1 claims in the other array, so its claims never
// disturb a slower thread still checking level L (and the array of level L
// is claimed again only after barrier L + 1, which every check of level L
// precedes).  The levels are therefore the exact longest-path levels,
// whatever the timing.
// level_plan: [0] the round + 1 the levels belong to, [1] their number.
__global__ void __cluster_dims__(kPlaceCtas, 1, 1) __launch_bounds__(kClusterThreads, 1)
    k_place_levels(const SearchDesc* descs, int n) {
  extern __shared__ __align__(16) int32_t lv_owner[];
  __shared__ int ready_count[3];
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = int(cluster.block_rank());
  const SearchDesc& s = descs[blockIdx.x / kPlaceCtas];
  if (!search_live(s)) return;  // the same for every block of the cluster
  const int P = s.P, B = s.B;
  const int tid = threadIdx.x, lane = tid & 31;
  const long long rp = stream_ptrs(s)[0], wp = stream_ptrs(s)[1];
  if (!cluster_placement_applies(s, rp, wp)) return;
  const int local_P = (P + kPlaceCtas - 1) / kPlaceCtas;
  for (int i = tid; i < 2 * local_P; i += blockDim.x) lv_owner[i] = 0x7fffffff;
  if (tid == 0) ready_count[0] = ready_count[1] = ready_count[2] = 0;
  const int begin = (rank * kClusterThreads + tid) * kClusterPer;
  const int base = int(rp % s.stream_capacity);
  uint32_t cand[kClusterPer];
  uint32_t pending = 0;
#pragma unroll
  for (int t = 0; t < kClusterPer; ++t) {
    cand[t] = 0;
    if (begin + t < B) {
      cand[t] = child_draws(s, base, begin + t);
      pending |= 1u << t;
    }
  }
  // owner word of member m for levels of parity `par`
  auto owner_at = [&](int m, int par) -> int* {
    return cluster.map_shared_rank(lv_owner, m % kPlaceCtas) + par * local_P + m / kPlaceCtas;
  };
  int* counter0 = cluster.map_shared_rank(ready_count, 0);
  int16_t* __restrict__ level_of = s.child_level;
  cluster.sync();
  // one cluster barrier per level (count slots rotate as in k_place_cluster)
  int left = B, level = 0;
  for (; level <= B; ++level) {
    const int tag = (0x7fff - level) << 16, par = level & 1;
#pragma unroll
    for (int t = 0; t < kClusterPer; ++t)
      if (pending >> t & 1) {
        atomicMin(owner_at(int(cand[t] & 0xffff), par), tag | (begin + t));
        atomicMin(owner_at(int(cand[t] >> 16), par), tag | (begin + t));
      }
    cluster.sync();
    if (level > 0) {
      left -= counter0[(level - 1) % 3];
      if (left == 0) break;
    }
    if (rank == 0 && tid == 0) ready_count[(level + 1) % 3] = 0;
    uint32_t ready = 0;
#pragma unroll
    for (int t = 0; t < kClusterPer; ++t)
      if ((pending >> t & 1) && *owner_at(int(cand[t] & 0xffff), par) == (tag | (begin + t)) &&
          *owner_at(int(cand[t] >> 16), par) == (tag | (begin + t))) {
        ready |= 1u << t;
        level_of[begin + t] = int16_t(level);
      }
    pending &= ~ready;
    int placed_here = __popc(ready);
    for (int o = 16; o; o >>= 1) placed_here += __shfl_xor_sync(kFull, placed_here, o);
    if (lane == 0 && placed_here) atomicAdd(counter0 + level % 3, placed_here);
  }
  if (rank == 0 && tid == 0) {
    s.level_plan[1] = level;  // levels 0 .. level - 1 hold every child
    s.level_plan[0] = s.round[0] + 1;
  }
  cluster.sync();  // no block leaves while another may still read its shared memory
}

__global__ void __cluster_dims__(kPlaceCtas, 1, 1) __launch_bounds__(kClusterThreads, 1)
    k_place_cluster(const SearchDesc* descs, int n) {
  extern __shared__ __align__(16) uint64_t cl_keys[];
  __shared__ uint64_t scan_key[32];
  __shared__ int scan_idx[32];
  __shared__ uint64_t cta_key[kPlaceCtas];  // block totals (read from block 0)
  __shared__ int cta_idx[kPlaceCtas];
  __shared__ int redraw_at;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = int(cluster.block_rank());
  const SearchDesc& s = descs[blockIdx.x / kPlaceCtas];
  if (!search_live(s)) return;  // the same for every block of the cluster
  const long long t0 = clock64();
  const int P = s.P, B = s.B, cap = s.stream_capacity;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const long long rp = stream_ptrs(s)[0], wp = stream_ptrs(s)[1];
  // the children's results and keys (k_child_results leaves rounds of this
  // size to this kernel), formed before any decision so that the single-block
  // placement finds them too
  const int begin = (rank * kClusterThreads + tid) * kClusterPer;
  uint64_t kv[kClusterPer];  // the children's keys
  if (B >= kClusterMinChildren) {
    int reused_here = 0;
#pragma unroll
    for (int t = 0; t < kClusterPer; ++t) {
      kv[t] = ~0ULL;
      if (begin + t < B) {
        bool reused;
        kv[t] = child_result_of(s, begin + t, &reused);
        reused_here += reused;
      }
    }
    for (int o = 16; o; o >>= 1) reused_here += __shfl_xor_sync(kFull, reused_here, o);
    if (lane == 0 && reused_here)
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[1]), (unsigned long long)reused_here);
  }
  // the levels come from k_place_levels, run earlier in this round
  if (!cluster_placement_applies(s, rp, wp) || s.level_plan[0] != s.round[0] + 1) {
    if (rank == 0 && tid == 0) *s.place_state = 0;
    return;  // the same decision in every block
  }
  const int n_levels = s.level_plan[1];
  const int local_P = (P + kPlaceCtas - 1) / kPlaceCtas;
  uint64_t* keys = cl_keys;
  for (int i = tid; i < local_P; i += blockDim.x) {
    const int m = i * kPlaceCtas + rank;
    keys[i] = m < P ? s.key[m] : ~0ULL;
  }
  int32_t* __restrict__ placed = s.placed;
  for (int m = rank * kClusterThreads + tid; m < P; m += kPlaceCtas * kClusterThreads) placed[m] = -1;
  if (tid == 0) redraw_at = 0x7fffffff;
  const int base = int(rp % cap);
  uint32_t cand[kClusterPer];
  int lvl[kClusterPer];  // the children's placement levels
#pragma unroll
  for (int t = 0; t < kClusterPer; ++t) {
    const int j = begin + t;
    cand[t] = 0;
    lvl[t] = -1;
    if (j < B) {
      cand[t] = child_draws(s, base, j);
      lvl[t] = s.child_level[j];
    }
  }
  auto key_at = [&](int m) -> uint64_t* { return cluster.map_shared_rank(keys, m % kPlaceCtas) + m / kPlaceCtas; };
  cluster.sync();
  const long long level_start = clock64();
  // Level by level: the children of level L read both members' keys, the
  // worse member takes the child's key; a cluster barrier then makes the
  // writes visible to level L + 1.  Children of one level draw disjoint
  // members, so no two of them touch the same key.
  const int levels_run = n_levels;
  for (int level = 0; level < n_levels; ++level) {
#pragma unroll
    for (int t = 0; t < kClusterPer; ++t)
      if (lvl[t] == level) {
        const int d0 = int(cand[t] & 0xffff), d1 = int(cand[t] >> 16);
        const uint64_t k0 = *key_at(d0), k1 = *key_at(d1);
        // worst of the pair: the second replaces the first when the first is better
        const int v = (k0 < k1 || (k0 == k1 && d0 < d1)) ? d1 : d0;
        *key_at(v) = kv[t];
        placed[v] = begin + t;
        cand[t] = uint32_t(v);
      }
    cluster.sync();
  }
  const long long level_end = clock64();
  // best member before each child: (key, victim) minimum of this thread's
  // children, a warp scan, a block scan, then the blocks before this one
  uint64_t mk = ~0ULL;
  int mv = 0x7fffffff;
#pragma unroll
  for (int t = 0; t < kClusterPer; ++t)
    if (begin + t < B && key_before(kv[t], int(cand[t]), mk, mv)) { mk = kv[t]; mv = int(cand[t]); }
  for (int o = 1; o < 32; o <<= 1) {
    const uint64_t uk = __shfl_up_sync(kFull, mk, o);
    const int uv = __shfl_up_sync(kFull, mv, o);
    if (lane >= o && key_before(uk, uv, mk, mv)) { mk = uk; mv = uv; }
  }
  constexpr int kWarps = kClusterThreads / 32;
  if (lane == 31) { scan_key[warp] = mk; scan_idx[warp] = mv; }
  __syncthreads();
  if (warp == 0) {
    uint64_t wk = lane < kWarps ? scan_key[lane] : ~0ULL;
    int wv = lane < kWarps ? scan_idx[lane] : 0x7fffffff;
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t uk = __shfl_up_sync(kFull, wk, o);
      const int uv = __shfl_up_sync(kFull, wv, o);
      if (lane >= o && key_before(uk, uv, wk, wv)) { wk = uk; wv = uv; }
    }
    scan_key[lane] = wk;
    scan_idx[lane] = wv;
    if (lane == kWarps - 1) {
      *cluster.map_shared_rank(cta_key + rank, 0) = wk;
      *cluster.map_shared_rank(cta_idx + rank, 0) = wv;
    }
  }
  cluster.sync();
  const int best0 = s.best[0];
  const uint64_t best0_key = s.key[best0];
  int bv = best0;
  uint64_t bk = best0_key;
  {
    const uint64_t* tot_key = cluster.map_shared_rank(cta_key, 0);
    const int* tot_idx = cluster.map_shared_rank(cta_idx, 0);
    for (int r = 0; r < rank; ++r)
      if (key_before(tot_key[r], tot_idx[r], bk, bv)) { bk = tot_key[r]; bv = tot_idx[r]; }
    const uint64_t lk = __shfl_up_sync(kFull, mk, 1);
    const int lv = __shfl_up_sync(kFull, mv, 1);
    if (lane > 0 && key_before(lk, lv, bk, bv)) { bk = lk; bv = lv; }
    if (warp > 0 && key_before(scan_key[warp - 1], scan_idx[warp - 1], bk, bv)) {
      bk = scan_key[warp - 1];
      bv = scan_idx[warp - 1];
    }
  }
  // a child whose victim is the best member before it would have redrawn;
  // the earliest such child is noted in every block, so that no block reads
  // another's shared memory after the last cluster barrier
  bool hit = false;
#pragma unroll
  for (int t = 0; t < kClusterPer; ++t)
    if (!hit && begin + t < B) {
      const int v = int(cand[t]);
      if (v == bv) {
        for (int r = 0; r < kPlaceCtas; ++r) atomicMin(cluster.map_shared_rank(&redraw_at, r), begin + t);
        hit = true;
      } else if (key_before(kv[t], v, bk, bv)) {
        bk = kv[t];
        bv = v;
      }
    }
  cluster.sync();
  const bool done = redraw_at == 0x7fffffff;
  if (done) {
    // this block's members take their child's statistics
    const double* __restrict__ cfit = s.c_fitness;
    const uint32_t* __restrict__ cwrong = s.c_wrong;
    const uint32_t* __restrict__ cnodes = s.c_nodes;
    for (int i = tid; i < local_P; i += blockDim.x) {
      const int m = i * kPlaceCtas + rank;
      if (m >= P) continue;
      const int c = placed[m];
      if (c >= 0) {
        s.key[m] = keys[i];
        s.fitness[m] = cfit[c];
        s.wrong[m] = cwrong[c];
        s.nodes[m] = cnodes[c];
      }
    }
  }
  if (rank == 0 && tid == 0) {
    *s.place_state = done ? 1 : 2;
    if (done) {
      const uint64_t* tot_key = cta_key;
      int fv = best0;
      uint64_t fk = best0_key;
      for (int r = 0; r < kPlaceCtas; ++r)
        if (key_before(tot_key[r], cta_idx[r], fk, fv)) { fk = tot_key[r]; fv = cta_idx[r]; }
      s.best[0] = fv;
      // the next round's seed: the raw output after the 2B placement draws
      const long long pos = rp + 2LL * B;
      s.round_seed[0] = s.stream[pos % cap];
      stream_ptrs(s)[0] = pos + 1;
      const int r = s.round[0] + 1;
      s.round[0] = r;
      if (r >= s.total_rounds) s.round[2] = 1;
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[5]), (unsigned long long)(clock64() - t0));
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[14]), (unsigned long long)(level_end - level_start));
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[7]), (unsigned long long)levels_run);
    }
  }
}

// ------------------------------------------------------------ result export
// The final population ranked as the reference ranks it (by ranking key,
// ties by member index, selection.cpp:10-20): a member's rank is the number
// of members before it, counted against shared-memory tiles of the keys.
constexpr int kRankTile = 1024;
__global__ void __launch_bounds__(128) k_rank_members(const SearchDesc* desc, int32_t* rank) {
  __shared__ uint64_t tile[kRankTile];
  const SearchDesc& s = *desc;
  const int P = s.P;
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const uint64_t mk = m < P ? s.key[m] : 0;
  int r = 0;
  for (int base = 0; base < P; base += kRankTile) {
    __syncthreads();
    for (int i = threadIdx.x; i < kRankTile; i += blockDim.x) tile[i] = base + i < P ? s.key[base + i] : ~0ULL;
    __syncthreads();
    const int lim = min(kRankTile, P - base);
    if (m < P)
      for (int j = 0; j < lim; ++j) {
        const uint64_t k = tile[j];
        r += k < mk || (k == mk && base + j < m);
      }
  }
  if (m < P) rank[m] = r;
}

// Each member's statistics and transport row (construction expressions and
// constants, `width` entries per row, zero past its counts) at its rank:
// a warp per member.
__global__ void k_export_members(const SearchDesc* desc, const int32_t* rank, int width, double* fitness,
                                 int32_t* wrong, int32_t* nodes, int32_t* node_counts, int32_t* constant_counts,
                                 int32_t* origins, int64_t* constants) {
  const int m = int((size_t(blockIdx.x) * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
  const SearchDesc& s = *desc;
  if (m >= s.P) return;
  const int r = rank[m];
  const int32_t l = s.len[m];
  const int n = len_nodes(l), nc = len_consts(l);
  if (lane == 0) {
    fitness[r] = s.fitness[m];
    wrong[r] = s.has_wrong ? int32_t(s.wrong[m]) : -1;
    nodes[r] = s.fixed_nodes + n;
    node_counts[r] = n;
    constant_counts[r] = nc;
  }
  const uint64_t* node = s.node + size_t(m) * s.stride;
  const int64_t* cval = s.cval + size_t(m) * s.stride;
  for (int i = lane; i < width; i += 32) {
    origins[size_t(r) * width + i] = i < n && i < s.stride ? int32_t(node[i] & 0xffffu) : 0;
    constants[size_t(r) * width + i] = i < nc && i < s.stride ? cval[i] : 0;
  }
}

// commit_batch (phase_population_cpu.cpp:382-394): placed child rows replace
// members.  Thread per member.
constexpr int kCommitLanes = 16;  // threads per member row
__global__ void k_commit(const SearchDesc* descs, const int32_t* off, int n) {
  const size_t gid = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int item = int(gid / kCommitLanes), lane = int(gid % kCommitLanes);
  if (item >= off[n]) return;
  const int si = find_search(off, n, item);
  const SearchDesc& s = descs[si];
  if (s.round[3]) return;
  const int m = item - off[si];
  // this round's member index is spent: its slots start the next round empty
  if (s.mtab) {
    const int e = m * kCommitLanes + lane;
    if (e <= s.mtab_mask) s.mtab[e] = 0;
  }
  const int b = s.placed[m];
  if (b < 0) return;
  // the row's threads copy consecutive slots: coalesced reads and writes
  const int32_t l = s.clen[b];
  const uint64_t* from = s.cnode + size_t(b) * s.stride;
  const int64_t* cfrom = s.ccval + size_t(b) * s.stride;
  uint64_t* to = s.node + size_t(m) * s.stride;
  int64_t* cto = s.cval + size_t(m) * s.stride;
  for (int i = lane; i < len_nodes(l); i += kCommitLanes) to[i] = from[i];
  for (int i = lane; i < len_consts(l); i += kCommitLanes) cto[i] = cfrom[i];
  if (lane == 0) s.len[m] = l;
}

// ----------------------------------------------------------- generational
// The generational schedule's placement (reproduce, phase_population_cpu.cpp:
// 269-312, then the next evaluate's reuse, :243-265): child i becomes member
// i with its result.  Runs after k_child_results, which read the members'
// results for the reused children; k_commit then copies the rows.
__global__ void k_gen_place(const SearchDesc* descs, const int32_t* off, int n) {
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= off[n]) return;
  const int si = find_search(off, n, item);
  const SearchDesc& s = descs[si];
  if (!search_live(s)) return;
  const int m = item - off[si];
  s.fitness[m] = s.c_fitness[m];
  s.wrong[m] = s.c_wrong[m];
  s.nodes[m] = s.c_nodes[m];
  s.key[m] = s.c_key[m];
  s.placed[m] = m;
}

// End of a generational round, one block per search: the next round's
// elites and best member, its variation seed (the next run-generator output,
// one per generation as run_phase_population draws rng() per reproduce,
// evolve.cpp:300-301) and the round count.
__global__ void k_gen_finish(const SearchDesc* descs, int n) {
  __shared__ uint64_t mt[312], nw[312];
  __shared__ int32_t best_one[1];
  const SearchDesc& s = descs[blockIdx.x];
  if (!search_live(s)) return;
  if (s.elite_count > 0) {
    block_best_members(s, s.elite_count, s.elites);
  } else {
    block_best_members(s, 1, best_one);
  }
  __syncthreads();
  long long* head = stream_ptrs(s);
  const long long rp = head[0], wp = head[1];
  if (rp >= wp) {  // the run generator's next block (every 312 generations)
    for (int i = threadIdx.x; i < 312; i += blockDim.x) mt[i] = s.mt[i];
    __syncthreads();
    mt_block(s, mt, nw, wp);
    for (int i = threadIdx.x; i < 312; i += blockDim.x) s.mt[i] = mt[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    s.best[0] = s.elite_count > 0 ? s.elites[0] : best_one[0];
    s.round_seed[0] = s.stream[rp % s.stream_capacity];
    head[0] = rp + 1;
    if (rp >= wp) head[1] = wp + 312;
    const int done = s.round[0] + 1;
    s.round[0] = done;
    if (done >= s.total_rounds) s.round[2] = 1;
  }
}

}  // namespace gb
