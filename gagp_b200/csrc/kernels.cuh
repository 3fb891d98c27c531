// Kernels of one resident steady-state round and of search start-up.
//
// Every kernel works on a batch of searches: `descs` holds one SearchDesc per
// search and per-item kernels map a flat index to (search, item) with the
// offsets array (items of search i are [off[i], off[i+1])).  A single search
// is a batch of one.  Per round (run_phase_population_steady,
// cpp/src/evolution/evolve.cpp:388-427):
//   k_record (epoch start) -> k_vary -> k_lower -> k_vm_fast / k_vm_general
//   -> k_child_results -> k_place -> k_commit
#pragma once
#include "operators.cuh"
#include "vm.cuh"

namespace gb {

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
  const int i = item - off[si];
  const int site_limit = s.site_depth;
  const int ramp = site_limit < 2 ? site_limit : 2 + i % (site_limit - 1);
  uint64_t* node = s.node + size_t(i) * s.stride;
  int64_t* cval = s.cval + size_t(i) * s.stride;
  uint32_t pending[192];
  GenResult g{ST_INVALID, 0, 0};
  for (int logical = ramp, attempt = 0; g.status != ST_OK; ++attempt) {
    const int room = s.maxv < kCapacity ? s.maxv : kCapacity;
    g = generate(s, s.root_expression, 0, s.slot_max_depth, room,
                 mix64(s.seed ^ mix64((uint64_t(i) * 8 + 0) * 64 + uint64_t(attempt))), node, cval, logical, pending);
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
// that reuse no member's result.
__global__ void k_lower(const SearchDesc* descs, const int32_t* off, int n, int mode, ProgramRef* fast_list,
                        ProgramRef* general_list, int32_t* list_count) {
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= off[n]) return;
  const int si = find_search(off, n, item);
  const SearchDesc& s = descs[si];
  if (!search_live(s)) return;
  const int slot = item - off[si];
  LRow t;
  if (mode == 0) {
    const int32_t l = s.len[slot];
    t = LRow{s.node + size_t(slot) * s.stride, s.cval + size_t(slot) * s.stride, len_nodes(l), len_consts(l)};
  } else {
    if (!s.c_eval[slot]) return;
    const int32_t l = s.clen[slot];
    t = LRow{s.cnode + size_t(slot) * s.stride, s.ccval + size_t(slot) * s.stride, len_nodes(l), len_consts(l)};
  }
  int temps = 0, klen = 0;
  int len = lower_accumulator(s, t, s.code + size_t(slot) * s.code_stride, s.code_stride,
                              s.kpool + size_t(slot) * s.stride, &klen, &temps);
  if (len >= 0) {
    // exact bytecode length (a bound of every executed path) must fit the fuel
    int bytecode = 1;
    for (int i = 0; i < t.n; ++i) {
      const int nk = s.info[w_origin(t.node[i])].node_kind;
      bytecode += nk == TK_IF ? 2 : (nk == TK_AND || nk == TK_OR) ? 5 : 1;
    }
    if (bytecode > s.fuel) len = -1;
  }
  if (len >= 0) {
    s.code_len[slot] = len;
    s.code_temps[slot] = temps;
    fast_list[atomicAdd(&list_count[0], 1)] = ProgramRef{si, slot};
    return;
  }
  int nconst = 0, bound = 0;
  const int bl = lower_reference(s, t, s.bc + size_t(slot) * 5 * s.bc_stride, s.bc_stride,
                                 s.bc_consts + size_t(slot) * s.bc_stride, &nconst, &bound);
  if (bl < 0) {
    raise_error(s, 30);  // the phase compiler rejected a constructed program
    return;
  }
  s.bc_len[slot] = bl;
  s.code_temps[slot] = -1;
  general_list[atomicAdd(&list_count[1], 1)] = ProgramRef{si, slot};
}

__device__ __forceinline__ void store_result(const SearchDesc& s, int mode, int slot, int64_t loss, uint32_t wrong) {
  const double f = -double(loss);
  if (mode == 0) {
    s.fitness[slot] = f;
    s.wrong[slot] = s.has_wrong ? wrong : 0;
  } else {
    s.c_fitness[slot] = f;
    s.c_wrong[slot] = s.has_wrong ? wrong : 0;
  }
}

// Fast VM: persistent warps over the fast list.  Per warp shared memory:
// temporaries (kMaxTemps x lanes x 32), the staged code (code_stride) and
// constants (stride).
template <int K>
__device__ __forceinline__ void run_k(const SearchDesc& s, int slot, const VmWarpSmem& w, int64_t& loss,
                                      uint32_t& wrong, uint64_t& ops) {
  switch (s.n_inputs) {
    case 1: run_accumulator<K, 1>(s, slot, w, loss, wrong, ops); break;
    case 2: run_accumulator<K, 2>(s, slot, w, loss, wrong, ops); break;
    default: run_accumulator<K, 0>(s, slot, w, loss, wrong, ops); break;
  }
}
__global__ void k_vm_fast(const SearchDesc* descs, int mode, const ProgramRef* list, const int32_t* list_count,
                          int temp_stride, int code_stride, int const_stride) {
  extern __shared__ __align__(16) int64_t smem_vm[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int warps = blockDim.x >> 5;
  const size_t per_warp = size_t(temp_stride) + size_t(code_stride) + size_t(const_stride);  // int64 units
  int64_t* base = smem_vm + size_t(warp) * per_warp;
  const VmWarpSmem w{base, reinterpret_cast<uint2*>(base + temp_stride), base + temp_stride + code_stride};
  const int count = *list_count;
  for (int i = blockIdx.x * warps + warp; i < count; i += gridDim.x * warps) {
    const ProgramRef p = list[i];
    const SearchDesc& s = descs[p.search];
    int64_t loss = 0;
    uint32_t wrong = 0;
    uint64_t ops = 0;
    switch (s.vm_cases_per_lane) {
      case 1: run_k<1>(s, p.slot, w, loss, wrong, ops); break;
      case 2: run_k<2>(s, p.slot, w, loss, wrong, ops); break;
      case 4: run_k<4>(s, p.slot, w, loss, wrong, ops); break;
      default: run_k<8>(s, p.slot, w, loss, wrong, ops); break;
    }
    loss = warp_sum(loss);
    wrong = warp_sum(wrong);
    if (lane == 0) {
      store_result(s, mode, p.slot, loss, wrong);
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[0]), 1ULL);
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[2]), (unsigned long long)s.C);
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[3]), (unsigned long long)ops);
    }
  }
}

// General VM: one block per program of the general list, threads over cases.
__global__ void k_vm_general(const SearchDesc* descs, int mode, const ProgramRef* list, const int32_t* list_count) {
  __shared__ int64_t red_loss[32];
  __shared__ uint32_t red_wrong[32];
  const int count = *list_count;
  for (int i = blockIdx.x; i < count; i += gridDim.x) {
    const ProgramRef p = list[i];
    const SearchDesc& s = descs[p.search];
    const int32_t* code = s.bc + size_t(p.slot) * 5 * s.bc_stride;
    const int64_t* consts = s.bc_consts + size_t(p.slot) * s.bc_stride;
    const int n = s.bc_len[p.slot];
    int64_t loss = 0;
    uint32_t wrong = 0;
    uint64_t steps = 0;
    for (int c = threadIdx.x; c < s.C; c += blockDim.x) {
      int64_t value = 0;
      int tag = 0;
      if (run_reference(s, code, n, consts, c, value, tag, steps)) {
        loss += case_loss(s, tag, value, s.expected[c], wrong);
      } else {
        loss += error_loss(s);
        ++wrong;
      }
    }
    loss = warp_sum(loss);
    wrong = warp_sum(wrong);
    steps = warp_sum(steps);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) { red_loss[warp] = loss; red_wrong[warp] = wrong; }
    if (lane == 0) atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[3]), (unsigned long long)steps);
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t tl = 0;
      uint32_t tw = 0;
      for (int w = 0; w < (blockDim.x >> 5); ++w) { tl += red_loss[w]; tw += red_wrong[w]; }
      store_result(s, mode, p.slot, tl, tw);
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[0]), 1ULL);
      atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[2]), (unsigned long long)s.C);
    }
    __syncthreads();
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
// Twists `mt` (smem, 312 words) using scratch `nw` (312 words) and appends
// the tempered block to the stream ring at `wp`.
__device__ inline void mt_block(const SearchDesc& s, uint64_t* mt, uint64_t* nw, long long wp) {
  for (int i = threadIdx.x; i < 156; i += blockDim.x) nw[i] = mt_mix(mt[i], mt[i + 1], mt[i + 156]);
  __syncthreads();
  for (int i = 156 + threadIdx.x; i < 311; i += blockDim.x) nw[i] = mt_mix(mt[i], mt[i + 1], nw[i - 156]);
  __syncthreads();
  if (threadIdx.x == 0) nw[311] = mt_mix(mt[311], nw[0], nw[155]);
  __syncthreads();
  for (int i = threadIdx.x; i < 312; i += blockDim.x) {
    mt[i] = nw[i];
    const uint64_t out = mt_temper(nw[i]);
    const long long pos = (wp + i) % s.stream_capacity;
    s.stream[pos] = out;
    s.stream_mod[pos] = uint32_t(out % uint64_t(s.P));
  }
  __syncthreads();
}
// Serial fallback of one block, for a consumer that ran ahead of the buffer.
__device__ inline void mt_block_serial(const SearchDesc& s, uint64_t* mt, long long wp) {
  for (int i = 0; i < 312; ++i) mt[i] = mt_mix(mt[i], mt[(i + 1) % 312], mt[(i + 156) % 312]);
  for (int i = 0; i < 312; ++i) {
    const uint64_t out = mt_temper(mt[i]);
    const long long pos = (wp + i) % s.stream_capacity;
    s.stream[pos] = out;
    s.stream_mod[pos] = uint32_t(out % uint64_t(s.P));
  }
}

// stream_head as two 64-bit counters: [0] read, [1] written
__device__ __forceinline__ long long* stream_ptrs(const SearchDesc& s) { return s.stream_head; }

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
}

// ----------------------------------------------------------- one round
// History entry before every population/batch rounds (record(),
// evolve.cpp:360-371): the best member, its row, and the exact integer sum of
// member fitness (the host forms the long double mean).
__global__ void k_record(const SearchDesc* descs, int n, int only_epoch_start) {
  __shared__ long long partial[256];
  const SearchDesc& s = descs[blockIdx.x];
  if (!search_live(s)) return;
  const int round = s.round[0];
  if (only_epoch_start && round % s.rounds_per_epoch) return;
  const int entry = s.round[1];
  if (entry >= s.generations) return;
  long long sum = 0;
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

// make_batch (phase_population_cpu.cpp:322-353): one warp per child, rows
// staged in dynamic shared memory (warp_rows_bytes(stride) per warp).
__global__ void k_vary(const SearchDesc* descs, const int32_t* off, int n, int stride_max) {
  extern __shared__ __align__(16) char smem_rows[];
  const int warps = blockDim.x >> 5, warp = threadIdx.x >> 5;
  const int item = blockIdx.x * warps + warp;
  if (item >= off[n]) return;
  const int si = find_search(off, n, item);
  const SearchDesc& s = descs[si];
  if (!search_live(s)) return;
  const int child = item - off[si];
  WarpRows rows = carve_rows(smem_rows + size_t(warp) * warp_rows_bytes(stride_max), s.stride);
  int reuse = -1, parent = -1;
  const int error = warp_vary_child(s, child, s.round_seed[0], rows, &reuse, &parent);
  if ((threadIdx.x & 31) == 0) {
    s.c_parent[child] = parent;
    s.c_reuse[child] = reuse;
    s.c_error[child] = error;
    s.c_eval[child] = error == 0 && reuse < 0;
    if (error) raise_error(s, 100 + error);
  }
}

// Results of all children before any placement (evolve.cpp:403-413).
__global__ void k_child_results(const SearchDesc* descs, const int32_t* off, int n) {
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= off[n]) return;
  const int si = find_search(off, n, item);
  const SearchDesc& s = descs[si];
  if (!search_live(s)) return;
  const int b = item - off[si];
  const int source = s.c_reuse[b];
  double f;
  uint32_t w, nodes;
  if (source >= 0) {
    f = s.fitness[source];
    w = s.wrong[source];
    nodes = s.nodes[source];
    atomicAdd(reinterpret_cast<unsigned long long*>(&s.counters[1]), 1ULL);
  } else {
    f = s.c_fitness[b];
    w = s.c_wrong[b];
    nodes = s.has_wrong ? ranking_nodes(s, s.cnode + size_t(b) * s.stride, len_nodes(s.clen[b])) : 0;
  }
  s.c_fitness[b] = f;
  s.c_wrong[b] = w;
  s.c_nodes[b] = nodes;
  s.c_key[b] = pack_key(s, f, w, nodes);
}

// Steady-state placement (evolve.cpp:414-427): children in order, each
// replacing the worst of replacement_size uniform draws (redrawn when it is
// the current best).  The block pre-generates the run generator's outputs
// and stages their residues mod P as 16-bit draws in shared memory beside
// the members' ranking keys; one thread then runs the sequential placement.
// With the default replacement size 2 the next child's draws and keys are
// loaded one child ahead and the current child's key store is forwarded to
// them when they name the replaced member, so shared-memory latency leaves
// the dependency chain.  Then the next round's seed is drawn.  One block per
// search; `dyn_bytes`: dynamic shared memory of the launch.
__global__ void k_place(const SearchDesc* descs, int n, int dyn_bytes) {
  extern __shared__ __align__(16) uint64_t keys[];
  __shared__ uint64_t mt[312], nw[312];
  const SearchDesc& s = descs[blockIdx.x];
  if (!search_live(s)) return;
  const int P = s.P, B = s.B, rs = s.replacement_size, cap = s.stream_capacity;
  uint16_t* draws = reinterpret_cast<uint16_t*>(keys + P);
  const int slots = (dyn_bytes - int(sizeof(uint64_t)) * P) / int(sizeof(uint16_t));
  int32_t* __restrict__ placed = s.placed;
  for (int m = threadIdx.x; m < P; m += blockDim.x) {
    keys[m] = s.key[m];
    placed[m] = -1;
  }
  for (int i = threadIdx.x; i < 312; i += blockDim.x) mt[i] = s.mt[i];
  __syncthreads();
  const long long rp = stream_ptrs(s)[0];
  long long wp = stream_ptrs(s)[1];
  const long long need = (long long)B * rs + 1;
  while (wp - rp < need && wp - rp + 312 <= cap) {
    mt_block(s, mt, nw, wp);
    wp += 312;
  }
  const int avail = int(min((long long)slots, wp - rp));
  for (int i = threadIdx.x; i < avail; i += blockDim.x) draws[i] = uint16_t(s.stream_mod[(rp + i) % cap]);
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t* __restrict__ smod = s.stream_mod;
    const uint64_t* __restrict__ ckey = s.c_key;
    long long gen_wp = wp;
    // residue of the draw `idx` positions after rp (staged, else the ring)
    auto draw = [&](int idx) -> int {
      if (idx < avail) return draws[idx];
      const long long pos = rp + idx;
      while (pos >= gen_wp) {  // ran ahead of the buffer: one serial block
        mt_block_serial(s, mt, gen_wp);
        gen_wp += 312;
      }
      return int(smod[pos % cap]);
    };
    int best = s.best[0];
    uint64_t best_key = keys[best];
    int di = 0;
    bool failed = false;
    if (rs == 2) {
      int d0 = draw(0), d1 = draw(1);
      uint64_t k0 = keys[d0], k1 = keys[d1];
      uint64_t ck = ckey[0];
      for (int b = 0; b < B; ++b) {
        di += 2;
        const uint64_t ck_next = b + 1 < B ? ckey[b + 1] : 0;
        // worst of the pair: the second replaces the first when the first is better
        int v = (k0 < k1 || (k0 == k1 && d0 < d1)) ? d1 : d0;
        for (int guard = 0; v == best; ++guard) {
          if (guard > (1 << 20)) { failed = true; break; }
          d0 = draw(di); d1 = draw(di + 1); di += 2;
          k0 = keys[d0]; k1 = keys[d1];
          v = (k0 < k1 || (k0 == k1 && d0 < d1)) ? d1 : d0;
        }
        if (failed) break;
        int n0 = 0, n1 = 0;
        uint64_t nk0 = 0, nk1 = 0;
        if (b + 1 < B) {
          n0 = draw(di);
          n1 = draw(di + 1);
          nk0 = keys[n0];
          nk1 = keys[n1];
        }
        keys[v] = ck;
        placed[v] = b;
        if (n0 == v) nk0 = ck;
        if (n1 == v) nk1 = ck;
        if (ck < best_key || (ck == best_key && v < best)) { best = v; best_key = ck; }
        d0 = n0; d1 = n1; k0 = nk0; k1 = nk1; ck = ck_next;
      }
    } else {
      for (int b = 0; b < B && !failed; ++b) {
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
        if (v < 0) { failed = true; break; }
        keys[v] = ck;
        placed[v] = b;
        if (ck < best_key || (ck == best_key && v < best)) { best = v; best_key = ck; }
      }
    }
    if (failed) raise_error(s, 40);
    // the next round's variation seed: the raw output at the next position
    const long long pos = rp + di;
    while (pos >= gen_wp) {
      mt_block_serial(s, mt, gen_wp);
      gen_wp += 312;
    }
    s.round_seed[0] = s.stream[pos % cap];
    s.best[0] = best;
    stream_ptrs(s)[0] = pos + 1;
    stream_ptrs(s)[1] = gen_wp;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 312; i += blockDim.x) s.mt[i] = mt[i];
  for (int m = threadIdx.x; m < P; m += blockDim.x) {
    const int b = placed[m];
    if (b >= 0) {
      s.key[m] = keys[m];
      s.fitness[m] = s.c_fitness[b];
      s.wrong[m] = s.c_wrong[b];
      s.nodes[m] = s.c_nodes[b];
    }
  }
  if (threadIdx.x == 0) {
    const int r = s.round[0] + 1;
    s.round[0] = r;
    if (r >= s.total_rounds) s.round[2] = 1;
  }
}

// commit_batch (phase_population_cpu.cpp:382-394): placed child rows replace
// members.  Thread per member.
__global__ void k_commit(const SearchDesc* descs, const int32_t* off, int n) {
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= off[n]) return;
  const int si = find_search(off, n, item);
  const SearchDesc& s = descs[si];
  if (s.round[3]) return;
  const int m = item - off[si];
  const int b = s.placed[m];
  if (b < 0) return;
  const int32_t l = s.clen[b];
  const uint64_t* from = s.cnode + size_t(b) * s.stride;
  const int64_t* cfrom = s.ccval + size_t(b) * s.stride;
  uint64_t* to = s.node + size_t(m) * s.stride;
  int64_t* cto = s.cval + size_t(m) * s.stride;
  for (int i = 0; i < len_nodes(l); ++i) to[i] = from[i];
  for (int i = 0; i < len_consts(l); ++i) cto[i] = cfrom[i];
  s.len[m] = l;
}

}  // namespace gb
