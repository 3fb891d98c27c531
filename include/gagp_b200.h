/*
 * gagp_b200 -- C ABI of the B200 resident GAGP search engine.
 *
 * The engine replaces the reference's resident GPU owner
 * (NativePhasePopulation, cpp/src/evolution/repro/gpu/phase_population.hpp:15-60)
 * and the steady-state search loop that drives it
 * (run_phase_population_steady, cpp/src/evolution/evolve.cpp:331-441).
 * Plain pointers and sizes only; every device resource is owned by the
 * engine handle.  Inputs are copied in; exports are copied into caller
 * buffers.  API calls on one engine must be serialized by the caller.
 *
 * Data formats (the admitted phase tables) follow the reference's
 * HostPhaseGrammar / DeviceSlot layout
 * (cpp/src/evolution/repro/gpu/phase_grammar.hpp:17-40,
 *  cpp/src/evolution/repro/gpu/phase_operators.cuh:25).
 */
#ifndef GAGP_B200_H
#define GAGP_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status (reference: invalid_argument = decline, runtime_error = failure) */
typedef int32_t gagp_status;
enum {
  GAGP_OK = 0,
  GAGP_DECLINED = 1,          /* admission decline: rerun on the native representation */
  GAGP_INVALID_ARGUMENT = 2,
  GAGP_OUT_OF_MEMORY = 3,
  GAGP_DEVICE_ERROR = 4,      /* the engine is poisoned; later calls are refused */
  GAGP_TIMEOUT_CAP = 5,       /* a device loop hit its iteration cap */
  GAGP_NOT_READY = 6,
  GAGP_NO_EXTENSION = 7
};

#define GAGP_MAX_ARITY 8
#define GAGP_MAX_LOCALS 64
#define GAGP_PHASE_CAPACITY 1024  /* physical phase row capacity of the reference */

/* ValueTag (cpp/include/gagp/core/value.hpp:16-27) */
enum { GAGP_TAG_INT = 0, GAGP_TAG_FLOAT = 1, GAGP_TAG_BOOL = 2, GAGP_TAG_INTLIST = 5, GAGP_TAG_INVALID = 9 };

/* One generation record (PhaseExpression, device/phase_generate.cuh:79-92).
 * kind: PhaseExpressionKind; node_*: the PhaseTreeNode it emits
 * (device/phase_compile.cuh:64-74). */
typedef struct gagp_expression {
  int32_t kind;
  int32_t node_kind;
  int32_t opcode;
  int32_t operand;
  int32_t arity;
  uint32_t fuel;
  uint32_t merge_fuel;
  int32_t type;
  int32_t target;
  int32_t scope_count;
  int32_t children[GAGP_MAX_ARITY];
  int8_t child_scope[GAGP_MAX_ARITY];
} gagp_expression;

typedef struct gagp_production {   /* PhaseProduction */
  int32_t expression;
  int32_t reserved;
  double weight;
} gagp_production;

typedef struct gagp_nonterminal {  /* PhaseNonterminal */
  int32_t production_offset;
  int32_t production_count;
  int32_t scope_count;
  int32_t normalized_weights;
  int32_t fixed;
} gagp_nonterminal;

typedef struct gagp_domain {       /* PhaseDomain */
  int32_t value_offset;
  int32_t value_count;
  int32_t integer_range;
  int32_t reserved;
  int64_t minimum;
  int64_t maximum;
} gagp_domain;

typedef struct gagp_value {        /* scalar Value: tag + payload */
  int64_t i;
  int32_t tag;
  int32_t reserved;
} gagp_value;

/* A traversal table entry: the reference's PhaseRegionInfo for a traversal
 * (cpp/src/evolution/repro/gpu/device/phase_compile.cuh:47-60), filled by
 * compile_phase_grammar (cpp/src/evolution/repro/gpu/phase_grammar.hpp:263-285).
 * A Traverse node's operand indexes this table.  Its children are source,
 * start, [begin, end,] initial state and body; the body binds element, index
 * and state as binder numbers binders[0..2]. */
typedef struct gagp_region {
  int32_t traversal;                /* 1: forward, 2: reverse (0: a bounded region, declined) */
  int32_t ranged;                   /* 1: traverse_range (begin and end operands) */
  int32_t fuel_profile;             /* 1: per-event fuel charges (event_cost), else every instruction costs 1 */
  int32_t binders[3];               /* binder numbers of element, index, state */
  int32_t operand_types[6];         /* ValueTag each child must complete with */
  int32_t binding_types[3];         /* ValueTag of element, index, state */
  int32_t result_type;              /* ValueTag of the traversal's (or the bounded region's) value */
  uint32_t event_cost[26];          /* PhaseFuelEvent charges when fuel_profile */
  /* A bounded region (traversal 0): a coordinate recurrence (RegionPlan,
   * cpp/include/gagp/core/region_plan.hpp:64-91, laid out as compile_phase_grammar
   * lays it out, phase_grammar.hpp:331-385).  Its children are `operands`
   * values -- the state_count initial states, then the bound operands --
   * and its `phases` phase subtrees: base predicate (Bool), base body,
   * combine and boundary.  Phase p sees phase_bindings[p] values as its
   * first locals, each from a bank of the current frame. */
  int32_t operands;
  int32_t phases;                   /* 4 */
  int32_t captures;                 /* parameters the phases may read from the caller */
  int32_t capture_kind[8];          /* 0 evaluator input, 1 grammar local, 2 binder */
  int32_t capture_target[8];        /* evaluator input position, grammar local or binder number */
  int32_t phase_type[8];            /* ValueTag phase p yields */
  int32_t phase_bindings[8];
  int32_t binding_bank[8][8];       /* 0 state, 1 parameter, 3 request result (RegionSlotBank) */
  int32_t binding_slot[8][8];
  int32_t phase_binding_types[8][8];
  int32_t state_count;              /* Int coordinates, 1..4 */
  int32_t request_count;            /* 1..8 */
  int32_t axis_count;               /* 1..4 */
  int32_t inclusive;                /* coordinate endpoint: 1 inclusive upper bound, 0 exclusive */
  int32_t memoized;
  uint32_t frames;                  /* frame limit, <= 128 */
  uint32_t cells;                   /* memo cell limit, <= 256 */
  uint32_t entry_fuel;              /* charged when a frame is entered */
  int32_t parameter_types[8];
  int32_t transition_kind[8][4];    /* request r, state s: 0 copy a state, 1 offset a coordinate */
  int32_t transition_source[8][4];
  int32_t axis_slot[4];             /* the state each coordinate axis reads */
  int32_t lower_kind[4];            /* 0 literal, 1 operand */
  int32_t upper_kind[4];
  int32_t reserved;
  int64_t transition_offset[8][4];
  int64_t lower[4];                 /* the literal, or the operand index */
  int64_t upper[4];
} gagp_region;

/* The admitted grammar of one search: phase tables plus its single
 * whole-program slot (expression entry: program(block(return phase)), four
 * fixed nodes; Program entry: the whole statement program, no fixed nodes
 * and no terminator). */
typedef struct gagp_grammar {
  const gagp_expression* expressions; int32_t expression_count;
  const gagp_production* productions; int32_t production_count;
  const gagp_nonterminal* nonterminals; int32_t nonterminal_count;
  const gagp_domain* domains; int32_t domain_count;
  const gagp_value* values; int32_t value_count;
  const uint32_t* minimum;          /* [expression][depth][logical] */
  int32_t depth_count;
  int32_t logical_depth_count;
  int32_t site_depth;               /* 0: no site-depth limit */
  int32_t root_expression;
  int32_t slot_max_depth;
  int32_t slot_type;                /* ValueTag of the phase result, or 0xF0 (kPhaseStatement) for a
                                       Program entry's statement program, whose returns carry its type */
  int32_t local_count;              /* evaluator inputs, sorted by name */
  int32_t local_types[GAGP_MAX_LOCALS];
  int32_t max_nodes;                /* grammar search_limits.max_nodes */
  int32_t fixed_nodes;              /* AST nodes outside the phase */
  uint32_t return_fuel;             /* fuel of the appended RETURN */
  const gagp_region* regions;       /* traversal table (HostPhaseGrammar::regions) */
  int32_t region_count;
} gagp_grammar;

/* Fitness cases: inputs[case * input_count + j] is the payload of evaluator
 * input j (an Int, 0/1 for a Bool, or for an IntList the index in
 * list_values of the list's length word, its elements following); tags per
 * input.  The reference keeps list inputs as payload handles into its
 * payload registry (cpp/src/runtime/payload/payload.cpp); here they are
 * read-only views into one flat array. */
typedef struct gagp_cases {
  int32_t case_count;
  int32_t input_count;
  const int64_t* inputs;
  const int32_t* input_tags;
  const int64_t* expected;
  int32_t expected_tag;
  const int64_t* list_values;       /* IntList inputs: length words and elements (NULL: none) */
  int64_t list_value_count;
} gagp_cases;

/* FitnessMetric (cpp/include/gagp/core/fitness_policy.hpp:4) */
enum { GAGP_METRIC_LEGACY = 0, GAGP_METRIC_ABSOLUTE = 1, GAGP_METRIC_EXACT = 2 };

/* gagp-search-config-v1 semantics (spec/search_config.md) of a resident run. */
typedef struct gagp_search_config {
  int32_t population;
  int32_t generations;
  uint64_t seed;
  int32_t tournament_size;
  int32_t crossover_attempts;
  double crossover_probability;
  double mutation_probability;
  int32_t mutation_max_nodes;
  int32_t counted_sites;            /* sites.draw: counted (1) / reservoir (0) */
  int32_t uniform_phase;            /* sites.scope: uniform_phase (1) / genome (0) */
  int32_t steady_state;             /* schedule.mode: steady_state (1) / generational (0) */
  int32_t batch;                    /* steady_state batch (0: population) */
  int32_t replacement_size;
  int32_t elite_count;              /* generational only */
  int32_t fuel;
  double penalty;                   /* case_cap */
  int32_t metric;
  int32_t grammar_site_ranking;     /* ranking.tie_break: grammar_sites */
  int32_t reduction_lanes;          /* 512 in gagp run */
  int32_t reserved;
} gagp_search_config;

/* A population of phase rows in transport form: row r has node_counts[r]
 * nodes whose construction expressions are origins[r*stride + i] and
 * constant_counts[r] Int constants constants[r*stride + k] in prefix order. */
typedef struct gagp_rows {
  int32_t count;
  int32_t stride;
  int32_t* node_counts;
  int32_t* origins;
  int32_t* constant_counts;
  int64_t* constants;
} gagp_rows;

/* Result of one search (history per generation-equivalent, final ranked
 * population), in caller-allocated arrays. */
typedef struct gagp_search_result {
  int32_t generations;              /* in: capacity of the history arrays; out: entries written */
  double* history_best_fitness;
  double* history_mean_fitness;
  int32_t* history_best_wrong;
  int32_t* history_best_nodes;
  gagp_rows history_best;           /* champion row per history entry */
  int32_t population;               /* capacity of the final arrays (the best `population` members) */
  double* final_fitness;            /* ranked: best first */
  int32_t* final_wrong;
  int32_t* final_nodes;
  gagp_rows final_rows;
  uint64_t evaluated_programs;      /* program evaluations run */
  uint64_t reused_programs;         /* children reusing a completed result: their parent's when
                                       unchanged, else an identical current member's */
  uint64_t program_cases;           /* evaluated (program, case) pairs */
} gagp_search_result;

/* ------------------------------------------------------------------ engine */
typedef struct gagp_engine gagp_engine;

const char* gagp_b200_last_error(void);
const char* gagp_b200_version(void);

/* Creates the engine on `device`. `arena_bytes` bounds the device memory the
 * engine may hold for resident searches (0: 80% of free memory). */
gagp_status gagp_b200_engine_create(int32_t device, uint64_t arena_bytes, gagp_engine** out);
void gagp_b200_engine_destroy(gagp_engine* engine);

/* Device bytes a search with this grammar, case set and config needs. */
gagp_status gagp_b200_search_bytes(const gagp_grammar* grammar, const gagp_cases* cases,
                                   const gagp_search_config* config, uint64_t* out_bytes);

/* Admits one search (NativePhasePopulation ctor, phase_population.cu:489-629):
 * uploads its tables and cases and builds its initial population on the
 * device, generated from the seed as generate_phase_initial_population does
 * (phase_population_cpu.cpp:54-113).  With `initial` (not NULL) the first
 * `population` of its rows are the initial population instead, in order, as
 * `gagp run --init` imports one (run.cpp:146-174, rows as the reference's
 * import_native_phase_layout gives them): each row must derive from the
 * grammar's root, fit the node budget and the site depth limit
 * (GAGP_INVALID_ARGUMENT otherwise). */
gagp_status gagp_b200_search_create(gagp_engine* engine, const gagp_grammar* grammar,
                                    const gagp_cases* cases, const gagp_search_config* config,
                                    const gagp_rows* initial, int32_t* out_search);
gagp_status gagp_b200_search_destroy(gagp_engine* engine, int32_t search);

/* Runs a search to completion on the device (the whole steady-state loop,
 * evolve.cpp:331-441, with no host round trip per round). */
gagp_status gagp_b200_search_run(gagp_engine* engine, int32_t search);

/* Advances every listed search together, one generation-equivalent per
 * launch sequence, until all have finished (batched engine). */
gagp_status gagp_b200_batch_run(gagp_engine* engine, const int32_t* searches, int32_t count);

/* Advances every listed unfinished search by one generation-equivalent;
 * `finished[i]` is set to 1 once search i has completed. */
gagp_status gagp_b200_batch_step(gagp_engine* engine, const int32_t* searches, int32_t count,
                                 int32_t* finished);

/* Runs start-up (initial population, initial evaluation, run generator) of
 * every listed search that has not started; synchronous. */
gagp_status gagp_b200_batch_start(gagp_engine* engine, const int32_t* searches, int32_t count);

/* Enqueues `rounds` steady-state rounds of the listed (started) searches and
 * waits.  *device_ms: summed CUDA-event time of the rounds on the engine
 * stream; with flush_l2 a 256 MiB buffer is written before each round,
 * outside the timed region, so no round starts with a warm L2. */
gagp_status gagp_b200_batch_advance(gagp_engine* engine, const int32_t* searches, int32_t count,
                                    int32_t rounds, int32_t flush_l2, double* device_ms);

/* Rounds done, total rounds and completion flag of a search (synchronous). */
gagp_status gagp_b200_search_progress(gagp_engine* engine, int32_t search, int32_t* rounds_done,
                                      int32_t* total_rounds, int32_t* finished);

/* Work counters of a search so far: [0] program evaluations, [1] children
 * that reused their parent's result, [2] evaluated (program, case) pairs,
 * [3] accumulator-VM instructions executed over all cases (added when a
 * program's last case tile finishes), [24] bytecode instructions the exact
 * VM executed (the reference's fuel consumed by those programs), [4..6] SM
 * clock cycles of
 * the placement phases (stream generation, draw staging, placement),
 * [7] placement levels (+2^20 per sequential replay), [8] and [10..23]
 * only while kernel profiling is on (gagp_b200_engine_profile): [8] bytes the
 * variation kernel moved (parent, donor and child rows, tournament keys,
 * per-child outputs), [9] bytes the lowering kernel moved (rows read, code
 * and constants written), [10..13] SM clock cycles of the variation warps
 * summed over children (selection, crossover, mutation subtree generation,
 * the rest), [14] cycles of the placement's level loop, [15] the most
 * cycles one child's variation took, [16..19] the most cycles of one child
 * in each variation phase, [20] children whose variation took over 200000
 * cycles, [21] subtree-generation steps (tasks) of mutations, [22] the
 * most steps of one generation, [23] mutation subtree generations.
 * Copies min(count, GAGP_COUNTERS) entries
 * (synchronous). */
/* Bytes this engine's calls have copied host->device and device->host since
 * it was created (uploads at admission and batch launches, progress and
 * result reads). */
gagp_status gagp_b200_engine_transfers(gagp_engine* engine, uint64_t* h2d_bytes, uint64_t* d2h_bytes);

#define GAGP_COUNTERS 25
gagp_status gagp_b200_search_counters(gagp_engine* engine, int32_t search, uint64_t* out, int32_t count);

/* Per-kernel CUDA-event timing: enable (resets) or disable, then read the
 * accumulated time and launch count of kernel index 0.. (INVALID_ARGUMENT
 * past the last kernel). */
gagp_status gagp_b200_engine_profile(gagp_engine* engine, int32_t enable);
gagp_status gagp_b200_engine_kernel_stats(gagp_engine* engine, int32_t kernel, const char** name,
                                          double* total_ms, int64_t* launches);
/* The timed launches of the last batch of rounds read back (profiling on),
 * in launch order: kernel index, start and end in ms after the batch's first
 * timed launch started.  *count is the number held; at most `capacity` are
 * written. */
gagp_status gagp_b200_engine_timeline(gagp_engine* engine, int32_t capacity, int32_t* kernel, float* start_ms,
                                      float* end_ms, int32_t* count);

/* Fitness and wrong-case counts of phase rows (host `rows`) on a case set:
 * each row is lowered on the device and run on every case, with the case
 * scores of `config` (metric, penalty, fuel).  Replaces the reference's
 * evaluator call over lowered owner programs, FitnessSessionGpu::eval_programs
 * (cpp/include/gagp/runtime/gpu/fitness_gpu.hpp:91-121) as the resident owner
 * uses it (NativePhasePopulation::evaluate, phase_population.cu:637-664).
 * fitness[rows->count], wrong[rows->count] (wrong may be null). */
gagp_status gagp_b200_evaluate_rows(gagp_engine* engine, const gagp_grammar* grammar, const gagp_cases* cases,
                                    const gagp_search_config* config, const gagp_rows* rows, double* fitness,
                                    uint32_t* wrong);

/* The verdict of one program on a case set, as the reference judges a run's
 * best program on the task's test split (judge / judge_case,
 * cpp/src/cli/run.cpp:176-238): cases, correct cases, runtime errors (a
 * failed execution, or a value that is not an Int where an Int is expected)
 * and the summed case loss (absolute metric: the integer gap capped at the
 * penalty, the penalty for an error or a wrong non-Int value; exact metric:
 * 1 per case that is not correct; 0 for a correct case).  The reference
 * reports mean_loss = loss / cases and solved = (correct == cases). */
typedef struct gagp_verdict {
  int32_t cases, correct, runtime_errors, reserved;
  double loss;
} gagp_verdict;
/* Verdicts of phase rows (host `rows`, e.g. a result's best row) on a case
 * set (e.g. the test split), lowered and run on the device like
 * gagp_b200_evaluate_rows; out[rows->count]. */
gagp_status gagp_b200_judge_rows(gagp_engine* engine, const gagp_grammar* grammar, const gagp_cases* cases,
                                 const gagp_search_config* config, const gagp_rows* rows, gagp_verdict* out);

/* gagp_b200_evaluate_rows without any device allocation -- no counterpart in
 * the reference.  For callers that must not call cudaMalloc: a host
 * application that hands all device memory to its own allocator (a framework
 * caching allocator or a fixed arena), or a latency-critical scoring loop
 * that cannot pay for an allocation and a free on every call.  Every device
 * buffer of the call lives in one static 32 MiB device array that each GPU
 * loading this library holds until exit; a call needing more (many rows,
 * long rows or many cases) is rejected with GAGP_INVALID_ARGUMENT and a
 * message naming the bytes needed.  Runs on the current device and `stream`
 * (a cudaStream_t; NULL: the default stream); it copies its inputs from
 * host memory, waits for the stream and returns when the results are in the
 * host arrays.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and sets kernel attributes; make that first
 * call before any stream capture.  All calls share the one array, and it
 * keeps the last call's contents (the call clears what must start at zero):
 * calls that overlap on the GPU, from several host threads or streams, race
 * and must be serialized. */
gagp_status gagp_b200_evaluate_rows_static(const gagp_grammar* grammar, const gagp_cases* cases,
                                           const gagp_search_config* config, const gagp_rows* rows,
                                           double* fitness, uint32_t* wrong, void* stream);

/* ----------------------------------------------------------------- serving
 * A request loop over one engine with continuous batching.  No counterpart
 * in the reference, which runs one search per process.  Requests are queued
 * on submit; every gagp_b200_server_step admits queued requests in arrival
 * order while their device bytes fit the server's memory budget (a request
 * waits, it is not reordered), starts the newly admitted searches, runs
 * steady-state rounds of every running search in one batched launch
 * sequence (gagp_b200_server_set_rounds_per_step), and retires the searches
 * that finished: their history and final
 * population are copied to host memory and their device memory is released
 * at once for the next admissions.  A request's result is the same as that
 * search run alone (every kernel works per search; the batch only shares
 * launches).  Calls on one server are serialized by the caller; the server
 * uses its engine exclusively while it exists. */
typedef struct gagp_server gagp_server;
enum {
  GAGP_REQUEST_QUEUED = 0,
  GAGP_REQUEST_RUNNING = 1,
  GAGP_REQUEST_DONE = 2,
  GAGP_REQUEST_FAILED = 3
};
/* memory_budget: device bytes the running searches may hold (0: the
 * engine's arena limit); max_active: running searches at most (0: no cap). */
gagp_status gagp_b200_server_create(gagp_engine* engine, uint64_t memory_budget, int32_t max_active,
                                    gagp_server** out);
void gagp_b200_server_destroy(gagp_server* server);
/* Rounds each step runs (1..4096, default 1) before it reads the searches'
 * states: the batch's round is captured once and replayed, and the host
 * reads states and retires searches once per step.  A search that finishes
 * within a step waits for the step's end; results do not depend on it. */
gagp_status gagp_b200_server_set_rounds_per_step(gagp_server* server, int32_t rounds);
/* Queues a search request (the blobs are copied).  Declines at once what
 * the engine would decline at admission (GAGP_DECLINED) and what can never
 * fit the budget (GAGP_OUT_OF_MEMORY). */
gagp_status gagp_b200_server_submit(gagp_server* server, const gagp_grammar* grammar, const gagp_cases* cases,
                                    const gagp_search_config* config, int64_t* ticket);
/* One serving step (see above); the counts after it. */
gagp_status gagp_b200_server_step(gagp_server* server, int32_t* running, int32_t* queued, int32_t* finished_now);
/* GAGP_REQUEST_* state of a ticket. */
gagp_status gagp_b200_server_poll(gagp_server* server, int64_t ticket, int32_t* state);
/* Seconds on the server's monotonic clock when the ticket was submitted,
 * admitted and finished (negative: not yet). */
gagp_status gagp_b200_server_times(gagp_server* server, int64_t ticket, double* submitted, double* admitted,
                                   double* finished);
/* Copies a finished request's result (as gagp_b200_search_result) and
 * releases the ticket; GAGP_NOT_READY before it finishes. */
gagp_status gagp_b200_server_result(gagp_server* server, int64_t ticket, gagp_search_result* out);
/* Drops a ticket in any state (a running search is stopped and freed). */
gagp_status gagp_b200_server_cancel(gagp_server* server, int64_t ticket);

/* Copies a finished search's history and final ranked population out (the
 * population is ranked and put in transport form on the device; in
 * final_rows, entries past a row's counts are set to 0). */
gagp_status gagp_b200_search_result(gagp_engine* engine, int32_t search, gagp_search_result* out);

#ifdef __cplusplus
}
#endif
#endif
