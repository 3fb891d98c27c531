/*
 * TEST INFRASTRUCTURE ONLY -- the oracle.  A serial C restatement of the
 * reference's CPU resident search path (HostPhasePopulation + the
 * steady-state loop), used by tests, smoke() and bench.py's CPU baseline as
 * the checker.  The product never links, loads or calls it.
 *
 * Parity pin: its outputs are checked against golden vectors produced by the
 * reference's own CPU engine compiled from source (oracle/ref_driver.cpp,
 * tests/golden/make_golden.py).
 */
#ifndef GAGP_ORACLE_H
#define GAGP_ORACLE_H
#include "../include/gagp_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Whole search: steady state (or generational), history and final ranked
 * population.  Returns 0 on success, nonzero with a message on failure. */
int gagp_oracle_search(const gagp_grammar* grammar, const gagp_cases* cases,
                       const gagp_search_config* config, const gagp_rows* initial,
                       gagp_search_result* out);

/* Initial population rows (generate_phase_initial_population). */
int gagp_oracle_initial_population(const gagp_grammar* grammar, const gagp_search_config* config,
                                   gagp_rows* out);

/* Fitness of rows (phase compiler + CPU VM + ordered reduction). */
/* gagp_oracle_search with the reference's reuse of any identical member's
 * result (member_reuse 1) or of the parent's only (0, as gagp_oracle_search). */
int gagp_oracle_search_reuse(const gagp_grammar* grammar, const gagp_cases* cases,
                             const gagp_search_config* config, const gagp_rows* initial,
                             gagp_search_result* result, int member_reuse);
/* One make_batch over the generated initial population (no cases needed). */
int gagp_oracle_make_batch(const gagp_grammar* grammar, const gagp_search_config* config, const double* selection,
                           uint64_t seed, gagp_rows* children, int32_t* reuse);
int gagp_oracle_evaluate(const gagp_grammar* grammar, const gagp_cases* cases,
                         const gagp_search_config* config, const gagp_rows* rows,
                         double* fitness, uint32_t* wrong, uint64_t* instructions);

/* Lowered bytecode of one row: code as (op, flags, a, b, fuel) quintuples,
 * constants as Int payloads.  Returns the instruction count or -1. */
int gagp_oracle_compile(const gagp_grammar* grammar, const int32_t* origins, int32_t node_count,
                        const int64_t* constants, int32_t constant_count, int32_t* code,
                        int32_t code_capacity, int64_t* out_constants, int32_t* out_constant_count,
                        int32_t* stack_bound);

/* MT19937-64 outputs (the run generator of evolve.cpp:339). */
void gagp_oracle_mt19937_64(uint64_t seed, uint64_t* out, int32_t count);

const char* gagp_oracle_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
