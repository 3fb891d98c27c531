/*
 * TEST INFRASTRUCTURE ONLY -- the oracle (see gagp_oracle.h).
 *
 * A plain serial C restatement of the reference's CPU resident search for
 * expression-entry grammars.  Every function cites the reference code it
 * follows; paths are relative to the reference project root.  Unlike the
 * product it keeps the reference's data layout (PhaseTreeNode, origins,
 * PhaseGeneSite and Value rows) so that it reads line by line against it.
 */
#include "gagp_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static char g_error[512];
const char* gagp_oracle_last_error(void) { return g_error; }
#define FAIL(...) do { snprintf(g_error, sizeof g_error, __VA_ARGS__); return -1; } while (0)

/* ----------------------------------------------------------------- types */
enum { EK_OPERATION, EK_CONSTANT, EK_BOUND, EK_REFERENCE, EK_INPUT, EK_ALIAS };
enum { TK_CONSTANT, TK_LOCAL, TK_OPERATION, TK_IF, TK_AND, TK_OR, TK_PROGRAM, TK_BLOCK, TK_NIL, TK_ASSIGN,
       TK_RETURN, TK_FOR_RANGE, TK_VAR };
#define STATEMENT_TAG 0xF0     /* kPhaseStatement, device/phase_compile.cuh:23 */
#define NAMED_LOCALS 16        /* kPhaseNamedLocals */
enum { ST_OK, ST_INVALID, ST_UNSUPPORTED, ST_CAPACITY };
enum {
  OP_PUSH_CONST = 0, OP_LOAD = 1, OP_STORE = 2, OP_NEG = 3, OP_NOT = 4, OP_ADD = 5, OP_SUB = 6,
  OP_MUL = 7, OP_DIV = 8, OP_MOD = 9, OP_LT = 10, OP_LE = 11, OP_GT = 12, OP_GE = 13, OP_EQ = 14,
  OP_NE = 15, OP_JMP = 16, OP_JMP_IF_FALSE = 17, OP_JMP_IF_TRUE = 18, OP_CALL_BUILTIN = 19,
  OP_RETURN = 20
};
enum { B_ABS = 0, B_MIN = 1, B_MAX = 2, B_IDIV0 = 13, B_IMOD0 = 14, B_TRUNC_DIV0 = 28, B_TRUNC_MOD0 = 29 };
#define NO_ID 0xFFFFFFFFu
#define FIXED_SITE (1 << 30)   /* kPhaseFixedSite, device/phase_generate.cuh:20 */
#define CAPACITY 1024          /* phase_operators.cuh:13 */
#define MAX_STACK 64

typedef struct { int kind, opcode, operand, arity; unsigned fuel, merge_fuel; int type; } Node;
typedef struct { int nonterminal, entry_expression, parent_scope, scope; } Site;
typedef struct { int64_t i; int tag; int b; } Val;
typedef struct { int status, nodes, constants, steps; } Gen;

typedef struct {
  const Node* nodes; const int* origins; const Site* sites; const Val* constants;
  int node_count, constant_count;
} View;
typedef struct { Node* nodes; int* origins; Site* sites; Val* constants; int capacity; } Out;

/* Fixed-capacity rows, the reference's host layout (phase_population_cpu.cpp:28-35). */
typedef struct {
  int cap;
  Node* nodes; int* origins; Site* sites; Val* constants; Gen* lengths;
} Trees;

static int trees_alloc(Trees* t, int rows, int cap) {
  t->cap = cap;
  t->nodes = calloc((size_t)rows * cap, sizeof(Node));
  t->origins = calloc((size_t)rows * cap, sizeof(int));
  t->sites = calloc((size_t)rows * cap, sizeof(Site));
  t->constants = calloc((size_t)rows * cap, sizeof(Val));
  t->lengths = calloc((size_t)rows, sizeof(Gen));
  return t->nodes && t->origins && t->sites && t->constants && t->lengths ? 0 : -1;
}
static void trees_free(Trees* t) {
  free(t->nodes); free(t->origins); free(t->sites); free(t->constants); free(t->lengths);
}
static View view_of(const Trees* t, int row) {
  View v = {t->nodes + (size_t)row * t->cap, t->origins + (size_t)row * t->cap,
            t->sites + (size_t)row * t->cap, t->constants + (size_t)row * t->cap,
            t->lengths[row].nodes, t->lengths[row].constants};
  return v;
}
static Out out_of(const Trees* t, int row) {
  Out o = {t->nodes + (size_t)row * t->cap, t->origins + (size_t)row * t->cap,
           t->sites + (size_t)row * t->cap, t->constants + (size_t)row * t->cap, CAPACITY};
  return o;
}

/* The admitted grammar view (PhaseGrammarView, device/phase_generate.cuh:107-117). */
typedef struct {
  const gagp_grammar* g;
  Node* expr_node;   /* PhaseExpression::node per expression */
} Grammar;

static Node expression_node(const gagp_expression* e) {
  Node n = {e->node_kind, e->opcode, e->operand, e->arity, e->fuel, e->merge_fuel, e->type};
  return n;
}

/* Definite assignment of grammar locals in a statement program
 * (phase_locals_defined, device/phase_compile.cuh:170-200): a local is
 * readable after an assign, inside a for_range body naming it, and after a
 * statement if only when both branches assigned it; a loop body's
 * assignments end with the loop; inputs are always defined. */
static int locals_defined(const Node* nodes, int count) {
  struct { int index, seen; unsigned saved, branch; } frames[64];
  int depth = 0;
  unsigned mask = 0;
#define LOCAL_BIT(operand) ((operand) >= 0 && (operand) < NAMED_LOCALS ? 1u << (operand) : 0u)
  for (int i = 0; i < count; ++i) {
    const Node node = nodes[i];
    if (node.kind == TK_VAR && !(mask & LOCAL_BIT(node.operand))) return 0;
    if (node.arity > 0) {
      if (depth == 64) return 0;
      frames[depth].index = i; frames[depth].seen = 0; frames[depth].saved = mask; frames[depth].branch = 0;
      ++depth;
      continue;
    }
    while (depth) {
      const Node owner = nodes[frames[depth - 1].index];
      const int seen = ++frames[depth - 1].seen;
      if (owner.kind == TK_FOR_RANGE && seen == 1) {
        frames[depth - 1].saved = mask; mask |= LOCAL_BIT(owner.operand);
      } else if (owner.kind == TK_IF && owner.type == STATEMENT_TAG) {
        if (seen == 1) frames[depth - 1].saved = mask;
        else if (seen == 2) { frames[depth - 1].branch = mask; mask = frames[depth - 1].saved; }
        else mask &= frames[depth - 1].branch;
      }
      if (seen < owner.arity) break;
      if (owner.kind == TK_ASSIGN) mask |= LOCAL_BIT(owner.operand);
      else if (owner.kind == TK_FOR_RANGE) mask = frames[depth - 1].saved;
      --depth;
    }
  }
#undef LOCAL_BIT
  return depth == 0;
}

/* ------------------------------------------------ grammar random (SplitMix64)
 * DGrammarRandom, cpp/src/evolution/repro/gpu/device/grammar_random.cuh:10-51 */
typedef struct { uint64_t state; } Rng;
static uint64_t rng_next(Rng* r) {
  uint64_t v = (r->state += 0x9e3779b97f4a7c15ULL);
  v = (v ^ (v >> 30)) * 0xbf58476d1ce4e5b9ULL;
  v = (v ^ (v >> 27)) * 0x94d049bb133111ebULL;
  return v ^ (v >> 31);
}
static uint64_t rng_bounded(Rng* r, uint64_t upper) {
  const uint64_t threshold = (0 - upper) % upper;
  for (;;) {
    const uint64_t v = rng_next(r);
    if (v >= threshold) return v % upper;
  }
}
static int64_t rng_integer(Rng* r, int64_t minimum, int64_t maximum) {
  const uint64_t sign = 1ULL << 63;
  const uint64_t first = (uint64_t)minimum ^ sign, last = (uint64_t)maximum ^ sign;
  const uint64_t width = last - first + 1;
  const uint64_t bits = (first + (width ? rng_bounded(r, width) : rng_next(r))) ^ sign;
  if (bits < sign) return (int64_t)bits;
  return INT64_MIN + (int64_t)(bits - sign);
}
static double rng_unit(Rng* r) { return (double)(rng_next(r) >> 11) * 0x1.0p-53; }

/* ---------------------------------------------------------------- MT19937-64
 * std::mt19937_64 (the run generator, cpp/src/evolution/evolve.cpp:339): the
 * published Matsumoto-Nishimura 64-bit Mersenne Twister. */
typedef struct { uint64_t mt[312]; int index; } Mt;
static void mt_seed(Mt* m, uint64_t seed) {
  m->mt[0] = seed;
  for (int i = 1; i < 312; ++i) m->mt[i] = 6364136223846793005ULL * (m->mt[i - 1] ^ (m->mt[i - 1] >> 62)) + (uint64_t)i;
  m->index = 312;
}
static uint64_t mt_next(Mt* m) {
  if (m->index >= 312) {
    for (int i = 0; i < 312; ++i) {
      const uint64_t x = (m->mt[i] & 0xFFFFFFFF80000000ULL) | (m->mt[(i + 1) % 312] & 0x7FFFFFFFULL);
      m->mt[i] = m->mt[(i + 156) % 312] ^ (x >> 1) ^ ((x & 1) ? 0xB5026F5AA96619E9ULL : 0);
    }
    m->index = 0;
  }
  uint64_t x = m->mt[m->index++];
  x ^= (x >> 29) & 0x5555555555555555ULL;
  x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
  x ^= (x << 37) & 0xFFF7EEE000000000ULL;
  x ^= x >> 43;
  return x;
}
void gagp_oracle_mt19937_64(uint64_t seed, uint64_t* out, int32_t count) {
  Mt m;
  mt_seed(&m, seed);
  for (int i = 0; i < count; ++i) out[i] = mt_next(&m);
}

/* ------------------------------------------------------------ tree utilities
 * device/phase_variation.cuh:81-142 */
static int subtree_end(const View* t, int start) {
  if (!t->nodes || start < 0 || start >= t->node_count || t->node_count > 1024) return -1;
  int pending = 1;
  for (int i = start; i < t->node_count; ++i) {
    const int arity = t->nodes[i].arity;
    if (arity < 0 || arity > 8) return -1;
    pending += arity - 1;
    if (!pending) return i + 1;
  }
  return -1;
}
static int node_depth(const View* t, int position) {
  if (!t->nodes || position < 0 || position >= t->node_count || t->node_count > 1024) return -1;
  int pending[64], depth = 1;
  pending[0] = 1;
  for (int i = 0; i <= position; ++i) {
    while (depth && !pending[depth - 1]) --depth;
    if (!depth) return -1;
    if (i == position) return depth;
    --pending[depth - 1];
    const int arity = t->nodes[i].arity;
    if (arity < 0 || arity > 8) return -1;
    if (arity) { if (depth == 64) return -1; pending[depth++] = arity; }
  }
  return -1;
}
static int site_depth(const Node* nodes, const Site* sites, int count, int position) {
  if (!nodes || !sites || count <= 0 || count > 1024 || position >= count) return -1;
  int pending[64], incoming[64], depth = 1, maximum = 0;
  pending[0] = 1; incoming[0] = 0;
  for (int i = 0; i < count; ++i) {
    while (depth && !pending[depth - 1]) --depth;
    if (!depth) return -1;
    if (i == position) return incoming[depth - 1];
    const int arity = nodes[i].arity;
    if (arity < 0 || arity > 8) return -1;
    const int value = incoming[depth - 1] + (sites[i].nonterminal >= 0 ? 1 : 0);
    maximum = value > maximum ? value : maximum;
    --pending[depth - 1];
    if (arity) { if (depth == 64) return -1; pending[depth] = arity; incoming[depth++] = value; }
  }
  while (depth && !pending[depth - 1]) --depth;
  return depth ? -1 : maximum;
}

/* splice_phase_tree<FusedDepth=true>, device/phase_variation.cuh:147-207 */
static Gen splice(const View* base, int destination, const View* donor, int source, Out out,
                  int max_depth, int site_limit) {
  Gen result = {ST_INVALID, 0, 0, 0};
  if (out.capacity <= 0 || out.capacity > 1024 || max_depth <= 0 || max_depth > 64 ||
      base->node_count <= 0 || base->node_count > 1024 || donor->node_count <= 0 || donor->node_count > 1024 ||
      base->constant_count < 0 || base->constant_count > base->node_count || donor->constant_count < 0 ||
      donor->constant_count > donor->node_count || destination < 0 || destination >= base->node_count ||
      source < 0 || source >= donor->node_count)
    return result;
  const Site a = base->sites[destination], b = donor->sites[source];
  if (a.nonterminal < 0 || a.nonterminal != b.nonterminal || a.scope != b.scope) return result;
  const int end = subtree_end(base, destination), donor_end = subtree_end(donor, source);
  if (end < 0 || donor_end < 0) return result;
  const int length = base->node_count - (end - destination) + donor_end - source;
  if (length > out.capacity) { result.status = ST_CAPACITY; return result; }
  int pending[64], depth = 1, maximum = 1;
  pending[0] = 1;
  for (int i = 0; i < length; ++i) {
    const int incoming = i >= destination && i < destination + donor_end - source;
    const View* tree = incoming ? donor : base;
    const int index = incoming ? source + i - destination : i < destination ? i : i + (end - destination) - (donor_end - source);
    Node node = tree->nodes[index];
    while (depth && !pending[depth - 1]) --depth;
    if (!depth || node.arity < 0 || node.arity > 8) return result;
    maximum = depth > maximum ? depth : maximum;
    --pending[depth - 1];
    if (node.arity) { if (depth == 64) return result; pending[depth++] = node.arity; }
    if (node.kind == TK_CONSTANT) {
      if (node.operand < 0 || node.operand >= tree->constant_count) return result;
      node.operand = result.constants;
      out.constants[result.constants++] = tree->constants[tree->nodes[index].operand];
    }
    out.nodes[i] = node; out.origins[i] = tree->origins[index]; out.sites[i] = tree->sites[index];
  }
  out.sites[destination] = a;
  while (depth && !pending[depth - 1]) --depth;
  if (depth) return result;
  if (maximum > max_depth) { result.status = ST_CAPACITY; return result; }
  if (site_limit) {
    const int height = site_depth(out.nodes, out.sites, length, -1);
    if (height < 0) return result;
    if (height > site_limit) { result.status = ST_CAPACITY; return result; }
  }
  result.nodes = length; result.status = ST_OK;
  return result;
}

/* ---------------------------------------------------------------- generation
 * generate_phase<CompactTasks, EmitSites, false>, device/phase_generate.cuh:125-270 */
static unsigned minimum_of(const gagp_grammar* g, int expression, int d, int logical) {
  if (expression < 0 || expression >= g->expression_count || d < 0 || d >= g->depth_count ||
      logical < 0 || logical >= g->logical_depth_count)
    return NO_ID;
  return g->minimum[((size_t)expression * g->depth_count + d) * g->logical_depth_count + logical];
}
typedef struct { unsigned expression, depth, scope_count, logical, scope; } Task;

static Gen generate_phase(const Grammar* G, int root_expression, int scope_count, int depth, int capacity,
                          uint64_t seed, Node* nodes, int* origins, Val* constants, Site* sites,
                          int logical_depth) {
  const gagp_grammar* g = G->g;
  Gen result = {ST_INVALID, 0, 0, 0};
  Site next_site = {-1, -1, 0, 0};
  const int site_limited = g->site_depth > 0;
  if (root_expression < 0 || root_expression >= g->expression_count || scope_count < 0 || scope_count > 15 ||
      depth <= 0 || depth >= g->depth_count || depth > 64 || logical_depth < 0 ||
      logical_depth >= g->logical_depth_count || capacity <= 0 || capacity > 1024 || g->expression_count > 131071)
    return result;
  const unsigned unselected = 131071;
  Task pending[192];
  int count = 1;
  pending[0].expression = (unsigned)root_expression; pending[0].depth = (unsigned)depth;
  pending[0].scope_count = (unsigned)scope_count; pending[0].scope = 0; pending[0].logical = (unsigned)logical_depth;
  unsigned reserved = minimum_of(g, root_expression, depth, logical_depth);
  if (reserved > (unsigned)capacity) { result.status = ST_CAPACITY; return result; }
  Rng random = {seed};
  while (count) {
    if (++result.steps > 8192) { result.status = ST_CAPACITY; return result; }
    const Task task = pending[--count];
    const unsigned required = minimum_of(g, (int)task.expression, (int)task.depth, (int)task.logical);
    if (required > reserved) return result;
    reserved -= required;
    const gagp_expression* expression = &g->expressions[task.expression];
    if (expression->kind == EK_REFERENCE) {
      if (expression->target < 0 || expression->target >= g->nonterminal_count || expression->scope_count < 0 ||
          expression->scope_count > 8)
        return result;
      const gagp_nonterminal* nt = &g->nonterminals[expression->target];
      if (sites) {
        if (next_site.nonterminal >= 0) return result;
        next_site.nonterminal = expression->target; next_site.entry_expression = (int)task.expression;
        next_site.parent_scope = (int)task.scope_count;
        next_site.scope = expression->scope_count | (nt->fixed ? FIXED_SITE : 0);
      }
      if (nt->scope_count != expression->scope_count || nt->production_offset < 0 || nt->production_count <= 0 ||
          nt->production_offset > g->production_count || nt->production_count > g->production_count - nt->production_offset)
        return result;
      if (site_limited && task.logical == 0) { result.status = ST_CAPACITY; return result; }
      Task next = {unselected, task.depth, (unsigned)expression->scope_count,
                   task.logical - (site_limited ? 1u : 0u), 0};
      if (reserved > (unsigned)(capacity - result.nodes)) { result.status = ST_CAPACITY; return result; }
      const unsigned available = (unsigned)(capacity - result.nodes) - reserved;
      double maximum = nt->normalized_weights ? 1 : 0, total = 0;
      if (!nt->normalized_weights)
        for (int i = 0; i < nt->production_count; ++i) {
          const gagp_production* p = &g->productions[nt->production_offset + i];
          if (minimum_of(g, p->expression, (int)task.depth, (int)next.logical) <= available && p->weight > maximum)
            maximum = p->weight;
        }
      if (!(maximum > 0)) { result.status = ST_CAPACITY; return result; }
      for (int i = 0; i < nt->production_count; ++i) {
        const gagp_production* p = &g->productions[nt->production_offset + i];
        if (minimum_of(g, p->expression, (int)task.depth, (int)next.logical) <= available)
          total += nt->normalized_weights ? p->weight : p->weight / maximum;
      }
      double choice = (double)(rng_next(&random) >> 11) * 0x1.0p-53 * total;
      for (int i = 0; i < nt->production_count; ++i) {
        const gagp_production* p = &g->productions[nt->production_offset + i];
        if (minimum_of(g, p->expression, (int)task.depth, (int)next.logical) > available) continue;
        if (p->expression < 0 || p->expression >= g->expression_count) return result;
        next.expression = (unsigned)p->expression;
        choice -= nt->normalized_weights ? p->weight : p->weight / maximum;
        if (choice < 0) break;
      }
      if (next.expression == unselected || count >= 192) return result;
      reserved += minimum_of(g, (int)next.expression, (int)next.depth, (int)next.logical);
      pending[count++] = next;
      continue;
    }
    if (expression->kind == EK_ALIAS) {
      const int child = expression->children[0];
      if (child < 0 || child >= g->expression_count || count >= 192) return result;
      Task next = task;
      next.expression = (unsigned)child;
      next.scope_count = expression->child_scope[0] >= 0 ? (unsigned)expression->child_scope[0] : task.scope_count;
      reserved += minimum_of(g, child, (int)task.depth, (int)task.logical);
      pending[count++] = next;
      continue;
    }
    if (task.depth <= 0 || result.nodes >= capacity) { result.status = ST_CAPACITY; return result; }
    Node node = G->expr_node[task.expression];
    if (node.arity < 0 || node.arity > 8) return result;
    if (expression->kind == EK_BOUND) {
      if (node.arity != 0 || node.operand < 0 || node.operand >= 16) return result;
    } else if (expression->kind == EK_CONSTANT) {
      if (expression->target < 0 || expression->target >= g->domain_count || node.arity != 0) return result;
      const gagp_domain* domain = &g->domains[expression->target];
      Val value = {0, GAGP_TAG_INVALID, 0};
      if (domain->integer_range) {
        if (domain->minimum > domain->maximum) return result;
        value.tag = GAGP_TAG_INT;
        value.i = rng_integer(&random, domain->minimum, domain->maximum);
      } else {
        if (domain->value_offset < 0 || domain->value_count <= 0 || domain->value_offset > g->value_count ||
            domain->value_count > g->value_count - domain->value_offset)
          return result;
        const gagp_value* v = &g->values[domain->value_offset + rng_bounded(&random, (uint64_t)domain->value_count)];
        value.tag = v->tag;
        if (v->tag == GAGP_TAG_BOOL) value.b = v->i != 0; else value.i = v->i;
      }
      if (value.tag == GAGP_TAG_INVALID) return result;
      node.operand = result.constants;
      constants[result.constants++] = value;
    } else if (expression->kind != EK_OPERATION && expression->kind != EK_INPUT) {
      return result;
    }
    if (sites) { sites[result.nodes] = next_site; next_site.nonterminal = -1; next_site.entry_expression = -1;
                 next_site.parent_scope = 0; next_site.scope = 0; }
    origins[result.nodes] = (int)task.expression;
    nodes[result.nodes++] = node;
    for (int i = node.arity - 1; i >= 0; --i) {
      if (count >= 192) { result.status = ST_CAPACITY; return result; }
      const int child = expression->children[i];
      const unsigned need = minimum_of(g, child, (int)task.depth - 1, (int)task.logical);
      if (need > (unsigned)(capacity - result.nodes) || reserved > (unsigned)(capacity - result.nodes) - need) {
        result.status = ST_CAPACITY; return result;
      }
      Task next = task;
      next.expression = (unsigned)child;
      --next.depth;
      next.scope_count = expression->child_scope[i] >= 0 ? (unsigned)expression->child_scope[i] : task.scope_count;
      pending[count++] = next;
      reserved += need;
    }
  }
  if (reserved || !result.nodes) return result;
  result.status = ST_OK;
  return result;
}

/* ---------------------------------------------------------------- operators
 * phase_operators.cuh:38-265 (Warp=false bodies) */
typedef struct { int parent, crossover_attempted, crossover, crossover_rejected, mutation, changed, error, reusable_parent; } Stat;
typedef struct { int counted_sites, uniform_phase; double crossover_probability; int crossover_attempts, mutation_max_nodes; } Policy;
typedef struct { int row, node; } SiteRef;

static int valid(const Gen* r) {
  return r->status == ST_OK && r->nodes > 0 && r->nodes <= CAPACITY && r->constants >= 0 && r->constants <= r->nodes;
}
static void copy_tree(const Trees* from, int source, Trees* to, int target) {
  const Gen r = from->lengths[source];
  memset(&to->lengths[target], 0, sizeof(Gen));
  to->lengths[target].status = ST_INVALID;
  if (!valid(&r)) return;
  const View a = view_of(from, source);
  const Out b = out_of(to, target);
  for (int i = 0; i < r.nodes; ++i) { b.nodes[i] = a.nodes[i]; b.origins[i] = a.origins[i]; b.sites[i] = a.sites[i]; }
  for (int i = 0; i < r.constants; ++i) b.constants[i] = a.constants[i];
  to->lengths[target] = r;
}
/* Tournament on selection values (phase_operators.cuh:46-50). */
static int tournament(const double* fitness, int population, int pressure, Rng* random) {
  int best = (int)rng_bounded(random, (uint64_t)population);
  for (int i = 1; i < pressure; ++i) {
    const int candidate = (int)rng_bounded(random, (uint64_t)population);
    if (fitness[candidate] > fitness[best]) best = candidate;
  }
  return best;
}
static int site_matches(const View* t, int i, int nt, int scope) {
  return t->sites[i].nonterminal >= 0 && !(t->sites[i].scope & FIXED_SITE) &&
         (nt < 0 || (t->sites[i].nonterminal == nt && t->sites[i].scope == scope));
}
static SiteRef choose_site(const Trees* trees, int program, int slots, Rng* random, int counted, int nt, int scope,
                           int selected_slot) {
  SiteRef none = {-1, -1};
  if (selected_slot < -1 || selected_slot >= slots) return none;
  const int first = selected_slot < 0 ? 0 : selected_slot, last = selected_slot < 0 ? slots : selected_slot + 1;
  if (counted) {
    unsigned count = 0;
    for (int k = first; k < last; ++k) {
      const int row = program * slots + k;
      if (!valid(&trees->lengths[row])) return none;
      const View t = view_of(trees, row);
      for (int i = 0; i < t.node_count; ++i) if (site_matches(&t, i, nt, scope)) ++count;
    }
    if (!count) return none;
    unsigned rank = (unsigned)rng_bounded(random, count);
    for (int k = first; k < last; ++k) {
      const int row = program * slots + k;
      const View t = view_of(trees, row);
      for (int i = 0; i < t.node_count; ++i)
        if (site_matches(&t, i, nt, scope)) {
          if (rank == 0) { SiteRef s = {row, i}; return s; }
          --rank;
        }
    }
    return none;
  }
  SiteRef selected = none;
  unsigned count = 0;
  for (int k = first; k < last; ++k) {
    const int row = program * slots + k;
    if (!valid(&trees->lengths[row])) return none;
    const View t = view_of(trees, row);
    for (int i = 0; i < t.node_count; ++i)
      if (site_matches(&t, i, nt, scope))
        if (rng_bounded(random, ++count) == 0) { selected.row = row; selected.node = i; }
  }
  return selected;
}

typedef struct {
  Grammar G;
  int root, scope, max_depth, logical_depth, type;
} Slot;

static void crossover_child(int child, const Trees* input, Trees* output, const Slot* slots, int slot_count,
                            int population, int max_variable_nodes, const double* fitness, int pressure,
                            uint64_t seed, const Policy* policy, Stat* stat) {
  Rng random = {seed ^ (0x617089e168ULL + (uint64_t)child)};
  memset(stat, 0, sizeof *stat);
  stat->parent = -1; stat->reusable_parent = -1;
  const int parent = tournament(fitness, population, pressure, &random);
  const int donor = tournament(fitness, population, pressure, &random);
  stat->parent = parent;
  int total = 0;
  for (int k = 0; k < slot_count; ++k) {
    const int row = parent * slot_count + k;
    if (!valid(&input->lengths[row])) { stat->error = 1; return; }
    total += input->lengths[row].nodes;
    copy_tree(input, row, output, child * slot_count + k);
  }
  if (policy->crossover_probability < 1 && rng_unit(&random) >= policy->crossover_probability) return;
  stat->crossover_attempted = 1;
  const int selected_slot = policy->uniform_phase ? (int)rng_bounded(&random, (uint64_t)slot_count) : -1;
  for (int attempt = 0; attempt < policy->crossover_attempts; ++attempt) {
    const SiteRef destination = choose_site(input, parent, slot_count, &random, policy->counted_sites, -1, -1, selected_slot);
    if (destination.node < 0) break;
    const View a = view_of(input, destination.row);
    const Site contract = a.sites[destination.node];
    const SiteRef source = choose_site(input, donor, slot_count, &random, policy->counted_sites, contract.nonterminal,
                                       contract.scope, selected_slot);
    if (source.node < 0) { ++stat->crossover_rejected; continue; }
    const View b = view_of(input, source.row);
    const int ae = subtree_end(&a, destination.node), be = subtree_end(&b, source.node);
    if (ae < 0 || be < 0) { stat->error = 3; return; }
    if (total - (ae - destination.node) + (be - source.node) > max_variable_nodes) { ++stat->crossover_rejected; continue; }
    const int slot = destination.row % slot_count, target = child * slot_count + slot;
    const Slot* s = &slots[slot];
    const Gen r = splice(&a, destination.node, &b, source.node, out_of(output, target), s->max_depth, s->logical_depth);
    /* a statement program must read only definitely assigned locals
     * (locals_defined, phase_operators.cuh:148-154,185) */
    if (r.status == ST_OK && (s->type != STATEMENT_TAG || locals_defined(out_of(output, target).nodes, r.nodes))) {
      output->lengths[target] = r;
      stat->crossover = 1;
      return;
    }
    copy_tree(input, destination.row, output, target);
    ++stat->crossover_rejected;
  }
}

static void mutate_child(int child, Trees* input, Trees* output, Trees* scratch, const Slot* slots, int slot_count,
                         int max_variable_nodes, double probability, uint64_t seed, const Policy* policy, Stat* stat) {
  if (stat->error) return;
  int total = 0;
  for (int k = 0; k < slot_count; ++k) {
    const int row = child * slot_count + k;
    if (!valid(&input->lengths[row])) { stat->error = 4; return; }
    total += input->lengths[row].nodes;
  }
  Rng random = {seed ^ (0x124ab512bf01ULL + (uint64_t)child)};
  if (rng_unit(&random) >= probability) return;
  const int selected_slot = policy->uniform_phase ? (int)rng_bounded(&random, (uint64_t)slot_count) : -1;
  const SiteRef destination = choose_site(input, child, slot_count, &random, policy->counted_sites, -1, -1, selected_slot);
  if (destination.node < 0) return;
  const View a = view_of(input, destination.row);
  const int end = subtree_end(&a, destination.node), depth = node_depth(&a, destination.node);
  if (end < 0 || depth < 0) { stat->error = 6; return; }
  const Site site = a.sites[destination.node];
  const Slot* slot = &slots[destination.row % slot_count];
  Out tmp = out_of(scratch, child);
  const int incoming = slot->logical_depth ? site_depth(a.nodes, a.sites, a.node_count, destination.node) : 0;
  if (incoming < 0 || incoming > slot->logical_depth) { stat->error = 6; return; }
  const int logical = slot->logical_depth - incoming;
  const int replaced = end - destination.node;
  const int whole = max_variable_nodes - (total - replaced), phase = CAPACITY - (a.node_count - replaced);
  const int available = whole < phase ? whole : phase, uncapped = available < CAPACITY ? available : CAPACITY;
  const int capped = policy->mutation_max_nodes > 0 && policy->mutation_max_nodes < uncapped;
  const int bounded = capped ? policy->mutation_max_nodes : uncapped;
  const Gen generated = generate_phase(&slot->G, site.entry_expression, site.parent_scope, slot->max_depth - depth + 1,
                                       bounded, rng_next(&random), tmp.nodes, tmp.origins, tmp.constants, tmp.sites, logical);
  if (capped && generated.status == ST_CAPACITY) return;
  if (generated.status != ST_OK) { stat->error = 7; return; }
  scratch->lengths[child] = generated;
  const View donor = view_of(scratch, child);
  const Gen r = splice(&a, destination.node, &donor, 0, out_of(output, child), slot->max_depth, slot->logical_depth);
  if (r.status != ST_OK) { stat->error = 8; return; }
  /* an undefined local read drops the mutation; the crossed child stands */
  if (slot->type == STATEMENT_TAG && !locals_defined(out_of(output, child).nodes, r.nodes)) return;
  output->lengths[child] = r;
  copy_tree(output, child, input, destination.row);
  stat->mutation = 1;
}

static void compare_child(int child, const Trees* parents, const Trees* children, int population, int slot_count, Stat* stat) {
  if (stat->error) return;
  const int parent = stat->parent;
  if (parent < 0 || parent >= population) { stat->error = 9; return; }
  int equal = 1, reusable = 1;
  for (int k = 0; k < slot_count && equal; ++k) {
    const View a = view_of(parents, parent * slot_count + k), b = view_of(children, child * slot_count + k);
    if (a.node_count != b.node_count || a.constant_count != b.constant_count) { equal = 0; break; }
    for (int i = 0; i < a.node_count && equal; ++i) {
      const Node x = a.nodes[i], y = b.nodes[i];
      equal = x.kind == y.kind && x.opcode == y.opcode && x.operand == y.operand && x.arity == y.arity &&
              x.fuel == y.fuel && x.merge_fuel == y.merge_fuel && a.origins[i] == b.origins[i];
    }
    for (int i = 0; i < a.constant_count && equal; ++i) {
      const Val x = a.constants[i], y = b.constants[i];
      equal = x.tag == y.tag && (x.tag == GAGP_TAG_BOOL ? x.b == y.b : x.i == y.i);
      reusable = reusable && x.i == y.i && x.b == y.b;
    }
  }
  stat->changed = !equal;
  stat->reusable_parent = equal && reusable ? parent : -1;
}

/* ------------------------------------------------------------------ lowering
 * compile_phase_tree for value phases (Constant, Local, Operation, If, And,
 * Or), device/phase_compile.cuh:207-895, followed by patch_whole_program's
 * RETURN (phase_layout.hpp:476-500). */
typedef struct { int op, flags, a, b; unsigned fuel; } Instr;
typedef struct {
  Instr* code; Val* consts; int code_cap, const_cap;
  int status, code_count, const_count, stack_bound, stack;
} Emit;
/* Exact-identity reuse of any current member's result (the CPU owner's
 * member_hashes lookup, phase_population_cpu.cpp:318-320,341-344, with
 * hash_program / equal_program of parent_fitness_cache.cuh:15-43): a child
 * whose genotype equals some member's takes that member's completed result.
 * The hash only chooses candidates; equality of every field decides. */
static uint64_t fnv_mix(uint64_t h, uint64_t x) { return (h ^ x) * 0x100000001b3ULL; }
static uint64_t row_hash(const View* t) {
  uint64_t h = 0xcbf29ce484222325ULL;
  h = fnv_mix(fnv_mix(h, (uint64_t)t->node_count), (uint64_t)t->constant_count);
  for (int i = 0; i < t->node_count; ++i) {
    const Node* n = &t->nodes[i];
    h = fnv_mix(h, (unsigned)n->kind); h = fnv_mix(h, (unsigned)n->opcode); h = fnv_mix(h, (uint64_t)(int64_t)n->operand);
    h = fnv_mix(h, (uint64_t)(int64_t)n->arity); h = fnv_mix(h, n->fuel); h = fnv_mix(h, n->merge_fuel);
    h = fnv_mix(h, (uint64_t)(int64_t)t->origins[i]);
  }
  for (int i = 0; i < t->constant_count; ++i) {
    const Val* v = &t->constants[i];
    h = fnv_mix(h, (unsigned)v->tag); h = fnv_mix(h, (uint64_t)v->i); h = fnv_mix(h, (uint64_t)(int64_t)v->b);
  }
  return h;
}
static int rows_equal(const View* x, const View* y) {
  if (x->node_count != y->node_count || x->constant_count != y->constant_count) return 0;
  for (int i = 0; i < x->node_count; ++i) {
    const Node* u = &x->nodes[i]; const Node* v = &y->nodes[i];
    if (u->kind != v->kind || u->opcode != v->opcode || u->operand != v->operand || u->arity != v->arity ||
        u->fuel != v->fuel || u->merge_fuel != v->merge_fuel || x->origins[i] != y->origins[i]) return 0;
  }
  for (int i = 0; i < x->constant_count; ++i) {
    const Val* u = &x->constants[i]; const Val* v = &y->constants[i];
    if (u->tag != v->tag || u->i != v->i || u->b != v->b) return 0;
  }
  return 1;
}
/* The lowest-indexed member equal to `child` of `children`, or -1. */
static int find_member(const Trees* members, const uint64_t* member_hash, int population, const Trees* children, int child) {
  const View c = view_of(children, child);
  const uint64_t h = row_hash(&c);
  for (int m = 0; m < population; ++m) {
    if (member_hash[m] != h) continue;
    const View v = view_of(members, m);
    if (rows_equal(&v, &c)) return m;
  }
  return -1;
}

static int emit(Emit* o, int op, unsigned fuel, int a, int b, int flags) {
  if (o->code_count >= o->code_cap) { o->status = ST_CAPACITY; return 0; }
  if (fuel > 0x7fffffffU) { o->status = ST_INVALID; return 0; }
  Instr x = {op, flags, a, b, fuel};
  o->code[o->code_count++] = x;
  return 1;
}
static int add_const(Emit* o, Val v) {
  if (o->const_count >= o->const_cap) { o->status = ST_CAPACITY; return -1; }
  o->consts[o->const_count] = v;
  return o->const_count++;
}
static void grow(Emit* o, int by) { o->stack += by; if (o->stack > o->stack_bound) o->stack_bound = o->stack; }

static int operation_type(const Node* node, const int* args) {
  const int I = GAGP_TAG_INT, B = GAGP_TAG_BOOL, X = GAGP_TAG_INVALID;
  if (node->opcode == OP_NEG) return node->arity == 1 && args[0] == I ? I : X;
  if (node->opcode == OP_NOT) return node->arity == 1 && args[0] == B ? B : X;
  switch (node->opcode) {
    case OP_ADD: case OP_SUB: case OP_MUL: case OP_MOD:
      return node->arity == 2 && args[0] == I && args[1] == I ? I : X;
    case OP_LT: case OP_LE: case OP_GT: case OP_GE:
      return node->arity == 2 && args[0] == I && args[1] == I ? B : X;
    case OP_EQ: case OP_NE:
      return node->arity == 2 && args[0] == args[1] && (args[0] == I || args[0] == B) ? B : X;
    case OP_CALL_BUILTIN: break;
    default: return X;
  }
  switch (node->operand) {
    case B_TRUNC_DIV0: case B_TRUNC_MOD0: case B_IDIV0: case B_IMOD0: case B_MIN: case B_MAX:
      return node->arity == 2 && args[0] == I && args[1] == I ? I : X;
    default: return X;
  }
}

typedef struct { Node node; int base_stack, first_jump, second_jump; int args[3]; int seen; } Frame;

static int compile_row(const Node* nodes, int node_count, const Val* constants, int constant_count,
                       const int* local_types, int local_count, int expected, Emit* out) {
  out->status = ST_INVALID; out->code_count = out->const_count = out->stack_bound = out->stack = 0;
  if (!nodes || node_count <= 0 || node_count > 4096 || local_count < 0 || local_count > 64) return -1;
  Frame frames[64];
  int depth = 0, cursor = 0, have_value = 0, completed = GAGP_TAG_INVALID;
  for (;;) {
    if (!have_value) {
      if (cursor >= node_count) return -1;
      const Node node = nodes[cursor++];
      if (node.kind == TK_CONSTANT) {
        if (node.arity != 0 || node.operand < 0 || node.operand >= constant_count) return -1;
        const Val v = constants[node.operand];
        if (v.tag != GAGP_TAG_INT && v.tag != GAGP_TAG_BOOL) { out->status = ST_UNSUPPORTED; return -1; }
        const int index = add_const(out, v);
        if (index < 0 || !emit(out, OP_PUSH_CONST, node.fuel, index, 0, 1)) return -1;
        grow(out, 1);
        completed = v.tag; have_value = 1;
      } else if (node.kind == TK_LOCAL) {
        if (node.arity != 0 || node.operand < 0 || node.operand >= local_count) return -1;
        completed = local_types[node.operand];
        if (!emit(out, OP_LOAD, node.fuel, node.operand, 0, 1)) return -1;
        grow(out, 1);
        have_value = 1;
      } else {
        if (node.arity < 1 || node.arity > 3) return -1;
        if (node.kind == TK_IF) { if (node.arity != 3) return -1; }
        else if (node.kind == TK_AND || node.kind == TK_OR) { if (node.arity != 2) return -1; }
        else if (node.kind != TK_OPERATION) { out->status = ST_UNSUPPORTED; return -1; }
        if (depth == 64) { out->status = ST_CAPACITY; return -1; }
        Frame f = {node, out->stack, -1, -1, {0, 0, 0}, 0};
        frames[depth++] = f;
        continue;
      }
    }
    if (depth == 0) {
      if (cursor != node_count || out->stack != 1 || completed != expected) return -1;
      if (out->stack_bound > MAX_STACK) { out->status = ST_CAPACITY; return -1; }
      out->status = ST_OK;
      return 0;
    }
    Frame* frame = &frames[depth - 1];
    const Node node = frame->node;
    if (frame->seen < 3) frame->args[frame->seen] = completed;
    ++frame->seen;
    const int branch = node.kind == TK_IF || node.kind == TK_AND || node.kind == TK_OR;
    if (branch && frame->seen == 1) {
      if (completed != GAGP_TAG_BOOL) return -1;
      frame->first_jump = out->code_count;
      if (!emit(out, node.kind == TK_OR ? OP_JMP_IF_TRUE : OP_JMP_IF_FALSE, node.fuel, 0, 0, 1)) return -1;
      --out->stack;
    } else if (node.kind == TK_IF && frame->seen == 2) {
      frame->second_jump = out->code_count;
      if (!emit(out, OP_JMP, node.merge_fuel, 0, 0, 1)) return -1;
      out->code[frame->first_jump].a = out->code_count;
      out->stack = frame->base_stack;
    }
    if (frame->seen < node.arity) { have_value = 0; continue; }
    if (node.kind == TK_IF) {
      if (frame->args[1] != frame->args[2]) return -1;
      out->code[frame->second_jump].a = out->code_count;
    } else if (node.kind == TK_AND || node.kind == TK_OR) {
      if (completed != GAGP_TAG_BOOL) return -1;
      if (!emit(out, OP_NOT, node.fuel, 0, 0, 0) || !emit(out, OP_NOT, node.fuel, 0, 0, 0)) return -1;
      const int finish = out->code_count;
      if (!emit(out, OP_JMP, node.fuel, 0, 0, 1)) return -1;
      out->code[frame->first_jump].a = out->code_count;
      out->stack = frame->base_stack;
      Val v = {0, GAGP_TAG_BOOL, node.kind == TK_OR};
      const int index = add_const(out, v);
      if (index < 0 || !emit(out, OP_PUSH_CONST, node.fuel, index, 0, 1)) return -1;
      grow(out, 1);
      out->code[finish].a = out->code_count;
    } else {
      completed = operation_type(&node, frame->args);
      if (completed == GAGP_TAG_INVALID) {
        if (node.type == GAGP_TAG_INVALID) { out->status = ST_UNSUPPORTED; return -1; }
        completed = node.type;
      } else if (node.type != GAGP_TAG_INVALID && node.type != completed) {
        return -1;
      }
      if (node.opcode == OP_CALL_BUILTIN) {
        if (!emit(out, node.opcode, node.fuel, node.operand, node.arity, 3)) return -1;
      } else if (!emit(out, node.opcode, node.fuel, 0, 0, 0)) {
        return -1;
      }
      out->stack -= node.arity - 1;
    }
    --depth;
  }
}

/* ----------------------------------------------------------------------- VM
 * run_code_impl<SemanticFuel=false>, cpp/src/runtime/cpu/execute_bytecode_cpu.cpp:152-626,
 * with value semantics of cpp/include/gagp/core/value_semantics.hpp:33-190 and
 * builtins of cpp/src/runtime/cpu/builtins_cpu.cpp:131-218, for Int/Bool values. */
typedef struct { int error; int timeout; Val value; int64_t steps; } Exec;

static int64_t wrap_add(int64_t a, int64_t b) { return (int64_t)((uint64_t)a + (uint64_t)b); }
static int64_t wrap_sub(int64_t a, int64_t b) { return (int64_t)((uint64_t)a - (uint64_t)b); }
static int64_t wrap_mul(int64_t a, int64_t b) { return (int64_t)((uint64_t)a * (uint64_t)b); }
static int64_t wrap_neg(int64_t a) { return (int64_t)(0ULL - (uint64_t)a); }
static int64_t py_mod(int64_t a, int64_t b) {
  if (b == -1) return 0;
  int64_t r = a % b;
  if (r != 0 && ((r < 0) != (b < 0))) r += b;
  return r;
}

static Exec run_code(const Instr* code, int n, const Val* consts, int n_consts, const Val* locals, int n_locals, int fuel) {
  Exec out = {0, 0, {0, GAGP_TAG_INVALID, 0}, 0};
  Val stack[256];
  int sp = 0, ip = 0;
#define ERR() do { out.error = 1; return out; } while (0)
  while (ip < n) {
    if (fuel <= 0) { out.error = 1; out.timeout = 1; return out; }
    fuel -= 1;
    ++out.steps;
    const Instr ins = code[ip++];
    switch (ins.op) {
      case OP_PUSH_CONST:
        if (!(ins.flags & 1) || ins.a < 0 || ins.a >= n_consts || sp >= 256) ERR();
        stack[sp++] = consts[ins.a];
        break;
      case OP_LOAD:
        if (!(ins.flags & 1) || ins.a < 0 || ins.a >= n_locals || sp >= 256) ERR();
        if (locals[ins.a].tag == GAGP_TAG_INVALID) ERR();
        stack[sp++] = locals[ins.a];
        break;
      case OP_NEG: case OP_NOT: {
        if (!sp) ERR();
        const Val x = stack[--sp];
        Val r = {0, 0, 0};
        if (ins.op == OP_NEG) { if (x.tag != GAGP_TAG_INT) ERR(); r.tag = GAGP_TAG_INT; r.i = wrap_neg(x.i); }
        else { if (x.tag != GAGP_TAG_BOOL) ERR(); r.tag = GAGP_TAG_BOOL; r.b = !x.b; }
        stack[sp++] = r;
        break;
      }
      case OP_ADD: case OP_SUB: case OP_MUL: case OP_DIV: case OP_MOD: {
        if (sp < 2) ERR();
        const Val b = stack[--sp], a = stack[--sp];
        if (a.tag != GAGP_TAG_INT || b.tag != GAGP_TAG_INT) ERR();
        if ((ins.op == OP_DIV || ins.op == OP_MOD) && b.i == 0) ERR();
        if (ins.op == OP_DIV) ERR();  /* Float result: outside the resident subset */
        Val r = {0, GAGP_TAG_INT, 0};
        r.i = ins.op == OP_ADD ? wrap_add(a.i, b.i) : ins.op == OP_SUB ? wrap_sub(a.i, b.i)
            : ins.op == OP_MUL ? wrap_mul(a.i, b.i) : py_mod(a.i, b.i);
        stack[sp++] = r;
        break;
      }
      case OP_LT: case OP_LE: case OP_GT: case OP_GE: case OP_EQ: case OP_NE: {
        if (sp < 2) ERR();
        const Val b = stack[--sp], a = stack[--sp];
        Val r = {0, GAGP_TAG_BOOL, 0};
        if (ins.op == OP_EQ || ins.op == OP_NE) {
          if (a.tag != b.tag) ERR();
          int eq;
          if (a.tag == GAGP_TAG_BOOL) eq = a.b == b.b;
          else if (a.tag == GAGP_TAG_INT) eq = a.i == b.i;
          else ERR();
          r.b = ins.op == OP_EQ ? eq : !eq;
        } else {
          if (a.tag != GAGP_TAG_INT || b.tag != GAGP_TAG_INT) ERR();
          r.b = ins.op == OP_LT ? a.i < b.i : ins.op == OP_LE ? a.i <= b.i : ins.op == OP_GT ? a.i > b.i : a.i >= b.i;
        }
        stack[sp++] = r;
        break;
      }
      case OP_JMP:
        if (!(ins.flags & 1) || ins.a < 0 || ins.a > n) ERR();
        ip = ins.a;
        break;
      case OP_JMP_IF_FALSE: case OP_JMP_IF_TRUE: {
        if (!sp) ERR();
        if (!(ins.flags & 1) || ins.a < 0 || ins.a > n) ERR();
        const Val c = stack[--sp];
        if (c.tag != GAGP_TAG_BOOL) ERR();
        if (ins.op == OP_JMP_IF_FALSE && !c.b) ip = ins.a;
        if (ins.op == OP_JMP_IF_TRUE && c.b) ip = ins.a;
        break;
      }
      case OP_CALL_BUILTIN: {
        const int argc = (ins.flags & 2) ? ins.b : -1;
        if (argc < 0 || sp < argc) ERR();
        const Val* args = stack + sp - argc;
        Val r = {0, GAGP_TAG_INT, 0};
        switch (ins.a) {
          case B_ABS:
            if (argc != 1 || args[0].tag != GAGP_TAG_INT) ERR();
            r.i = args[0].i < 0 ? wrap_neg(args[0].i) : args[0].i;
            break;
          case B_MIN: case B_MAX:
            if (argc != 2 || args[0].tag != GAGP_TAG_INT || args[1].tag != GAGP_TAG_INT) ERR();
            r.i = ins.a == B_MIN ? (args[0].i < args[1].i ? args[0].i : args[1].i)
                                 : (args[0].i > args[1].i ? args[0].i : args[1].i);
            break;
          case B_IDIV0: case B_IMOD0: case B_TRUNC_DIV0: case B_TRUNC_MOD0: {
            if (argc != 2 || args[0].tag != GAGP_TAG_INT || args[1].tag != GAGP_TAG_INT) ERR();
            const int64_t a = args[0].i, b = args[1].i;
            if (b == 0) r.i = 0;
            else if (ins.a == B_TRUNC_DIV0) r.i = (a == INT64_MIN && b == -1) ? 0 : a / b;
            else if (ins.a == B_TRUNC_MOD0) r.i = (a == INT64_MIN && b == -1) ? 0 : a % b;
            else if (ins.a == B_IDIV0) r.i = b == -1 ? wrap_neg(a) : a / b;
            else r.i = py_mod(a, b);
            break;
          }
          default: ERR();
        }
        sp -= argc;
        stack[sp++] = r;
        break;
      }
      case OP_RETURN:
        if (!sp) ERR();
        out.value = stack[sp - 1];
        return out;
      default: ERR();
    }
  }
#undef ERR
  out.error = 1;  /* program finished without return */
  return out;
}

/* ------------------------------------------------------------------ fitness
 * fitness_case_score (cpp/include/gagp/core/fitness_policy.hpp:28-58) and the
 * ordered reduction of eval_fitness_cpu (cpp/src/runtime/cpu/fitness_cpu.cpp:44-176). */
static double canonical_acc(double value) {
  if (!isfinite(value) || value == 0.0) return value == 0.0 ? 0.0 : value;
  int exponent = 0;
  const double mantissa = frexp(value, &exponent);
  const long long q = llround(ldexp(mantissa, 48));
  return ldexp((double)q, exponent - 48);
}
static double canonical_rank(double value) {
  if (!isfinite(value) || value == 0.0) return value == 0.0 ? 0.0 : value;
  int exponent = 0;
  const double mantissa = frexp(value, &exponent);
  const long long q = llround(ldexp(mantissa, 40));
  return ldexp((double)q, exponent - 40);
}
static double error_ceiling(int metric, double penalty) { return metric == GAGP_METRIC_EXACT ? 1.0 : fabs(penalty); }
static double case_score(const Val* actual, const Val* expected, double penalty, int metric) {
  const int numeric = (actual->tag == GAGP_TAG_INT || actual->tag == GAGP_TAG_FLOAT) &&
                      (expected->tag == GAGP_TAG_INT || expected->tag == GAGP_TAG_FLOAT);
  if (metric == GAGP_METRIC_EXACT) {
    if (actual->tag == GAGP_TAG_INT && expected->tag == GAGP_TAG_INT) return actual->i == expected->i ? 0.0 : -1.0;
    if (actual->tag != expected->tag || actual->tag == GAGP_TAG_INVALID) return -1.0;
    return (actual->tag == GAGP_TAG_BOOL ? actual->b == expected->b : actual->i == expected->i) ? 0.0 : -1.0;
  }
  if (!numeric) return -error_ceiling(metric, penalty);
  double error;
  if (actual->tag == GAGP_TAG_INT && expected->tag == GAGP_TAG_INT) {
    const int64_t a = actual->i, b = expected->i;
    error = (double)(a >= b ? (uint64_t)a - (uint64_t)b : (uint64_t)b - (uint64_t)a);
  } else {
    return -error_ceiling(metric, penalty);
  }
  return -fmin(error, fabs(penalty));
}
static int exact_match(const Val* actual, const Val* expected) {
  if (actual->tag == GAGP_TAG_INT && expected->tag == GAGP_TAG_INT) return actual->i == expected->i;
  if (actual->tag != expected->tag || actual->tag == GAGP_TAG_INVALID) return 0;
  return actual->tag == GAGP_TAG_BOOL ? actual->b == expected->b : actual->i == expected->i;
}

typedef struct {
  const gagp_cases* cases;
  Val* locals;    /* case-major input values */
  Val* expected;
  int fuel, metric, lanes;
  double penalty;
} CaseSet;

static double evaluate_program(const Instr* code, int n, const Val* consts, int n_consts, int n_locals,
                               const CaseSet* cs, unsigned* wrong_out, uint64_t* steps) {
  const int C = cs->cases->case_count, L = cs->lanes;
  double partial_buffer[2048];
  double* partial = L <= 2048 ? partial_buffer : malloc(sizeof(double) * (size_t)L);
  unsigned wrong = 0;
  for (int lane = 0; lane < L; ++lane) {
    const size_t begin = ((size_t)C * (size_t)lane) / (size_t)L, end = ((size_t)C * (size_t)(lane + 1)) / (size_t)L;
    double local = 0.0;
    for (size_t c = begin; c < end; ++c) {
      const Exec e = run_code(code, n, consts, n_consts, cs->locals + c * (size_t)n_locals, n_locals, cs->fuel);
      if (steps) *steps += (uint64_t)e.steps;
      if (e.error) {
        ++wrong;
        local = canonical_acc(local - error_ceiling(cs->metric, cs->penalty));
        continue;
      }
      local = canonical_acc(local + case_score(&e.value, &cs->expected[c], cs->penalty, cs->metric));
      if (!exact_match(&e.value, &cs->expected[c])) ++wrong;
    }
    partial[lane] = local;
  }
  double score = 0.0;
  if (cs->metric == GAGP_METRIC_LEGACY) {
    for (int i = 0; i < L; ++i) score = canonical_acc(score + partial[i]);
  } else {
    for (int base = 0; base < L; base += 32) {
      double warp = 0;
      for (int i = base; i < base + 32 && i < L; ++i) warp = canonical_acc(warp + partial[i]);
      score = canonical_acc(score + warp);
    }
  }
  if (partial != partial_buffer) free(partial);
  *wrong_out = wrong;
  return score;
}

/* Lowers and scores one row; -1 when the phase compiler rejects it. */
static int score_row(const Slot* slot, const gagp_grammar* g, const View* t, const CaseSet* cs,
                     double* fitness, unsigned* wrong, uint64_t* steps) {
  static Instr code[4 * CAPACITY + 1];
  static Val consts[CAPACITY + 8];
  Emit out = {code, consts, 4 * CAPACITY, CAPACITY, ST_INVALID, 0, 0, 0, 0};
  if (compile_row(t->nodes, t->node_count, t->constants, t->constant_count, g->local_types, g->local_count,
                  slot->type, &out) != 0 || out.status != ST_OK || out.stack_bound < 1)
    return -1;
  if (out.code_count >= 4 * CAPACITY + 1) return -1;
  Instr ret = {OP_RETURN, 0, 0, 0, g->return_fuel};
  code[out.code_count] = ret;
  *fitness = evaluate_program(code, out.code_count + 1, consts, out.const_count, g->local_count, cs, wrong, steps);
  return 0;
}

/* ----------------------------------------------------------------- set-up */
typedef struct {
  const gagp_grammar* g;
  Slot slot;
  Node* expr_node;
  int maxv;   /* max variable nodes */
} Search;

static int search_init(Search* s, const gagp_grammar* g) {
  memset(s, 0, sizeof *s);
  s->g = g;
  if (g->expression_count <= 0 || g->root_expression < 0 || g->root_expression >= g->expression_count)
    FAIL("invalid grammar tables");
  s->expr_node = malloc(sizeof(Node) * (size_t)g->expression_count);
  if (!s->expr_node) FAIL("out of memory");
  for (int i = 0; i < g->expression_count; ++i) s->expr_node[i] = expression_node(&g->expressions[i]);
  s->slot.G.g = g;
  s->slot.G.expr_node = s->expr_node;
  s->slot.root = g->root_expression;
  s->slot.scope = 0;
  s->slot.max_depth = g->slot_max_depth;
  s->slot.logical_depth = g->site_depth;
  s->slot.type = g->slot_type;
  s->maxv = g->max_nodes - g->fixed_nodes;
  if (s->maxv <= 0 || s->maxv > CAPACITY) FAIL("node budget");
  return 0;
}

static int case_set_init(CaseSet* cs, const gagp_cases* cases, const gagp_grammar* g, const gagp_search_config* cfg) {
  cs->cases = cases;
  cs->fuel = cfg->fuel;
  cs->metric = cfg->metric;
  cs->penalty = cfg->penalty;
  cs->lanes = cfg->reduction_lanes > 0 ? cfg->reduction_lanes : 1;
  if (cases->input_count != g->local_count) FAIL("case inputs must cover the grammar inputs");
  cs->locals = malloc(sizeof(Val) * (size_t)cases->case_count * (size_t)(cases->input_count ? cases->input_count : 1));
  cs->expected = malloc(sizeof(Val) * (size_t)cases->case_count);
  if (!cs->locals || !cs->expected) FAIL("out of memory");
  for (int c = 0; c < cases->case_count; ++c) {
    for (int j = 0; j < cases->input_count; ++j) {
      Val v = {0, cases->input_tags[j], 0};
      const int64_t x = cases->inputs[(size_t)c * cases->input_count + j];
      if (v.tag == GAGP_TAG_BOOL) v.b = x != 0; else v.i = x;
      cs->locals[(size_t)c * cases->input_count + j] = v;
    }
    Val e = {0, cases->expected_tag, 0};
    if (e.tag == GAGP_TAG_BOOL) e.b = cases->expected[c] != 0; else e.i = cases->expected[c];
    cs->expected[c] = e;
  }
  return 0;
}
static void case_set_free(CaseSet* cs) { free(cs->locals); free(cs->expected); }

/* SplitMix64 finaliser used to derive initial-phase seeds (phase_population_cpu.cpp:77-78). */
static uint64_t mix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

/* generate_phase_initial_population for a one-phase whole program
 * (phase_population_cpu.cpp:54-113); the rows carry generated sites, which
 * equal the import-time annotation of the same nodes. */
static int initial_rows(const Search* s, int population, uint64_t seed, int site_limit, Trees* rows) {
  const gagp_grammar* g = s->g;
  if (population <= 0 || population > 16384 || site_limit < 1 || site_limit > 15)
    FAIL("initial population size/site depth");
  const int available = s->maxv;
  for (int i = 0; i < population; ++i) {
    const int ramp = site_limit < 2 ? site_limit : 2 + i % (site_limit - 1);
    Gen generated = {ST_INVALID, 0, 0, 0};
    Out o = out_of(rows, i);
    for (int logical = ramp, attempt = 0; generated.status != ST_OK; ++attempt) {
      const long room = available < CAPACITY ? available : CAPACITY;
      if (room <= 0) FAIL("initial phase budget");
      generated = generate_phase(&s->slot.G, g->root_expression, 0, g->slot_max_depth, (int)room,
                                 mix64(seed ^ mix64(((uint64_t)i * 8 + 0) * 64 + (uint64_t)attempt)),
                                 o.nodes, o.origins, o.constants, o.sites, logical);
      /* a statement program that reads an unassigned local is retried
       * (phase_population_cpu.cpp:95-96) */
      if (generated.status == ST_OK && g->slot_type == STATEMENT_TAG && !locals_defined(o.nodes, generated.nodes))
        generated.status = ST_INVALID;
      if (generated.status != ST_OK && attempt % 4 == 3 && logical < site_limit) ++logical;
      if (attempt >= 256) FAIL("initial phase generation failed");
    }
    rows->lengths[i] = generated;
  }
  return 0;
}

/* Rebuilds nodes and sites of transport rows (origins + constants) by
 * replaying the construction records (annotate_phase_tree,
 * device/phase_variation.cuh:23-79). */
static int import_row(const Search* s, const int32_t* origins, int n, const int64_t* constants, int nc, Trees* t, int row) {
  const gagp_grammar* g = s->g;
  if (n <= 0 || n > s->maxv || nc < 0 || nc > n) FAIL("imported phase capacity");
  Out o = out_of(t, row);
  int k = 0;
  for (int i = 0; i < n; ++i) {
    if (origins[i] < 0 || origins[i] >= g->expression_count) FAIL("missing expression origin");
    Node node = s->expr_node[origins[i]];
    if (g->expressions[origins[i]].kind == EK_CONSTANT) {
      if (k >= nc) FAIL("constant count");
      node.operand = k;
      o.constants[k].tag = GAGP_TAG_INT; o.constants[k].i = constants[k]; o.constants[k].b = 0;
      ++k;
    }
    o.nodes[i] = node;
    o.origins[i] = origins[i];
  }
  if (k != nc) FAIL("constant count");
  /* annotate */
  struct { int expression; Site site; } pending[192];
  int count = 1, cursor = 0, steps = 0;
  pending[0].expression = g->root_expression;
  pending[0].site.nonterminal = -1; pending[0].site.entry_expression = -1;
  pending[0].site.parent_scope = 0; pending[0].site.scope = 0;
  while (count) {
    if (++steps > 8192 || cursor >= n) FAIL("import site annotation failed");
    const int e_id = pending[count - 1].expression;
    const Site site = pending[count - 1].site;
    --count;
    const gagp_expression* e = &g->expressions[e_id];
    if (e->kind == EK_REFERENCE) {
      const gagp_nonterminal* nt = &g->nonterminals[e->target];
      int production = -1;
      for (int i = 0; i < nt->production_count && production < 0; ++i) {
        int x = g->productions[nt->production_offset + i].expression;
        for (int hop = 0; hop < 64 && x >= 0 && g->expressions[x].kind == EK_ALIAS; ++hop) x = g->expressions[x].children[0];
        if (x == origins[cursor]) production = g->productions[nt->production_offset + i].expression;
      }
      if (production < 0 || site.nonterminal >= 0 || count >= 192) FAIL("import site annotation failed");
      pending[count].expression = production;
      pending[count].site.nonterminal = e->target;
      pending[count].site.entry_expression = e_id;
      pending[count].site.parent_scope = 0;
      pending[count].site.scope = e->scope_count | (nt->fixed ? FIXED_SITE : 0);
      ++count;
      continue;
    }
    if (origins[cursor] != e_id) FAIL("import site annotation failed");
    o.sites[cursor++] = site;
    for (int i = e->arity - 1; i >= 0; --i) {
      if (count >= 192) FAIL("import site annotation failed");
      pending[count].expression = e->children[i];
      pending[count].site.nonterminal = -1; pending[count].site.entry_expression = -1;
      pending[count].site.parent_scope = 0; pending[count].site.scope = 0;
      ++count;
    }
  }
  if (cursor != n) FAIL("import site annotation failed");
  Gen r = {ST_OK, n, nc, 0};
  t->lengths[row] = r;
  if (g->site_depth && site_depth(o.nodes, o.sites, n, -1) > g->site_depth) FAIL("import site depth");
  return 0;
}

static void export_row(const Trees* t, int row, const gagp_rows* out, int index) {
  const View v = view_of(t, row);
  out->node_counts[index] = v.node_count;
  out->constant_counts[index] = v.constant_count;
  for (int i = 0; i < v.node_count && i < out->stride; ++i) out->origins[(size_t)index * out->stride + i] = v.origins[i];
  for (int i = 0; i < v.constant_count && i < out->stride; ++i) out->constants[(size_t)index * out->stride + i] = v.constants[i].i;
}

static unsigned row_nodes(const Search* s, const Trees* t, int row, int grammar_sites) {
  const View v = view_of(t, row);
  if (!grammar_sites) return (unsigned)(s->g->fixed_nodes + v.node_count);
  unsigned count = 0;
  for (int j = 0; j < v.node_count; ++j) count += v.sites[j].nonterminal >= 0;
  return count;
}

/* ---------------------------------------------------------- steady state
 * run_phase_population_steady, cpp/src/evolution/evolve.cpp:331-441 */
typedef struct {
  const double* fitness; const unsigned* wrong; const unsigned* nodes; int has_wrong;
} Rank;
static const Rank* g_rank;
static int better(const Rank* r, int a, int b) {
  if (r->fitness[a] != r->fitness[b]) return r->fitness[a] > r->fitness[b];
  if (r->has_wrong) {
    if (r->wrong[a] != r->wrong[b]) return r->wrong[a] < r->wrong[b];
    if (r->nodes[a] != r->nodes[b]) return r->nodes[a] < r->nodes[b];
  }
  return a < b;
}
static int order_cmp(const void* x, const void* y) {
  const int a = *(const int*)x, b = *(const int*)y;
  if (a == b) return 0;
  return better(g_rank, a, b) ? -1 : 1;
}

int gagp_oracle_search(const gagp_grammar* g, const gagp_cases* cases, const gagp_search_config* cfg,
                       const gagp_rows* initial, gagp_search_result* out) {
  return gagp_oracle_search_reuse(g, cases, cfg, initial, out, 0);
}

int gagp_oracle_search_reuse(const gagp_grammar* g, const gagp_cases* cases, const gagp_search_config* cfg,
                             const gagp_rows* initial, gagp_search_result* out, int member_reuse) {
  Search s;
  if (search_init(&s, g) != 0) return -1;
  CaseSet cs;
  if (case_set_init(&cs, cases, g, cfg) != 0) { free(s.expr_node); return -1; }
  const int P = cfg->population, B = cfg->batch > 0 ? cfg->batch : cfg->population;
  int rc = -1;
  if (!cfg->steady_state) { snprintf(g_error, sizeof g_error, "only the steady-state schedule is restated"); goto done0; }
  if (P <= 0 || B <= 0 || B > P || P % B || cfg->generations <= 0 || cfg->replacement_size < 1) {
    snprintf(g_error, sizeof g_error, "steady-state batch contract"); goto done0;
  }
  const int cap = s.maxv;
  Trees current, crossed, next, scratch;
  memset(&current, 0, sizeof current); memset(&crossed, 0, sizeof crossed);
  memset(&next, 0, sizeof next); memset(&scratch, 0, sizeof scratch);
  if (trees_alloc(&current, P, cap) || trees_alloc(&crossed, P, cap) || trees_alloc(&next, P, cap) ||
      trees_alloc(&scratch, P, cap)) { snprintf(g_error, sizeof g_error, "out of memory"); goto done1; }
  if (initial) {
    if (initial->count != P) { snprintf(g_error, sizeof g_error, "initial population size"); goto done1; }
    for (int p = 0; p < P; ++p)
      if (import_row(&s, initial->origins + (size_t)p * initial->stride, initial->node_counts[p],
                     initial->constants + (size_t)p * initial->stride, initial->constant_counts[p], &current, p))
        goto done1;
  } else if (initial_rows(&s, P, cfg->seed, g->site_depth, &current)) {
    goto done1;
  }
  const int pressure = cfg->tournament_size < 1 ? 1 : cfg->tournament_size > P ? P : cfg->tournament_size;
  const int has_wrong = cfg->metric != GAGP_METRIC_LEGACY;
  double* fitness = calloc((size_t)P, sizeof(double));
  double* selection = calloc((size_t)P, sizeof(double));
  unsigned* wrong = calloc((size_t)P, sizeof(unsigned));
  unsigned* nodes = calloc((size_t)P, sizeof(unsigned));
  int* order = calloc((size_t)P, sizeof(int));
  int* placed = calloc((size_t)P, sizeof(int));
  int* reuse = calloc((size_t)B, sizeof(int));
  double* child_fitness = calloc((size_t)B, sizeof(double));
  unsigned* child_wrong = calloc((size_t)B, sizeof(unsigned));
  unsigned* child_count = calloc((size_t)B, sizeof(unsigned));
  Stat* stats = calloc((size_t)B, sizeof(Stat));
  uint64_t* member_hash = calloc((size_t)P, sizeof(uint64_t));
  if (!fitness || !selection || !wrong || !nodes || !order || !placed || !reuse || !child_fitness || !child_wrong ||
      !child_count || !stats || !member_hash) { snprintf(g_error, sizeof g_error, "out of memory"); goto done2; }
  Policy policy = {cfg->counted_sites, cfg->uniform_phase, cfg->crossover_probability, cfg->crossover_attempts,
                   cfg->mutation_max_nodes};
  Mt rng;
  mt_seed(&rng, cfg->seed);
  out->evaluated_programs = out->reused_programs = out->program_cases = 0;
  /* Initial evaluation (HostPhasePopulation::evaluate, phase_population_cpu.cpp:243-267). */
  for (int i = 0; i < P; ++i) {
    const View v = view_of(&current, i);
    unsigned w = 0;
    double f = 0;
    if (score_row(&s.slot, g, &v, &cs, &f, &w, NULL)) { snprintf(g_error, sizeof g_error, "phase compiler rejected a member"); goto done2; }
    fitness[i] = canonical_rank(f);
    wrong[i] = has_wrong ? w : 0;
    nodes[i] = has_wrong ? row_nodes(&s, &current, i, cfg->grammar_site_ranking) : 0;
    out->evaluated_programs++;
    out->program_cases += (uint64_t)cases->case_count;
  }
  Rank rank = {fitness, wrong, nodes, has_wrong};
  g_rank = &rank;
  for (int i = 0; i < P; ++i) order[i] = i;
  qsort(order, (size_t)P, sizeof(int), order_cmp);
  for (int i = 0; i < P; ++i) selection[i] = fitness[i];
  if (has_wrong) for (int r = 0; r < P; ++r) selection[order[r]] = (double)(P - r);
  int best = order[0];
  const uint64_t rounds = (uint64_t)P * (uint64_t)cfg->generations / (uint64_t)B;
  const uint64_t per_epoch = (uint64_t)(P / B);
  int recorded = 0;
#define RECORD() do { \
    const int b0 = order[0]; \
    if (recorded < out->generations) { \
      out->history_best_fitness[recorded] = fitness[b0]; \
      long double sum = 0; \
      for (int m = 0; m < P; ++m) sum += fitness[m]; \
      out->history_mean_fitness[recorded] = (double)(sum / P); \
      out->history_best_wrong[recorded] = has_wrong ? (int)wrong[b0] : -1; \
      out->history_best_nodes[recorded] = (int)row_nodes(&s, &current, b0, 0); \
      export_row(&current, b0, &out->history_best, recorded); \
    } \
    ++recorded; \
  } while (0)
  for (uint64_t round = 0; round < rounds; ++round) {
    if (round % per_epoch == 0) RECORD();
    const uint64_t seed = mt_next(&rng);
    /* make_batch (phase_population_cpu.cpp:322-353) */
    for (int child = 0; child < B; ++child) {
      crossover_child(child, &current, &crossed, &s.slot, 1, P, s.maxv, selection, pressure, seed, &policy, &stats[child]);
      mutate_child(child, &crossed, &next, &scratch, &s.slot, 1, s.maxv, cfg->mutation_probability, seed, &policy, &stats[child]);
      compare_child(child, &current, &crossed, P, 1, &stats[child]);
    }
    if (member_reuse)
      for (int m = 0; m < P; ++m) { const View v = view_of(&current, m); member_hash[m] = row_hash(&v); }
    for (int child = 0; child < B; ++child) {
      if (stats[child].error) { snprintf(g_error, sizeof g_error, "CPU genotype variation error %d", stats[child].error); goto done2; }
      reuse[child] = stats[child].reusable_parent;
      if (member_reuse && reuse[child] < 0) reuse[child] = find_member(&current, member_hash, P, &crossed, child);
    }
    /* evaluate_batch + results of all children first (evolve.cpp:403-413) */
    for (int b = 0; b < B; ++b) {
      const int source = reuse[b];
      if (source >= 0) {
        out->reused_programs++;
        child_fitness[b] = fitness[source];
        child_wrong[b] = has_wrong ? wrong[source] : 0;
        child_count[b] = has_wrong ? nodes[source] : 0;
        continue;
      }
      const View v = view_of(&crossed, b);
      unsigned w = 0;
      double f = 0;
      if (score_row(&s.slot, g, &v, &cs, &f, &w, NULL)) { snprintf(g_error, sizeof g_error, "phase compiler rejected a child"); goto done2; }
      out->evaluated_programs++;
      out->program_cases += (uint64_t)cases->case_count;
      child_fitness[b] = canonical_rank(f);
      child_wrong[b] = has_wrong ? w : 0;
      child_count[b] = has_wrong ? row_nodes(&s, &crossed, b, cfg->grammar_site_ranking) : 0;
    }
    /* placement (evolve.cpp:414-427) */
    for (int m = 0; m < P; ++m) placed[m] = -1;
    for (int b = 0; b < B; ++b) {
      int v;
      for (;;) {
        int worst = (int)(mt_next(&rng) % (uint64_t)P);
        for (int i = 1; i < cfg->replacement_size; ++i) {
          const int c = (int)(mt_next(&rng) % (uint64_t)P);
          if (better(&rank, worst, c)) worst = c;
        }
        if (worst != best) { v = worst; break; }
      }
      fitness[v] = child_fitness[b];
      if (has_wrong) wrong[v] = child_wrong[b];
      nodes[v] = child_count[b];
      placed[v] = b;
      if (!has_wrong) selection[v] = fitness[v];
      if (better(&rank, v, best)) best = v;
    }
    qsort(order, (size_t)P, sizeof(int), order_cmp);
    if (order[0] != best) { snprintf(g_error, sizeof g_error, "steady-state best tracking"); goto done2; }
    if (has_wrong) for (int r = 0; r < P; ++r) selection[order[r]] = (double)(P - r);
    /* commit_batch (phase_population_cpu.cpp:382-394) */
    for (int m = 0; m < P; ++m)
      if (placed[m] >= 0) copy_tree(&crossed, placed[m], &current, m);
  }
  if (recorded < cfg->generations) RECORD();
#undef RECORD
  out->generations = recorded < out->generations ? recorded : out->generations;
  for (int r = 0; r < P && r < out->population; ++r) {
    const int m = order[r];
    out->final_fitness[r] = fitness[m];
    out->final_wrong[r] = has_wrong ? (int)wrong[m] : -1;
    out->final_nodes[r] = (int)row_nodes(&s, &current, m, 0);
    export_row(&current, m, &out->final_rows, r);
  }
  rc = 0;
done2:
  free(fitness); free(selection); free(wrong); free(nodes); free(order); free(placed); free(reuse);
  free(child_fitness); free(child_wrong); free(child_count); free(stats); free(member_hash);
done1:
  trees_free(&current); trees_free(&crossed); trees_free(&next); trees_free(&scratch);
done0:
  case_set_free(&cs);
  free(s.expr_node);
  return rc;
}

int gagp_oracle_initial_population(const gagp_grammar* g, const gagp_search_config* cfg, gagp_rows* out) {
  Search s;
  if (search_init(&s, g) != 0) return -1;
  Trees rows;
  memset(&rows, 0, sizeof rows);
  int rc = -1;
  if (trees_alloc(&rows, cfg->population, s.maxv) == 0 && initial_rows(&s, cfg->population, cfg->seed, g->site_depth, &rows) == 0) {
    for (int i = 0; i < cfg->population && i < out->count; ++i) export_row(&rows, i, out, i);
    rc = 0;
  }
  trees_free(&rows);
  free(s.expr_node);
  return rc;
}

/* One make_batch (phase_population_cpu.cpp:322-353) over the generated
 * initial population: every child of the first `batch` (cfg->batch, or the
 * population) is varied with the given selection fitness and round seed;
 * the children's rows go to `children` and the members whose results they
 * reuse (their parent when unchanged, else an identical member; -1: none)
 * to `reuse`.  Variation needs no cases, so this also runs on tables whose
 * programs the oracle cannot evaluate. */
int gagp_oracle_make_batch(const gagp_grammar* g, const gagp_search_config* cfg, const double* selection,
                           uint64_t seed, gagp_rows* children, int32_t* reuse) {
  Search s;
  if (search_init(&s, g) != 0) return -1;
  const int P = cfg->population, B = cfg->batch > 0 ? cfg->batch : cfg->population;
  int rc = -1;
  Trees current, crossed, next, scratch;
  memset(&current, 0, sizeof current); memset(&crossed, 0, sizeof crossed);
  memset(&next, 0, sizeof next); memset(&scratch, 0, sizeof scratch);
  Stat* stats = calloc((size_t)(B > 0 ? B : 1), sizeof(Stat));
  if (P <= 0 || B <= 0 || B > P || !stats) { snprintf(g_error, sizeof g_error, "batch contract"); goto done; }
  if (trees_alloc(&current, P, s.maxv) || trees_alloc(&crossed, P, s.maxv) || trees_alloc(&next, P, s.maxv) ||
      trees_alloc(&scratch, P, s.maxv)) { snprintf(g_error, sizeof g_error, "out of memory"); goto done; }
  if (initial_rows(&s, P, cfg->seed, g->site_depth, &current)) goto done;
  {
    const int pressure = cfg->tournament_size < 1 ? 1 : cfg->tournament_size > P ? P : cfg->tournament_size;
    Policy policy = {cfg->counted_sites, cfg->uniform_phase, cfg->crossover_probability, cfg->crossover_attempts,
                     cfg->mutation_max_nodes};
    for (int child = 0; child < B; ++child) {
      crossover_child(child, &current, &crossed, &s.slot, 1, P, s.maxv, selection, pressure, seed, &policy, &stats[child]);
      mutate_child(child, &crossed, &next, &scratch, &s.slot, 1, s.maxv, cfg->mutation_probability, seed, &policy,
                   &stats[child]);
      compare_child(child, &current, &crossed, P, 1, &stats[child]);
    }
    uint64_t* member_hash = calloc((size_t)P, sizeof(uint64_t));
    if (!member_hash) { snprintf(g_error, sizeof g_error, "out of memory"); goto done; }
    for (int m = 0; m < P; ++m) { const View v = view_of(&current, m); member_hash[m] = row_hash(&v); }
    for (int child = 0; child < B; ++child) {
      if (stats[child].error) {
        snprintf(g_error, sizeof g_error, "CPU genotype variation error %d", stats[child].error);
        free(member_hash);
        goto done;
      }
      reuse[child] = stats[child].reusable_parent;
      if (reuse[child] < 0) reuse[child] = find_member(&current, member_hash, P, &crossed, child);
      if (child < children->count) export_row(&crossed, child, children, child);
    }
    free(member_hash);
  }
  rc = 0;
done:
  trees_free(&current); trees_free(&crossed); trees_free(&next); trees_free(&scratch);
  free(stats);
  free(s.expr_node);
  return rc;
}

int gagp_oracle_evaluate(const gagp_grammar* g, const gagp_cases* cases, const gagp_search_config* cfg,
                         const gagp_rows* rows, double* fitness, uint32_t* wrong, uint64_t* instructions) {
  Search s;
  if (search_init(&s, g) != 0) return -1;
  CaseSet cs;
  if (case_set_init(&cs, cases, g, cfg) != 0) { free(s.expr_node); return -1; }
  Trees t;
  memset(&t, 0, sizeof t);
  int rc = -1;
  if (trees_alloc(&t, 1, s.maxv) != 0) goto done;
  if (instructions) *instructions = 0;
  for (int r = 0; r < rows->count; ++r) {
    if (import_row(&s, rows->origins + (size_t)r * rows->stride, rows->node_counts[r],
                   rows->constants + (size_t)r * rows->stride, rows->constant_counts[r], &t, 0))
      goto done;
    const View v = view_of(&t, 0);
    unsigned w = 0;
    double f = 0;
    if (score_row(&s.slot, g, &v, &cs, &f, &w, instructions)) { snprintf(g_error, sizeof g_error, "phase compiler rejected a row"); goto done; }
    fitness[r] = f;
    wrong[r] = w;
  }
  rc = 0;
done:
  trees_free(&t);
  case_set_free(&cs);
  free(s.expr_node);
  return rc;
}

int gagp_oracle_compile(const gagp_grammar* g, const int32_t* origins, int32_t node_count, const int64_t* constants,
                        int32_t constant_count, int32_t* code, int32_t code_capacity, int64_t* out_constants,
                        int32_t* out_constant_count, int32_t* stack_bound) {
  Search s;
  if (search_init(&s, g) != 0) return -1;
  Trees t;
  memset(&t, 0, sizeof t);
  int rc = -1;
  static Instr buffer[4 * CAPACITY];
  static Val cbuf[CAPACITY];
  if (trees_alloc(&t, 1, s.maxv) != 0) goto done;
  if (import_row(&s, origins, node_count, constants, constant_count, &t, 0)) goto done;
  {
    Emit o = {buffer, cbuf, 4 * CAPACITY, CAPACITY, ST_INVALID, 0, 0, 0, 0};
    const View v = view_of(&t, 0);
    if (compile_row(v.nodes, v.node_count, v.constants, v.constant_count, g->local_types, g->local_count, s.slot.type, &o) ||
        o.status != ST_OK) { snprintf(g_error, sizeof g_error, "phase compiler rejected the row"); goto done; }
    if (o.code_count > code_capacity) { snprintf(g_error, sizeof g_error, "code capacity"); goto done; }
    for (int i = 0; i < o.code_count; ++i) {
      code[i * 5 + 0] = buffer[i].op; code[i * 5 + 1] = buffer[i].flags; code[i * 5 + 2] = buffer[i].a;
      code[i * 5 + 3] = buffer[i].b; code[i * 5 + 4] = (int32_t)buffer[i].fuel;
    }
    for (int i = 0; i < o.const_count; ++i) out_constants[i] = cbuf[i].tag == GAGP_TAG_BOOL ? cbuf[i].b : cbuf[i].i;
    *out_constant_count = o.const_count;
    *stack_bound = o.stack_bound;
    rc = o.code_count;
  }
done:
  trees_free(&t);
  free(s.expr_node);
  return rc;
}
