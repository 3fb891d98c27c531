// Test harness: the reference-side binding of gagp_b200, compiled against the
// reference's own sources (oracle/Makefile, target `boundary`) and linked with
// the reference's CPU engine and libgagp_b200.so.  It is the adapter a
// maintainer adds to the reference: the engine's
// tables come from the reference's own phase compiler, the search runs through
// the C ABI, and the result comes back through the reference's own phase-row
// export.  `main` runs one task both through this adapter and through the
// reference's CPU engine (evolve_population) and prints the comparison as JSON.
//
//   reference_adapter TASK.json SEARCH.json
#define __device__
#define __host__
#include <algorithm>
#include <cinttypes>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "gagp/cli/json.hpp"
#include "gagp/cli/program_json.hpp"
#include "gagp/cli/search_config.hpp"
#include "gagp/cli/task.hpp"
#include "gagp/evolution/case_set.hpp"
#include "gagp/evolution/evolve.hpp"
#include "gagp/evolution/grammar/definition.hpp"
#include "gagp/evolution/grammar/request.hpp"
#include "gagp/runtime/payload/payload.hpp"
#include "repro/gpu/phase_layout.hpp"
#include "repro/gpu/phase_population_cpu.hpp"
#include "repro/gpu/phase_variation.hpp"

#include "gagp_b200.h"

using namespace gagp;
namespace gg = gagp::evo::grammar;
namespace rp = gagp::evo::repro;

namespace gagp::evo {

// ------------------------------------------------------------------ adapter
// Runs the resident steady-state search of `cfg` on gagp_b200.  Returns false
// when the engine declines the search (the caller then keeps its own path, as
// the reference does after a resident decline, evolve.cpp:45-49); throws on a
// hard failure.
bool evolve_b200_phase_population(gagp_engine* engine, const EvolutionConfig& cfg, const std::vector<EvalCase>& cases,
                                  EvolutionResult& result, std::string* declined) {
  const auto& grammar = *cfg.compiled_grammar;
  const CaseSet case_set = prepare_case_set(cases);
  const auto& names = case_set.input_names;
  const int site_depth = cfg.gpu_phase_site_depth;
  // the layout of a whole-program phase, as the resident owner admits it
  // (phase_population_cpu.cpp:176-219): one generated prototype, its slot and
  // the slot's phase tables with statically normalised weights
  const auto prototype = rp::generate_phase_initial_population(grammar, *cfg.generation_request, names, 1, cfg.seed,
                                                                site_depth);
  rp::NativePhaseGrammarProfiles profiles(cfg.compiled_grammar, names);
  auto layout = rp::import_native_phase_layout(grammar, prototype.front(), &profiles, &names, true);
  if (!layout.whole_program || layout.slots.size() != 1) {
    *declined = "gagp_b200 runs one whole-program phase";
    return false;
  }
  layout.profiles[0] = rp::compile_phase_variation_grammar(grammar, layout.slots[0].nonterminal,
                                                           grammar.search_limits().max_depth, site_depth, &names);
  rp::HostPhaseGrammar g = layout.profiles[0];
  rp::normalize_static_phase_weights(g, g.nonterminals, g.productions);

  // 1. tables: HostPhaseGrammar field by field
  std::vector<gagp_expression> ex(g.expressions.size());
  for (std::size_t i = 0; i < g.expressions.size(); ++i) {
    const auto& e = g.expressions[i];
    auto& x = ex[i];
    x.kind = int32_t(e.kind);
    x.node_kind = int32_t(e.node.kind);
    x.opcode = int32_t(e.node.opcode);
    x.operand = e.node.operand;
    x.arity = e.node.arity;
    x.fuel = e.node.fuel;
    x.merge_fuel = e.node.merge_fuel;
    x.type = int32_t(e.node.type);
    x.target = e.target;
    x.scope_count = e.scope_count;
    for (int k = 0; k < GAGP_MAX_ARITY; ++k) {
      x.children[k] = e.children[k];
      x.child_scope[k] = e.child_scope[k];
    }
  }
  std::vector<gagp_production> pr(g.productions.size());
  for (std::size_t i = 0; i < g.productions.size(); ++i) pr[i] = {g.productions[i].expression, 0, g.productions[i].weight};
  std::vector<gagp_nonterminal> nt(g.nonterminals.size());
  for (std::size_t i = 0; i < g.nonterminals.size(); ++i) {
    const auto& n = g.nonterminals[i];
    nt[i] = {n.production_offset, n.production_count, n.scope_count, int32_t(n.normalized_weights), int32_t(n.fixed)};
  }
  std::vector<gagp_domain> dom(g.domains.size());
  for (std::size_t i = 0; i < g.domains.size(); ++i) {
    const auto& d = g.domains[i];
    dom[i] = {d.value_offset, d.value_count, int32_t(d.integer_range), 0, d.minimum, d.maximum};
  }
  std::vector<gagp_value> val(g.values.size());
  for (std::size_t i = 0; i < g.values.size(); ++i) val[i] = {g.values[i].i, int32_t(g.values[i].tag), 0};
  std::vector<gagp_region> reg(g.regions.size());
  for (std::size_t i = 0; i < g.regions.size(); ++i) {
    const auto& r = g.regions[i];
    auto& y = reg[i];
    y = gagp_region{};
    y.traversal = r.traversal;
    y.ranged = r.ranged;
    y.fuel_profile = r.fuel_profile;
    for (int k = 0; k < 3; ++k) {
      y.binders[k] = r.binders[k];
      y.binding_types[k] = int32_t(r.binding_types[0][k]);
    }
    for (int k = 0; k < 6; ++k) y.operand_types[k] = int32_t(r.operand_types[k]);
    y.result_type = int32_t(r.phase_type[0]);
    for (int k = 0; k < 26; ++k) y.event_cost[k] = r.event_cost[k];
    if (r.traversal == 0) {
      // a bounded region: its table entry, the phase bindings' sources and
      // the plan (HostPhaseGrammar::region_sources)
      const auto& source = g.region_sources.at(i);
      const auto& plan = source.plan;
      y.operands = r.operands; y.phases = r.phases; y.captures = r.captures;
      for (int c = 0; c < r.captures && c < 8; ++c) {
        y.capture_kind[c] = int32_t(r.capture_kind[c]);
        y.capture_target[c] = r.capture_target[c];
      }
      for (int p = 0; p < r.phases && p < 8; ++p) {
        y.phase_type[p] = int32_t(r.phase_type[p]);
        y.phase_bindings[p] = r.phase_bindings[p];
        for (int b = 0; b < r.phase_bindings[p] && b < 8; ++b) {
          y.phase_binding_types[p][b] = int32_t(r.binding_types[p][b]);
          y.binding_bank[p][b] = int32_t(source.sources.at(p).at(b).bank);
          y.binding_slot[p][b] = int32_t(source.sources.at(p).at(b).slot);
        }
      }
      y.result_type = int32_t(plan.result_type);
      y.state_count = int32_t(plan.state_types.size());
      y.request_count = int32_t(plan.requests.size());
      y.axis_count = int32_t(plan.coordinate_slots.size());
      y.inclusive = plan.coordinate_endpoint == DomainEndpoint::Inclusive;
      y.memoized = plan.memoized;
      y.frames = plan.limits.frames; y.cells = plan.limits.cells; y.entry_fuel = plan.limits.entry_fuel;
      for (std::size_t k = 0; k < plan.parameter_types.size() && k < 8; ++k)
        y.parameter_types[k] = int32_t(plan.parameter_types[k]);
      for (std::size_t q = 0; q < plan.requests.size() && q < 8; ++q)
        for (std::size_t k = 0; k < plan.requests[q].states.size() && k < 4; ++k) {
          const auto& t = plan.requests[q].states[k];
          y.transition_kind[q][k] = int32_t(t.kind);  // CopyState 0, CoordinateOffset 1 (others are declined)
          y.transition_source[q][k] = int32_t(t.source_state);
          y.transition_offset[q][k] = t.offset;
        }
      for (std::size_t a = 0; a < plan.coordinate_slots.size() && a < 4; ++a) {
        const auto& d = plan.coordinate_domains.at(a);
        y.axis_slot[a] = int32_t(plan.coordinate_slots[a]);
        y.lower_kind[a] = d.lower.kind == RegionBoundKind::Operand;
        y.upper_kind[a] = d.upper.kind == RegionBoundKind::Operand;
        y.lower[a] = d.lower.kind == RegionBoundKind::Operand ? int64_t(d.lower.operand) : d.lower.literal;
        y.upper[a] = d.upper.kind == RegionBoundKind::Operand ? int64_t(d.upper.operand) : d.upper.literal;
      }
    }
  }
  const auto& nts = grammar.nonterminals()[layout.slots[0].nonterminal];
  gagp_grammar tables{};
  tables.expressions = ex.data(); tables.expression_count = int32_t(ex.size());
  tables.productions = pr.data(); tables.production_count = int32_t(pr.size());
  tables.nonterminals = nt.data(); tables.nonterminal_count = int32_t(nt.size());
  tables.domains = dom.data(); tables.domain_count = int32_t(dom.size());
  tables.values = val.data(); tables.value_count = int32_t(val.size());
  tables.minimum = g.minimum.data();
  tables.depth_count = g.depth_count;
  tables.logical_depth_count = g.logical_depth_count;
  tables.site_depth = site_depth;
  tables.root_expression = g.root_expression;
  tables.slot_max_depth = int32_t(layout.slots[0].max_depth);
  tables.slot_type = int32_t(layout.program_terminator ? rp::phase_value_tag(nts.type) : rp::kPhaseStatement);
  tables.local_count = int32_t(names.size());
  for (std::size_t j = 0; j < names.size(); ++j)
    for (const auto& binding : grammar.inputs())
      if (binding.name == names[j]) tables.local_types[j] = int32_t(rp::phase_value_tag(binding.type));
  tables.max_nodes = int32_t(layout.budget.max_nodes);
  tables.fixed_nodes = int32_t(layout.fixed_nodes);
  tables.return_fuel = layout.program_return_fuel;
  tables.regions = reg.data();
  tables.region_count = int32_t(reg.size());

  // 2. cases: CaseSet bindings in evaluator order; IntList inputs as views
  // into one flat array (length word, then the elements)
  const int C = int(case_set.bindings.size()), NI = int(names.size());
  std::vector<int64_t> inputs(std::size_t(C) * NI, 0), expected(C, 0), lists;
  std::vector<int32_t> input_tags(NI, GAGP_TAG_INVALID);
  for (int c = 0; c < C; ++c) {
    for (const auto& b : case_set.bindings[c]) {
      int64_t payload = b.value.i;
      if (b.value.tag == ValueTag::Bool) payload = b.value.b ? 1 : 0;
      if (b.value.tag == ValueTag::IntList) {
        std::vector<Value> xs;
        if (!payload::lookup_list(b.value, &xs)) throw std::runtime_error("IntList input without a payload");
        payload = int64_t(lists.size());
        lists.push_back(int64_t(xs.size()));
        for (const auto& v : xs) lists.push_back(v.i);
      }
      inputs[std::size_t(c) * NI + b.idx] = payload;
      input_tags[b.idx] = int32_t(b.value.tag);
    }
    const Value& e = case_set.expected_values[c];
    expected[c] = e.tag == ValueTag::Bool ? (e.b ? 1 : 0) : e.i;
  }
  gagp_cases cs{};
  cs.case_count = C;
  cs.input_count = NI;
  cs.inputs = inputs.data();
  cs.input_tags = input_tags.data();
  cs.expected = expected.data();
  cs.expected_tag = C ? int32_t(case_set.expected_values[0].tag) : GAGP_TAG_INT;
  cs.list_values = lists.empty() ? nullptr : lists.data();
  cs.list_value_count = int64_t(lists.size());

  // 3. the effective search configuration
  const auto variation = cfg.phase_variation ? *cfg.phase_variation : PhaseVariationPolicy{};
  const auto schedule = cfg.phase_schedule ? *cfg.phase_schedule : PhaseSchedulePolicy{};
  gagp_search_config sc{};
  sc.population = cfg.population_size;
  sc.generations = cfg.generations;
  sc.seed = cfg.seed;
  sc.tournament_size = cfg.selection_pressure;
  sc.crossover_attempts = variation.crossover_attempts;
  sc.crossover_probability = variation.crossover_probability;
  sc.mutation_probability = cfg.mutation_rate;
  sc.mutation_max_nodes = variation.mutation_max_nodes;
  sc.counted_sites = variation.site_draw == PhaseSiteDraw::Counted;
  sc.uniform_phase = variation.site_scope == PhaseSiteScope::UniformPhase;
  sc.steady_state = schedule.mode == PhaseScheduleMode::SteadyState;
  sc.batch = schedule.batch;
  sc.replacement_size = schedule.replacement_size;
  sc.elite_count = cfg.elite_count;
  sc.fuel = cfg.fuel;
  sc.penalty = cfg.penalty;
  sc.metric = int32_t(cfg.fitness_policy.metric);
  sc.grammar_site_ranking = cfg.gpu_phase_site_parsimony;
  sc.reduction_lanes = cfg.gpu_blocksize;

  // 4. admit and run
  int32_t id = -1;
  gagp_status st = gagp_b200_search_create(engine, &tables, &cs, &sc, nullptr, &id);
  if (st == GAGP_DECLINED) {
    *declined = gagp_b200_last_error();
    return false;
  }
  if (st != GAGP_OK) throw std::runtime_error(gagp_b200_last_error());
  if (gagp_b200_search_run(engine, id) != GAGP_OK) throw std::runtime_error(gagp_b200_last_error());

  // 5. results into caller-owned arrays
  const int G = cfg.generations, P = cfg.population_size, stride = int(layout.budget.max_nodes);
  std::vector<double> hbest(G), hmean(G), ffit(P);
  std::vector<int32_t> hwrong(G), hnodes(G), fwrong(P), fnodes(P);
  std::vector<int32_t> hn(G), ho(std::size_t(G) * stride), hc(G), fn(P), fo(std::size_t(P) * stride), fc(P);
  std::vector<int64_t> hk(std::size_t(G) * stride), fk(std::size_t(P) * stride);
  gagp_search_result r{};
  r.generations = G;  // capacity of the history arrays; entries written on return
  r.history_best_fitness = hbest.data(); r.history_mean_fitness = hmean.data();
  r.history_best_wrong = hwrong.data(); r.history_best_nodes = hnodes.data();
  r.history_best = {G, stride, hn.data(), ho.data(), hc.data(), hk.data()};
  r.population = P;
  r.final_fitness = ffit.data(); r.final_wrong = fwrong.data(); r.final_nodes = fnodes.data();
  r.final_rows = {P, stride, fn.data(), fo.data(), fc.data(), fk.data()};
  st = gagp_b200_search_result(engine, id, &r);
  gagp_b200_search_destroy(engine, id);
  if (st != GAGP_OK) throw std::runtime_error(gagp_b200_last_error());

  // 6. rows back into the reference's genomes: each node is its construction
  // expression's node, a constant numbered in prefix order
  // (export_native_phase_layout, phase_layout.hpp:318)
  const auto genome_of = [&](const int32_t* origins, int n, const int64_t* constants, int nc) {
    rp::HostPhaseGene gene;
    int k = 0;
    for (int i = 0; i < n; ++i) {
      auto node = g.expressions.at(origins[i]).node;
      if (node.kind == rp::PhaseTreeKind::Constant) node.operand = k++;
      gene.nodes.push_back(node);
      gene.origins.push_back(origins[i]);
    }
    for (int i = 0; i < nc; ++i) gene.constants.push_back(Value::from_int(constants[i]));
    return rp::export_native_phase_layout(grammar, layout, {gene});
  };
  result = EvolutionResult{};
  result.reproduction_profile = "gagp_b200";
  for (int i = 0; i < r.generations; ++i) {
    ScoredGenome h;
    h.genome = genome_of(ho.data() + std::size_t(i) * stride, hn[i], hk.data() + std::size_t(i) * stride, hc[i]);
    h.fitness = hbest[i];
    h.wrong = hwrong[i];
    result.history_best.push_back(h);
    result.history_best_fitness.push_back(hbest[i]);
    result.history_mean_fitness.push_back(hmean[i]);
  }
  for (int i = 0; i < P; ++i) {
    ScoredGenome m;
    m.genome = genome_of(fo.data() + std::size_t(i) * stride, fn[i], fk.data() + std::size_t(i) * stride, fc[i]);
    m.fitness = ffit[i];
    m.wrong = fwrong[i];
    result.final_population.push_back(m);
  }
  result.best = result.final_population.front();
  result.timing.evaluation_totals.program_cases = r.program_cases;
  result.timing.evaluation_totals.fitness_reused_programs = r.reused_programs;
  return true;
}

}  // namespace gagp::evo

// ------------------------------------------------------------------ driver
namespace {
constexpr const char* kDefaultSearch = R"({
  "format": "gagp-search-config-v1", "representation": "resident",
  "population_size": 1024, "generations": 64,
  "selection": {"method": "tournament", "size": 2}, "elitism": 1,
  "crossover": {"probability": 0.7, "attempts": 8}, "mutation": {"probability": 0.3},
  "sites": {"scope": "uniform_phase", "draw": "counted"}, "limits": {"site_depth": 7},
  "ranking": {"tie_break": "ast_nodes"}, "schedule": {"mode": "steady_state", "replacement_size": 2}})";

std::string quote(const std::string& s) {
  std::string o = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') o += '\\';
    o += c;
  }
  return o + "\"";
}
}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: reference_adapter TASK.json SEARCH.json\n");
    return 2;
  }
  try {
    const auto task = cli_detail::load_task(argv[1]);
    const auto grammar =
        std::make_shared<const gg::CompiledGrammar>(gg::compile_grammar(gg::load_definition(task.grammar_path)));
    const auto cases = cli_detail::load_fitness_cases(task.train_path);
    evo::EvolutionConfig cfg;
    cfg.eval_engine = evo::EvalEngine::CPU;
    cfg.reproduction_backend = evo::repro::ReproductionBackend::Cpu;
    cfg.gpu_blocksize = 512;
    cfg.compiled_grammar = grammar;
    cfg.generation_request = gg::entry_request(*grammar);
    cfg.fuel = int(grammar->execution_limits().fuel);
    cfg.penalty = task.case_cap;
    cfg.fitness_policy = task.fitness;
    cfg.selection_pressure = 2;
    cfg.elite_count = 1;
    cfg.mutation_rate = .3;
    cfg.mutation_subtree_prob = 1;
    cfg.retain_final_population = true;
    cli_detail::apply_search_config(cli_detail::parse_search_config(cli_detail::JsonParser(kDefaultSearch).parse()),
                                    cfg);
    cli_detail::apply_search_config(cli_detail::load_search_config(argv[2]), cfg);

    gagp_engine* engine = nullptr;
    if (gagp_b200_engine_create(0, 0, &engine) != GAGP_OK) throw std::runtime_error(gagp_b200_last_error());
    evo::EvolutionResult mine;
    std::string declined;
    const bool ran = evo::evolve_b200_phase_population(engine, cfg, cases, mine, &declined);
    gagp_b200_engine_destroy(engine);
    const auto ref = evo::evolve_population(cases, cfg, nullptr);

    bool history = ran && mine.history_best.size() == ref.history_best.size();
    std::size_t history_diff = 0;
    std::string history_note;
    for (std::size_t i = 0; history && i < ref.history_best.size(); ++i) {
      const std::string a = cli_detail::program_text(mine.history_best[i].genome.ast);
      const std::string b = cli_detail::program_text(ref.history_best[i].genome.ast);
      history = mine.history_best_fitness[i] == ref.history_best_fitness[i] &&
                mine.history_mean_fitness[i] == ref.history_mean_fitness[i] &&
                mine.history_best[i].wrong == ref.history_best[i].wrong && a == b;
      if (!history) {
        history_diff = i;
        char buf[512];
        std::snprintf(buf, sizeof buf, "best %.17g/%.17g mean %a/%a wrong %d/%d", mine.history_best_fitness[i],
                      ref.history_best_fitness[i], mine.history_mean_fitness[i], ref.history_mean_fitness[i],
                      mine.history_best[i].wrong, ref.history_best[i].wrong);
        history_note = std::string(buf) + " text " + a + " / " + b;
      }
    }
    if (ran && mine.history_best.size() != ref.history_best.size())
      history_note = "history entries " + std::to_string(mine.history_best.size()) + " / " +
                     std::to_string(ref.history_best.size());
    bool final_same = ran && mine.final_population.size() == ref.final_population.size();
    std::size_t first_diff = 0;
    for (std::size_t i = 0; final_same && i < ref.final_population.size(); ++i) {
      const auto& a = mine.final_population[i];
      const auto& b = ref.final_population[i];
      final_same = a.fitness == b.fitness && a.wrong == b.wrong &&
                   a.genome.ast.nodes.size() == b.genome.ast.nodes.size() &&
                   cli_detail::program_text(a.genome.ast) == cli_detail::program_text(b.genome.ast);
      if (!final_same) first_diff = i;
    }
    const auto& tm = mine.timing.evaluation_totals;
    const auto& tr = ref.timing.evaluation_totals;
    std::printf("{\"ran\":%s,\"declined\":%s,\"reference_declined\":%s,\"history_equal\":%s,\"final_equal\":%s,"
                "\"first_history_difference\":%zu,\"history_note\":%s,"
                "\"first_final_difference\":%zu,\"program_cases\":[%llu,%llu],\"reused_programs\":[%llu,%llu],"
                "\"best\":[%s,%s]}\n",
                ran ? "true" : "false", quote(declined).c_str(), quote(ref.resident_declined).c_str(),
                history ? "true" : "false", final_same ? "true" : "false", history_diff, quote(history_note).c_str(),
                first_diff,
                (unsigned long long)tm.program_cases, (unsigned long long)tr.program_cases,
                (unsigned long long)tm.fitness_reused_programs, (unsigned long long)tr.fitness_reused_programs,
                ran ? quote(cli_detail::program_text(mine.best.genome.ast)).c_str() : "\"\"",
                quote(cli_detail::program_text(ref.best.genome.ast)).c_str());
    return 0;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "reference_adapter: %s\n", e.what());
    return 1;
  }
}
