// Test infrastructure only: a driver around the reference's own CPU engine,
// compiled from the reference sources (see oracle/Makefile) into oracle/_ref/.
// It is never linked into the product. It prints, as JSON on stdout:
//
//   ref_driver tables TASK.json [--search F] [--population N] [--seed S]
//       the phase-grammar tables and slot the resident owner admits
//       (compile_phase_variation_grammar + normalize_static_phase_weights,
//       cpp/src/evolution/repro/gpu/phase_population_cpu.cpp:36-47,196-219),
//       the case set in evaluator input order, and the initial population's
//       phase rows (generate_phase_initial_population, then the owner's import
//       and site annotation, phase_population_cpu.cpp:54-113,220-238).
//
//   ref_driver run TASK.json [--search F] [--population N] [--generations G] [--seed S] [--init POP.json]
//       one CPU-engine search (evolve_population, cpp/src/evolution/evolve.cpp:839)
//       with the gagp run defaults (cpp/src/cli/run.cpp:275-300), from the
//       generated population or, with --init, from the first programs of a
//       population document (as `gagp run --init`): the per-generation
//       history, and the final ranked population with fitness, wrong count,
//       node count, program text, program as ast-prefix-v2 JSON and phase row.
//
//   ref_driver lower TASK.json [--search F] [--population N] [--seed S] [--case-detail K]
//       the initial population lowered by the resident owner's phase compiler
//       (reference bytecode: op, flags, a, b, fuel; constants; locals; stack
//       bound), each program's fitness and wrong count from the CPU
//       evaluator, the outcome of its first K cases, and the program as
//       ast-prefix-v2 JSON (encode_ast_json, for `gagp eval`).
//
//   ref_driver batch TASK.json [--search F] [--population N] [--seed S] --round-seed R
//       one make_batch of the CPU resident owner (HostPhasePopulation,
//       phase_population_cpu.cpp:322-353) over the generated initial population
//       with the selection fitness sel[i] = (i * 7919) mod P + 1 and round seed
//       R: every child's reusable parent and phase row (the children committed
//       over members 0..B-1, then exported and imported back).
//
// These outputs are the golden vectors that pin the C restatement and the
// table builder.
#define __device__
#define __host__
#include <algorithm>
#include <array>
#include <cinttypes>
#include <cstdio>
#include <cstring>
#include <thread>
#include <memory>
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
#include "repro/gpu/phase_layout.hpp"
#include "repro/gpu/phase_population_cpu.hpp"
#include "repro/gpu/phase_operators.cuh"
#include "gagp/runtime/cpu/execute_bytecode_cpu.hpp"
#include "gagp/runtime/cpu/fitness_cpu.hpp"

using namespace gagp;
namespace gg = gagp::evo::grammar;
namespace rp = gagp::evo::repro;

namespace {
constexpr const char* kDefaultSearch = R"({
  "format": "gagp-search-config-v1", "representation": "resident",
  "population_size": 1024, "generations": 64,
  "selection": {"method": "tournament", "size": 2}, "elitism": 1,
  "crossover": {"probability": 0.7, "attempts": 8}, "mutation": {"probability": 0.3},
  "sites": {"scope": "uniform_phase", "draw": "counted"}, "limits": {"site_depth": 7},
  "ranking": {"tie_break": "ast_nodes"}, "schedule": {"mode": "steady_state", "replacement_size": 2}})";

struct Args {
  std::string mode, task, search, init;
  int population = 0, generations = 0;
  bool has_seed = false;
  std::uint64_t seed = 0;
  std::uint64_t round_seed = 0;
  int case_detail = 8;
};

std::string hex(double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%a", v);
  return b;
}
std::string num(double v) {
  char b[64];
  std::snprintf(b, sizeof b, "%.17g", v);
  return b;
}
std::string quote(const std::string& s) {
  std::string o = "\"";
  for (char c : s) {
    if (c == '"' || c == '\\') o += '\\';
    o += c;
  }
  return o + "\"";
}
std::string value_json(const Value& v) {
  char b[96];
  std::snprintf(b, sizeof b, "[%d,%" PRId64 ",%d]", int(v.tag), v.i, int(v.b));
  return b;
}

evo::EvolutionConfig make_config(const Args& a, const cli_detail::Task& task,
                                 std::shared_ptr<const gg::CompiledGrammar> grammar) {
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
  cfg.skip_final_eval = false;
  cfg.retain_final_population = true;
  cli_detail::apply_search_config(cli_detail::parse_search_config(cli_detail::JsonParser(kDefaultSearch).parse()), cfg);
  if (!a.search.empty()) cli_detail::apply_search_config(cli_detail::load_search_config(a.search), cfg);
  if (a.population) cfg.population_size = a.population;
  if (a.generations) cfg.generations = a.generations;
  if (a.has_seed) cfg.seed = a.seed;
  return cfg;
}

void print_profile(const rp::HostPhaseGrammar& g) {
  std::printf("{\"root_expression\":%d,\"depth_count\":%d,\"logical_depth_count\":%d,\"site_depth\":%d,",
              g.root_expression, g.depth_count, g.logical_depth_count, int(g.site_depth));
  std::printf("\"expressions\":[");
  for (std::size_t i = 0; i < g.expressions.size(); ++i) {
    const auto& e = g.expressions[i];
    std::printf("%s{\"kind\":%d,\"node\":[%d,%d,%d,%d,%u,%u,%d],\"native_kind\":%d,\"target\":%d,\"children\":[",
                i ? "," : "", int(e.kind), int(e.node.kind), int(e.node.opcode), e.node.operand, e.node.arity,
                e.node.fuel, e.node.merge_fuel, int(e.node.type), e.native_kind, e.target);
    for (int c = 0; c < rp::kPhaseMaxArity; ++c) std::printf("%s%d", c ? "," : "", e.children[c]);
    std::printf("],\"scope_count\":%d,\"child_scope\":[", e.scope_count);
    for (int c = 0; c < rp::kPhaseMaxArity; ++c) std::printf("%s%d", c ? "," : "", int(e.child_scope[c]));
    std::printf("],\"bind_argument\":%d}", e.bind_argument);
  }
  std::printf("],\"productions\":[");
  for (std::size_t i = 0; i < g.productions.size(); ++i)
    std::printf("%s[%d,\"%s\"]", i ? "," : "", g.productions[i].expression, hex(g.productions[i].weight).c_str());
  std::printf("],\"nonterminals\":[");
  for (std::size_t i = 0; i < g.nonterminals.size(); ++i) {
    const auto& n = g.nonterminals[i];
    std::printf("%s[%d,%d,%d,%d,%d]", i ? "," : "", n.production_offset, n.production_count, n.scope_count,
                int(n.normalized_weights), int(n.fixed));
  }
  std::printf("],\"domains\":[");
  for (std::size_t i = 0; i < g.domains.size(); ++i) {
    const auto& d = g.domains[i];
    std::printf("%s[%d,%d,%d,%" PRId64 ",%" PRId64 "]", i ? "," : "", d.value_offset, d.value_count,
                int(d.integer_range), d.minimum, d.maximum);
  }
  std::printf("],\"values\":[");
  for (std::size_t i = 0; i < g.values.size(); ++i) std::printf("%s%s", i ? "," : "", value_json(g.values[i]).c_str());
  std::printf("],\"minimum\":[");
  for (std::size_t i = 0; i < g.minimum.size(); ++i) std::printf("%s%u", i ? "," : "", g.minimum[i]);
  // the region table: traversals and bounded regions (PhaseRegionInfo)
  std::printf("],\"regions\":[");
  for (std::size_t i = 0; i < g.regions.size(); ++i) {
    const auto& r = g.regions[i];
    std::printf("%s{\"traversal\":%d,\"operands\":%d,\"phases\":%d,\"captures\":[", i ? "," : "", r.traversal,
                r.operands, r.phases);
    for (int c = 0; c < r.captures; ++c)
      std::printf("%s[%d,%d]", c ? "," : "", int(r.capture_kind[c]), r.capture_target[c]);
    std::printf("],\"operand_types\":[");
    for (int c = 0; c < r.operands; ++c) std::printf("%s%d", c ? "," : "", int(r.operand_types[c]));
    std::printf("],\"phase_types\":[");
    for (int p = 0; p < r.phases; ++p) std::printf("%s%d", p ? "," : "", int(r.phase_type[p]));
    std::printf("],\"binding_types\":[");
    for (int p = 0; p < r.phases; ++p) {
      std::printf("%s[", p ? "," : "");
      for (int b = 0; b < r.phase_bindings[p]; ++b) std::printf("%s%d", b ? "," : "", int(r.binding_types[p][b]));
      std::printf("]");
    }
    std::printf("]}");
  }
  std::printf("]}");
}

void print_row(const rp::HostPhaseGene& gene, const std::vector<rp::PhaseGeneSite>* sites) {
  std::printf("{\"nodes\":[");
  for (std::size_t j = 0; j < gene.nodes.size(); ++j) {
    const auto& n = gene.nodes[j];
    std::printf("%s[%d,%d,%d,%d,%u,%u,%d]", j ? "," : "", int(n.kind), int(n.opcode), n.operand, n.arity, n.fuel,
                n.merge_fuel, int(n.type));
  }
  std::printf("],\"origins\":[");
  for (std::size_t j = 0; j < gene.origins.size(); ++j) std::printf("%s%d", j ? "," : "", gene.origins[j]);
  std::printf("],\"constants\":[");
  for (std::size_t j = 0; j < gene.constants.size(); ++j)
    std::printf("%s%s", j ? "," : "", value_json(gene.constants[j]).c_str());
  std::printf("]");
  if (sites) {
    std::printf(",\"sites\":[");
    for (std::size_t j = 0; j < sites->size(); ++j) {
      const auto& s = (*sites)[j];
      std::printf("%s[%d,%d,%d,%d]", j ? "," : "", s.nonterminal, s.entry_expression, s.parent_scope, s.scope);
    }
    std::printf("]");
  }
  std::printf("}");
}

int run_tables(const Args& a) {
  const auto task = cli_detail::load_task(a.task);
  const auto grammar = std::make_shared<const gg::CompiledGrammar>(gg::compile_grammar(gg::load_definition(task.grammar_path)));
  const auto cases = cli_detail::load_fitness_cases(task.train_path);
  const auto cfg = make_config(a, task, grammar);
  const auto case_set = evo::prepare_case_set(cases);
  const auto& names = case_set.input_names;
  const int site_depth = cfg.gpu_phase_site_depth;
  const auto population = rp::generate_phase_initial_population(*grammar, *cfg.generation_request, names,
                                                                 cfg.population_size, cfg.seed, site_depth);
  rp::NativePhaseGrammarProfiles profiles(grammar, names);
  auto layout = rp::import_native_phase_layout(*grammar, population.front(), &profiles, &names, true);
  for (std::size_t k = 0; k < layout.slots.size(); ++k)
    layout.profiles[k] = rp::compile_phase_variation_grammar(*grammar, layout.slots[k].nonterminal,
                                                             grammar->search_limits().max_depth, site_depth, &names);
  std::printf("{\"inputs\":[");
  for (std::size_t i = 0; i < names.size(); ++i) std::printf("%s%s", i ? "," : "", quote(names[i]).c_str());
  std::printf("],\"fuel\":%d,\"penalty\":%s,\"metric\":%d,\"population\":%d,\"generations\":%d,\"seed\":\"%" PRIu64 "\",",
              cfg.fuel, num(cfg.penalty).c_str(), int(cfg.fitness_policy.metric), cfg.population_size,
              cfg.generations, cfg.seed);
  std::printf("\"site_depth\":%d,\"layout\":{\"fixed_nodes\":%zu,\"max_nodes\":%u,\"max_depth\":%u,"
              "\"whole_program\":%d,\"program_terminator\":%d,\"return_fuel\":%u},",
              site_depth, layout.fixed_nodes, layout.budget.max_nodes, layout.budget.max_depth,
              int(layout.whole_program), int(layout.program_terminator), layout.program_return_fuel);
  std::printf("\"slots\":[");
  std::vector<std::unique_ptr<rp::HostPhaseGrammar>> normalized;
  for (std::size_t k = 0; k < layout.slots.size(); ++k) {
    auto g = std::make_unique<rp::HostPhaseGrammar>(layout.profiles[k]);
    rp::normalize_static_phase_weights(*g, g->nonterminals, g->productions);
    const auto& nt = grammar->nonterminals()[layout.slots[k].nonterminal];
    const int type = layout.program_terminator || !layout.whole_program ? int(rp::phase_value_tag(nt.type))
                                                                         : int(rp::kPhaseStatement);
    std::printf("%s{\"nonterminal\":%u,\"max_depth\":%u,\"scope\":%zu,\"type\":%d,\"locals\":[", k ? "," : "",
                layout.slots[k].nonterminal, layout.slots[k].max_depth, nt.scope.size(), type);
    if (layout.whole_program) {
      for (std::size_t j = 0; j < names.size(); ++j)
        for (const auto& binding : grammar->inputs())
          if (binding.name == names[j]) std::printf("%s%d", j ? "," : "", int(rp::phase_value_tag(binding.type)));
    } else {
      for (std::size_t j = 0; j < nt.scope.size(); ++j)
        std::printf("%s%d", j ? "," : "", int(rp::phase_value_tag(nt.scope[j].type)));
    }
    std::printf("],\"profile\":");
    print_profile(*g);
    std::printf("}");
    normalized.push_back(std::move(g));
  }
  std::printf("],\"cases\":[");
  for (std::size_t c = 0; c < case_set.bindings.size(); ++c) {
    std::vector<Value> row(names.size(), Value::invalid());
    for (const auto& b : case_set.bindings[c]) row.at(b.idx) = b.value;
    std::printf("%s{\"inputs\":[", c ? "," : "");
    for (std::size_t j = 0; j < row.size(); ++j) std::printf("%s%s", j ? "," : "", value_json(row[j]).c_str());
    std::printf("],\"expected\":%s}", value_json(case_set.expected_values[c]).c_str());
  }
  std::printf("],\"initial\":[");
  for (std::size_t p = 0; p < population.size(); ++p) {
    const auto imported = rp::import_native_phase_layout(*grammar, population[p], &profiles, &names, false);
    std::printf("%s[", p ? "," : "");
    for (std::size_t k = 0; k < imported.genes.size(); ++k) {
      const auto& gene = imported.genes[k];
      const auto& g = *normalized[k];
      rp::PhaseGrammarView view{g.expressions.data(), int(g.expressions.size()), g.productions.data(),
                                int(g.productions.size()), g.nonterminals.data(), int(g.nonterminals.size()),
                                g.domains.data(), int(g.domains.size()), g.values.data(), int(g.values.size()),
                                g.minimum.data(), g.depth_count, g.logical_depth_count, g.site_depth,
                                g.regions.data(), int(g.regions.size())};
      std::vector<rp::PhaseGeneSite> sites(gene.nodes.size());
      const auto& nt = grammar->nonterminals()[layout.slots[k].nonterminal];
      const bool ok = rp::annotate_phase_tree(view, g.root_expression, int(nt.scope.size()), gene.nodes.data(),
                                              gene.origins.data(), int(gene.nodes.size()), sites.data());
      if (!ok) throw std::runtime_error("annotation failed");
      if (k) std::printf(",");
      print_row(gene, &sites);
    }
    std::printf("]");
  }
  std::printf("]}\n");
  return 0;
}

int run_batch(const Args& a) {
  const auto task = cli_detail::load_task(a.task);
  const auto grammar = std::make_shared<const gg::CompiledGrammar>(gg::compile_grammar(gg::load_definition(task.grammar_path)));
  const auto cases = cli_detail::load_fitness_cases(task.train_path);
  const auto cfg = make_config(a, task, grammar);
  const auto case_set = evo::prepare_case_set(cases);
  const auto& names = case_set.input_names;
  const int site_depth = cfg.gpu_phase_site_depth;
  const int P = cfg.population_size;
  const auto population = rp::generate_phase_initial_population(*grammar, *cfg.generation_request, names, P, cfg.seed,
                                                                 site_depth);
  rp::HostPhasePopulation owner(grammar, population, names, site_depth,
                                cfg.phase_variation ? *cfg.phase_variation : evo::PhaseVariationPolicy{});
  int B = P;
  if (cfg.phase_schedule && cfg.phase_schedule->batch > 0) B = cfg.phase_schedule->batch;
  owner.begin_steady(B);
  std::vector<double> selection(P);
  for (int i = 0; i < P; ++i) selection[i] = double((std::uint64_t(i) * 7919u) % std::uint64_t(P) + 1);
  const int pressure = std::clamp(cfg.selection_pressure, 1, P);
  const auto reuse = owner.make_batch(selection, pressure, cfg.mutation_rate, a.round_seed, nullptr);
  std::vector<std::array<int, 2>> placements;
  for (int b = 0; b < B; ++b) placements.push_back({b, b});
  owner.commit_batch(placements);
  rp::NativePhaseGrammarProfiles profiles(grammar, names);
  std::printf("{\"batch\":%d,\"round_seed\":\"%" PRIu64 "\",\"reuse\":[", B, a.round_seed);
  for (std::size_t b = 0; b < reuse.size(); ++b) std::printf("%s%d", b ? "," : "", reuse[b]);
  std::printf("],\"children\":[");
  for (int b = 0; b < B; ++b) {
    const auto imported = rp::import_native_phase_layout(*grammar, owner.export_member(std::size_t(b)), &profiles,
                                                         &names, false);
    std::printf("%s", b ? "," : "");
    print_row(imported.genes.at(0), nullptr);
  }
  std::printf("]}\n");
  return 0;
}

// The initial population lowered by the resident owner's phase compiler, as
// HostPhasePopulation::lower_member does for a batch child
// (phase_population_cpu.cpp:144-159: compile_phase_tree<true,true>, then
// patch_whole_program), and each program scored by the CPU evaluator
// (eval_fitness_cpu, cpp/src/runtime/cpu/fitness_cpu.cpp:57-176) with the
// first `case_detail` cases run one by one (execute_bytecode_cpu).
int run_lower(const Args& a) {
  const auto task = cli_detail::load_task(a.task);
  const auto grammar = std::make_shared<const gg::CompiledGrammar>(gg::compile_grammar(gg::load_definition(task.grammar_path)));
  const auto cases = cli_detail::load_fitness_cases(task.train_path);
  const auto cfg = make_config(a, task, grammar);
  const auto case_set = evo::prepare_case_set(cases);
  const auto& names = case_set.input_names;
  const int site_depth = cfg.gpu_phase_site_depth;
  const auto population = rp::generate_phase_initial_population(*grammar, *cfg.generation_request, names,
                                                                 cfg.population_size, cfg.seed, site_depth);
  rp::NativePhaseGrammarProfiles profiles(grammar, names);
  auto layout = rp::import_native_phase_layout(*grammar, population.front(), &profiles, &names, true);
  for (std::size_t k = 0; k < layout.slots.size(); ++k)
    layout.profiles[k] = rp::compile_phase_variation_grammar(*grammar, layout.slots[k].nonterminal,
                                                             grammar->search_limits().max_depth, site_depth, &names);
  if (!layout.whole_program || layout.slots.size() != 1) throw std::runtime_error("lower: one whole-program phase only");
  const auto& g = layout.profiles[0];
  const auto& nt = grammar->nonterminals()[layout.slots[0].nonterminal];
  const auto type = layout.program_terminator ? rp::phase_value_tag(nt.type) : rp::kPhaseStatement;
  std::vector<ValueTag> locals(names.size(), ValueTag::Invalid);
  for (std::size_t j = 0; j < names.size(); ++j)
    for (const auto& binding : grammar->inputs())
      if (binding.name == names[j]) locals[j] = rp::phase_value_tag(binding.type);
  std::vector<gagp::gpu_detail::DInstr> code(4 * 1024);
  std::vector<Value> values(1024);
  std::vector<std::vector<std::pair<int, Value>>> inputs(case_set.bindings.size());
  for (std::size_t c = 0; c < case_set.bindings.size(); ++c)
    for (const auto& b : case_set.bindings[c]) inputs[c].emplace_back(b.idx, b.value);
  const int detail = std::min<int>(a.case_detail, int(inputs.size()));
  std::printf("{\"fuel\":%d,\"rows\":[", cfg.fuel);
  for (std::size_t p = 0; p < population.size(); ++p) {
    const auto imported = rp::import_native_phase_layout(*grammar, population[p], &profiles, &names, false);
    const auto& gene = imported.genes.at(0);
    const auto r = rp::compile_phase_tree<true, true>(gene.nodes.data(), int(gene.nodes.size()), gene.constants.data(),
        int(gene.constants.size()), locals.data(), int(locals.size()), type, code.data(), int(code.size()),
        values.data(), int(values.size()), g.regions.data(), int(g.regions.size()));
    std::printf("%s{\"origins\":[", p ? "," : "");
    for (std::size_t j = 0; j < gene.origins.size(); ++j) std::printf("%s%d", j ? "," : "", gene.origins[j]);
    std::printf("],\"constants\":[");
    for (std::size_t j = 0; j < gene.constants.size(); ++j) std::printf("%s%" PRId64, j ? "," : "", gene.constants[j].i);
    std::printf("],\"status\":%d,\"program\":%s", int(r.status), cli_detail::encode_ast_json(population[p].ast).c_str());
    if (r.status != rp::PhaseCompileStatus::Ok) { std::printf("}"); continue; }
    BytecodeProgram program = imported.executable;
    rp::patch_whole_program(program, layout, code.data(), r.code_count, values.data(), r.constant_count, r);
    std::printf(",\"stack_bound\":%d,\"n_locals\":%d,\"fuel_table\":%d,\"code\":[", r.stack_bound, program.n_locals,
                int(!program.instruction_fuel.empty()));
    for (int i = 0; i < r.code_count; ++i)
      std::printf("%s[%d,%d,%d,%d,%u]", i ? "," : "", int(code[i].op), int(code[i].flags), code[i].a, code[i].b,
                  code[i].fuel);
    std::printf("],\"consts\":[");
    for (int i = 0; i < r.constant_count; ++i) std::printf("%s%s", i ? "," : "", value_json(values[i]).c_str());
    std::vector<unsigned> wrong;
    const auto fitness = eval_fitness_cpu({program}, case_set.bindings, case_set.expected_values, cfg.fuel,
                                          cfg.penalty, cfg.gpu_blocksize, cfg.fitness_policy, &wrong, nullptr);
    std::printf("],\"fitness\":%s,\"wrong\":%u,\"cases\":[", num(fitness.at(0)).c_str(), wrong.at(0));
    for (int c = 0; c < detail; ++c) {
      int fuel = cfg.fuel;
      const auto out = execute_bytecode_cpu(program, inputs[c], fuel);
      // [error code or -1, result tag, result payload, fuel left]
      std::printf("%s[%d,%d,%" PRId64 ",%d]", c ? "," : "", out.is_error ? int(out.err.code) : -1,
                  out.is_error ? -1 : int(out.value.tag), out.is_error ? 0 : out.value.i, fuel);
    }
    std::printf("]}");
  }
  std::printf("]}\n");
  return 0;
}

int run_search(const Args& a) {
  const auto task = cli_detail::load_task(a.task);
  const auto grammar = std::make_shared<const gg::CompiledGrammar>(gg::compile_grammar(gg::load_definition(task.grammar_path)));
  const auto cases = cli_detail::load_fitness_cases(task.train_path);
  const auto cfg = make_config(a, task, grammar);
  const auto case_set = evo::prepare_case_set(cases);
  // an imported initial population (`gagp run --init`, run.cpp:146-174): the
  // first population_size programs of a population document, in order
  std::vector<evo::ProgramGenome> initial;
  if (!a.init.empty()) {
    std::FILE* f = std::fopen(a.init.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open " + a.init);
    std::string text;
    char buf[65536];
    for (std::size_t got; (got = std::fread(buf, 1, sizeof buf, f)) > 0;) text.append(buf, got);
    std::fclose(f);
    const auto doc = cli_detail::JsonParser(text, {true, 512}).parse();
    for (const auto& program : doc.object_v.at("programs").array_v) {
      if (initial.size() == std::size_t(cfg.population_size)) break;
      evo::ProgramGenome g;
      g.ast = cli_detail::decode_ast_json(program);
      g.meta = evo::build_genome_meta(g.ast);
      g.derivation = std::make_shared<gg::DerivationMetadata>(gg::reconstruct_derivation(*grammar, g));
      initial.push_back(std::move(g));
    }
    if (initial.size() != std::size_t(cfg.population_size)) throw std::runtime_error("--init: too few programs");
  }
  const auto result = evo::evolve_population(cases, cfg, initial.empty() ? nullptr : &initial);
  rp::NativePhaseGrammarProfiles profiles(grammar, case_set.input_names);
  const auto& totals = result.timing.evaluation_totals;
  std::printf("{\"declined\":%s,\"time_ms\":%s,\"init_ms\":%s,\"program_cases\":%llu,\"reused_programs\":%llu,\"history\":[",
              quote(result.resident_declined).c_str(), num(result.timing.total_ms).c_str(),
              num(result.timing.init_population_ms).c_str(), (unsigned long long)totals.program_cases,
              (unsigned long long)totals.fitness_reused_programs);
  for (std::size_t i = 0; i < result.history_best.size(); ++i) {
    const auto& h = result.history_best[i];
    std::printf("%s{\"best_fitness\":%s,\"mean_fitness\":\"%s\",\"best_wrong\":%d,\"best_nodes\":%zu,\"text\":%s}",
                i ? "," : "", num(result.history_best_fitness[i]).c_str(), hex(result.history_mean_fitness[i]).c_str(),
                h.wrong, h.genome.ast.nodes.size(), quote(cli_detail::program_text(h.genome.ast)).c_str());
  }
  std::printf("],\"final\":[");
  for (std::size_t i = 0; i < result.final_population.size(); ++i) {
    const auto& m = result.final_population[i];
    std::printf("%s{\"fitness\":%s,\"wrong\":%d,\"nodes\":%zu,\"text\":%s,\"program\":%s,\"rows\":[", i ? "," : "",
                num(m.fitness).c_str(), m.wrong, m.genome.ast.nodes.size(),
                quote(cli_detail::program_text(m.genome.ast)).c_str(), cli_detail::encode_ast_json(m.genome.ast).c_str());
    if (result.resident_declined.empty()) {
      const auto imported = rp::import_native_phase_layout(*grammar, m.genome, &profiles, &case_set.input_names, false);
      for (std::size_t k = 0; k < imported.genes.size(); ++k) {
        if (k) std::printf(",");
        print_row(imported.genes[k], nullptr);
      }
    }
    std::printf("]}");
  }
  std::printf("]}\n");
  return 0;
}
}  // namespace

int main(int argc, char** argv) {
  if (argc >= 2 && std::string(argv[1]) == "--nproc") {
    std::printf("%u\n", std::thread::hardware_concurrency());
    return 0;
  }
  if (argc < 3) {
    std::fprintf(stderr, "usage: ref_driver tables|run|batch TASK.json [--search F] [--population N] [--generations G] "
                         "[--seed S] [--round-seed R]\n");
    return 2;
  }
  Args a;
  a.mode = argv[1];
  a.task = argv[2];
  for (int i = 3; i + 1 < argc; i += 2) {
    const std::string k = argv[i], v = argv[i + 1];
    if (k == "--search") a.search = v;
    else if (k == "--population") a.population = std::stoi(v);
    else if (k == "--generations") a.generations = std::stoi(v);
    else if (k == "--seed") { a.has_seed = true; a.seed = std::stoull(v); }
    else if (k == "--round-seed") a.round_seed = std::stoull(v);
    else if (k == "--case-detail") a.case_detail = std::stoi(v);
    else if (k == "--init") a.init = v;
    else { std::fprintf(stderr, "unknown option %s\n", k.c_str()); return 2; }
  }
  try {
    if (a.mode == "tables") return run_tables(a);
    if (a.mode == "run") return run_search(a);
    if (a.mode == "batch") return run_batch(a);
    if (a.mode == "lower") return run_lower(a);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "ref_driver: %s\n", e.what());
    return 1;
  }
  std::fprintf(stderr, "unknown mode\n");
  return 2;
}
