"""Converts the reference's own VM known-answer fixtures
(cpp/tests/fixtures/runtime/{scalar,control_flow,builtins,typed_values}.json,
format bytecode-fixture-v2) into tests/golden/vm_fixtures.json: the scenarios
and cases in the engine's subset, their programs in the 5-int instruction form
the engine's exact VM runs ([op, flags, a, b, fuel]).

Kept: programs of the subset's opcodes and builtins with Int/Bool constants;
cases whose inputs are Int, Bool or IntList and whose expectation is an Int or
Bool value, a ZeroDivisionError, a ValueError (index range) or a Timeout.
Left out, with the reason recorded: cases expecting TypeError or NameError
(the engine runs only the phase compiler's statically typed output, in which
neither can occur) and values of other types.

Run here (the container with the reference tree):
    python tests/golden/make_vm_fixtures.py [REFERENCE_ROOT]
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OPS = {"PUSH_CONST": 0, "LOAD": 1, "STORE": 2, "NEG": 3, "NOT": 4, "ADD": 5, "SUB": 6, "MUL": 7, "MOD": 9, "LT": 10,
       "LE": 11, "GT": 12, "GE": 13, "EQ": 14, "NE": 15, "JMP": 16, "JMP_IF_FALSE": 17, "JMP_IF_TRUE": 18,
       "CALL_BUILTIN": 19, "RETURN": 20}
BUILTINS = {0: "abs", 1: "min", 2: "max", 4: "len", 7: "index", 13: "idiv0", 14: "imod0", 28: "trunc_div0",
            29: "trunc_mod0"}
TAGS = {"int": 0, "bool": 2, "int_list": 5}
ERRORS = {"ZeroDivisionError", "ValueError", "Timeout"}


def convert(root):
    out, skipped = [], []
    for name in ("scalar", "control_flow", "builtins", "typed_values"):
        with open(os.path.join(root, "cpp", "tests", "fixtures", "runtime", name + ".json")) as f:
            doc = json.load(f)
        for sc in doc["scenarios"]:
            prog = sc["program"]
            code, ok = [], True
            for ins in prog["code"]:
                op = OPS.get(ins["op"])
                if op is None or (op == 19 and ins.get("a") not in BUILTINS):
                    ok = False
                    break
                flags = (1 if "a" in ins else 0) | (2 if "b" in ins else 0)
                code.append([op, flags, int(ins.get("a", 0)), int(ins.get("b", 0)), 1])
            consts = []
            for c in prog.get("consts", []):
                if c["type"] not in ("int", "bool"):
                    ok = False
                    break
                consts.append(int(c["value"]))
            if not ok:
                skipped.append({"fixture": name, "intent": sc["intent"], "why": "opcode, builtin or constant outside the subset"})
                continue
            cases = []
            for case in sc["cases"]:
                types = [i["value"]["type"] for i in case["inputs"]]
                err = case.get("expected_error")
                exp = case.get("expected")
                if any(t not in TAGS for t in types):
                    skipped.append({"fixture": name, "intent": sc["intent"], "why": "input type outside Int, Bool, IntList"})
                    continue
                if err is not None and err not in ERRORS:
                    skipped.append({"fixture": name, "intent": sc["intent"], "why": err + " cannot occur in typed lowered code"})
                    continue
                if err is None and exp["type"] not in ("int", "bool"):
                    skipped.append({"fixture": name, "intent": sc["intent"], "why": "result type outside Int and Bool"})
                    continue
                inputs = [{"idx": i["idx"], "tag": TAGS[i["value"]["type"]],
                           "value": i["value"]["value"] if i["value"]["type"] == "int_list" else int(i["value"]["value"])}
                          for i in case["inputs"]]
                cases.append({"inputs": inputs, "error": err,
                              "expected": None if err else {"tag": TAGS[exp["type"]], "value": int(exp["value"])}})
            if cases:
                out.append({"fixture": name, "intent": sc["intent"], "n_locals": prog["n_locals"], "fuel": doc["fuel"],
                            "code": code, "consts": consts, "cases": cases})
    return {"source": "cpp/tests/fixtures/runtime/*.json (bytecode-fixture-v2)", "scenarios": out, "skipped": skipped}


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get(
        "GAGP_REFERENCE", os.path.join(os.path.dirname(os.path.dirname(os.path.dirname(HERE))), "reference"))
    doc = convert(root)
    with open(os.path.join(HERE, "vm_fixtures.json"), "w") as f:
        json.dump(doc, f, indent=1)
    print(len(doc["scenarios"]), "scenarios,", sum(len(s["cases"]) for s in doc["scenarios"]), "cases;",
          len(doc["skipped"]), "left out")
