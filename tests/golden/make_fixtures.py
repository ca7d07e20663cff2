"""Generate the committed golden fixtures under tests/golden/.

Run here, where the reference sources are mounted (``--reference``); the GPU
box never runs this script. It writes

* ``known_answers.json`` - known answers read out of the reference's own test
  suite (haskell-tests/LLP.hs, LL.hs, RegularExpression.hs): the test
  grammars, the LLP(1,1) item collection and PSLS table of the paper grammar,
  LL(k) and LLP(q,k) parse results, FIRST/FOLLOW sets, regex match cases, and
  the README's ``12+(3*4)`` tree (README.md:81-108) converted to the compact
  productions-only form;
* ``records.json`` - response records written by the reference's C backend
  (oracle/_ref, built by oracle/build_ref.py) for small inputs of every grammar
  configuration, as hex;
* ``records_modes.json`` - the same for the lexer-mode and parser-mode
  programs (oracle/_ref/<config>_lexer, <config>_parser): bytes in for the
  lexer, terminal ids in for the parser.
"""

from __future__ import annotations

import argparse
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

# --------------------------------------------------------------------------
# A reader for the Haskell literals used in the reference's tests
# --------------------------------------------------------------------------

_TOKEN = re.compile(r'\s+|--[^\n]*|"(?:[^"\\]|\\.)*"|[A-Za-z_][A-Za-z0-9_\'.]*|[\[\](){},=]|\d+')


def tokens(text):
    for m in _TOKEN.finditer(text):
        t = m.group(0)
        if t.isspace() or t.startswith("--"):
            continue
        yield t


class HsReader:
    """Values: strings, ints, lists, tuples, records, and the constructors of
    the augmented grammar used by haskell-tests/LLP.hs."""

    def __init__(self, text):
        self.t = list(tokens(text))
        self.i = 0

    def peek(self):
        return self.t[self.i] if self.i < len(self.t) else None

    def take(self, want=None):
        tok = self.t[self.i]
        if want is not None and tok != want:
            raise ValueError("expected %r got %r at %d" % (want, tok, self.i))
        self.i += 1
        return tok

    def value(self):
        tok = self.peek()
        if tok == "[":
            self.take("[")
            out = []
            while self.peek() != "]":
                out.append(self.value())
                if self.peek() == ",":
                    self.take(",")
            self.take("]")
            return out
        if tok == "(":
            self.take("(")
            out = []
            while self.peek() != ")":
                out.append(self.value())
                if self.peek() == ",":
                    self.take(",")
            self.take(")")
            return out[0] if len(out) == 1 else {"tuple": out}
        if tok.startswith('"'):
            self.take()
            return json.loads(tok)
        if tok.isdigit():
            self.take()
            return int(tok)
        self.take()
        if tok == "Set.fromList":
            return {"set": self.value()}
        if tok in ("augT", "augNT", "augT'", "augNT'"):
            return {"ctor": tok, "arg": self.value()}
        if tok == "Item":
            return {"item": self.record()}
        if tok == "DotProduction":
            lhs = self.value()
            a = self.value()
            b = self.value()
            return {"dot": [lhs, a, b]}
        return {"ctor": tok}

    def record(self):
        self.take("{")
        out = {}
        while self.peek() != "}":
            k = self.take()
            self.take("=")
            out[k] = self.value()
            if self.peek() == ",":
                self.take(",")
        self.take("}")
        return out


def binding(src: str, name: str) -> str:
    """Text of the right-hand side of a top-level ``name = ...`` binding."""
    m = re.search(r"^%s\s*=\s*\n?(.*?)(?=^\S)" % re.escape(name), src + "\nEND", re.S | re.M)
    if not m:
        raise ValueError(name)
    return m.group(1)


def grammar_from(src: str, name: str):
    body = binding(src, name)
    start = re.search(r'start\s*=\s*"([^"]*)"', body).group(1)
    strlist = r'\[((?:\s*"(?:[^"\\]|\\.)*"\s*,?)*)\s*\]'
    terms = json.loads("[" + re.search(r"(?<!non)terminals\s*=\s*" + strlist, body, re.S).group(1) + "]")
    nts = json.loads("[" + re.search(r"nonterminals\s*=\s*" + strlist, body, re.S).group(1) + "]")
    prods = []
    symlist = r'\[((?:\s*(?:Nonterminal|Terminal)\s+"(?:[^"\\]|\\.)*"\s*,?)*)\s*\]'
    for m in re.finditer(r'Production\s+"([^"]*)"\s*' + symlist, body, re.S):
        syms = [[k, json.loads(v)] for k, v in re.findall(r'(Nonterminal|Terminal)\s+("(?:[^"\\]|\\.)*")', m.group(2))]
        prods.append([m.group(1), syms])
    return {"start": start, "terminals": terms, "nonterminals": nts, "productions": prods}


def known_answers(ref: str) -> dict:
    def rd(p):
        with open(os.path.join(ref, p), encoding="utf-8") as f:
            return f.read()

    llp = rd("haskell-tests/LLP.hs")
    ll = rd("haskell-tests/LL.hs")
    rex = rd("haskell-tests/RegularExpression.hs")
    out = {"source": "haskell-tests of CoderDue/alpacc"}
    out["llp_grammar"] = grammar_from(llp, "grammar")
    out["llp_collection"] = HsReader(binding(llp, "collection")).value()
    out["llp_psls"] = HsReader(binding(llp, "pslsTable").replace("Map.fromList", "")).value()
    m = re.search(r'input = map List.singleton "([^"]*)"', llp)
    exp = re.search(r"expected = Just \[([0-9, ]+)\]", llp[m.end():])
    out["llp_parse"] = {"input": list(m.group(1)), "expected": [int(x) for x in exp.group(1).split(",")],
                        "qk": [[q, k] for q in (1, 2, 3) for k in (1, 2, 3)]}
    for g in ("grammar", "followExtendedGrammar", "extendedGrammar", "bookGrammar"):
        out["ll_" + g] = grammar_from(ll, g)
    m = re.search(r'input = List.singleton <\$> "([^"]*)"\s*\n\s*result = llkParse\' .*?\n\s*expected = Just \(\[\], \[\], \[([0-9, ]+)\]\)',
                  ll, re.S)
    out["ll_parse"] = {"grammar": "extendedGrammar", "input": list(m.group(1)),
                       "expected": [int(x) for x in m.group(2).split(",")], "k": list(range(1, 11))}
    m = re.search(r'input = List.singleton <\$> "(ab\$)"', ll)
    out["ll_parse_fail"] = {"grammar": "extendedGrammar", "input": list(m.group(1)), "k": 1}

    def sets_of(block):
        return [[list(map(json.loads, re.findall(r'"(?:[^"\\]|\\.)*"', s))) for s in re.findall(r"\[(.*?)\]", one)]
                for one in re.findall(r"Set\.fromList \[((?:\[[^\]]*\](?:,\s*)?)*)\]", block)]

    out["first_small"] = {"grammar": "grammar", "k": 1, "expected": sets_of(binding(ll, "firstSmallTestCase"))}
    out["first_large"] = {"grammar": "bookGrammar", "k": 1, "expected": sets_of(binding(ll, "firstLargeTestCase"))}
    out["follow_small"] = {"grammar": "followExtendedGrammar", "k": 1,
                           "expected": sets_of(binding(ll, "followSmallTestCase"))}
    out["follow_large"] = {"grammar": "bookGrammar", "k": 1, "expected": sets_of(binding(ll, "followLargeTestCase"))}
    cases = []
    for m in re.finditer(r'regularExpressionMatchCase\s*\n\s*isMatch\s*\n\s*("(?:[^"\\]|\\.)*")\s*\n\s*(\[.*?\])\s*\n\s*(\[.*?\])',
                         rex, re.S):
        cases.append({"regex": json.loads(m.group(1)), "valid": json.loads(m.group(2)),
                      "invalid": json.loads(m.group(3))})
    out["regex_cases"] = cases
    # README.md:81-108: the example tree (terminal nodes included, older
    # format); its spans and terminal names spell the input 12+(3*4).
    out["readme_arithmetic"] = {"input": "12+(3*4)", "readme_nodes": readme_tree(rd("README.md"))}
    return out


def readme_tree(readme: str):
    """(parent, kind, name, span) rows of the README's example tree."""
    rows = []
    for m in re.finditer(r"\((\d+), #(production|terminal) \(#(\w+)\)(?: \((\d+), (\d+)\))?\)", readme):
        rows.append([int(m.group(1)), m.group(2), m.group(3),
                     [int(m.group(4)), int(m.group(5))] if m.group(4) else None])
    return rows


def records() -> dict:
    from oracle.ref import RefOracle, available
    from tests import cases

    out = {}
    for config in sorted(cases.CONFIGS):
        if not available(config):
            continue
        ref = RefOracle(config)
        items = []
        ins = list(cases.FIXED[cases.family(config)])
        for n in (16, 100, 700):
            ins.append(cases.generated(config, n, 7 + n))
        for d in ins:
            items.append({"input": d.hex(), "record": ref.run_case(d).hex()})
        out[config] = items
    return out


def mode_records() -> dict:
    from oracle.ref import RefOracle, available
    from tests import cases

    out = {}
    for config in cases.MODE_CONFIGS:
        for parts in ("lexer", "parser"):
            name = cases.mode_name(config, parts)
            if not available(name):
                continue
            ref = RefOracle(name)
            if parts == "lexer":
                ins = list(cases.FIXED[cases.family(config)])
                ins += [cases.generated(config, n, 7 + n) for n in (16, 100, 700)]
                ins += [b"\xff", b"\x00 \x7f"]  # bytes no grammar here lexes
            else:
                ins = cases.token_inputs(config, sizes=(16, 100), seeds=(0,))
            out[name] = [{"input": d.hex(), "record": ref.run_case(d).hex()} for d in ins]
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None, help="the reference sources (default: build_ref.reference_dir())")
    a = ap.parse_args(argv)
    if a.reference is None:
        from oracle.build_ref import reference_dir
        a.reference = reference_dir()
        if a.reference is None:
            raise SystemExit("the reference sources are not present (set ALPACC_REFERENCE)")
    ka = known_answers(a.reference)
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(ka, f, indent=1, sort_keys=True)
    rec = records()
    with open(os.path.join(HERE, "records.json"), "w") as f:
        json.dump(rec, f, indent=1, sort_keys=True)
    modes = mode_records()
    with open(os.path.join(HERE, "records_modes.json"), "w") as f:
        json.dump(modes, f, indent=1, sort_keys=True)
    print("known answers:", sorted(ka), "records:", {k: len(v) for k, v in rec.items()},
          "mode records:", {k: len(v) for k, v in modes.items()})


if __name__ == "__main__":
    main()
