"""A longer random-grammar campaign on the CPU (not collected by pytest).

For ``count`` random grammars (tests/random_grammars.py; parameters drawn
per grammar: 2-6 characters, 2-6 terminals, 1-4 nonterminals, 2-8
productions, (q, k) from the reference's matrix) whose tables the restated
generator builds, it checks

* the oracle's combined-mode and lexer-mode records against the reference's
  own C programs built from the same tables (oracle/build_ref.py);
* the lexer machine the GPU loader derives, walked on the CPU
  (tests/native/machine_lex.cpp), against lex_string;
* the dense pair table against lookup_key;

and prints every disagreement with the grammar's text. Needs the reference
sources. Usage: python tests/fuzz_campaign.py [seed] [count]
"""

import ctypes
import os
import subprocess
import sys
import tempfile
import time
import traceback

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)

from alpacc_b200.grammar.tables import GrammarError, generate_parts  # noqa: E402
from oracle.build_ref import build_tables  # noqa: E402
from oracle.port import PortOracle  # noqa: E402
from oracle.ref import RefOracle  # noqa: E402
from tests import test_machine as TM  # noqa: E402
from tests.random_grammars import QKS, RandomGrammar  # noqa: E402

REFERENCE = "/root/reference"


def harness():
    so = os.path.join(tempfile.mkdtemp(), "libmachine_lex.so")
    subprocess.check_call(["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-I",
                           os.path.join(REPO, "alpacc_b200", "csrc"), "-I", os.path.join(REPO, "include"),
                           os.path.join(HERE, "native", "machine_lex.cpp"),
                           os.path.join(REPO, "alpacc_b200", "csrc", "device_tables.cpp"), "-o", so])
    L = ctypes.CDLL(so)
    L.machine_lex.restype = ctypes.c_int
    L.machine_lex.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_uint64, ctypes.c_void_p, ctypes.c_uint64,
                              ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int)]
    L.pair_lookup.restype = ctypes.c_int
    L.pair_lookup.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
    return L


def main(seed: int, count: int) -> int:
    L = harness()
    rng = np.random.default_rng(seed)
    tried = done = bad = 0
    t0 = time.time()
    while done < count:
        gseed = int(rng.integers(0, 10 ** 9))
        q, k = QKS[int(rng.integers(0, len(QKS)))]
        params = dict(num_chars=int(rng.integers(2, 7)), num_terminals=int(rng.integers(2, 7)),
                      num_nonterminals=int(rng.integers(1, 5)), num_productions=int(rng.integers(2, 9)))
        tried += 1
        g = RandomGrammar(gseed, q, k, **params)
        try:
            t = generate_parts(g.text(), "c%d" % gseed, False, "both")
        except GrammarError:
            continue
        done += 1
        name = "c%d" % gseed
        try:
            ins = g.inputs(gseed, exhaustive=3, sentences=(8, 64, 500), noise=(100, 2000))
            for parts, tt in (("both", t), ("lexer", generate_parts(g.text(), name, False, "lexer"))):
                nm = name if parts == "both" else name + "_lexer"
                po, ro = PortOracle(tt), RefOracle(nm, build_tables(tt, nm, REFERENCE))
                for d in ins:
                    if po.run_case(d) != ro.run_case(d):
                        raise AssertionError("%s record differs on %r" % (parts, d[:60]))
                if parts == "lexer":
                    TM._compare(L, tt, ins)
            TM._check_pairs(L, t)
        except Exception:
            bad += 1
            print("DISAGREEMENT", gseed, q, k, params)
            traceback.print_exc()
            print(g.text())
    print("%d grammars of %d drawn, %d disagreements, %.0fs" % (done, tried, bad, time.time() - t0))
    return 1 if bad else 0


if __name__ == "__main__":
    sys.exit(main(int(sys.argv[1]) if len(sys.argv) > 1 else 1, int(sys.argv[2]) if len(sys.argv) > 2 else 100))
