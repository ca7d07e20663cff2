"""Build recipe for the reference's own CUDA backend (a baseline, not the product).

TEST AND MEASUREMENT INFRASTRUCTURE ONLY. Assembles the program alpacc's CUDA
emitter would generate for a grammar in combined mode
(src/Alpacc/Generator/Cuda/Generator.hs:94-135, ``Both`` case) from

* the constant sections, restated here from the generated tables
  (Cuda/Generator.hs:24-92 terminal enum, index/length aliases and device
  constants; Cuda/Lexer.hs:22-70 the lexer constants; Cuda/Parser.hs:27-105
  the parser constants and the 16-byte ``HashRecord`` table), and
* the reference's CUDA templates, read where they lie:
  ``backends/cuda/{common,scan,lexer,pse,parser,cli}.cu``,

and compiles it with nvcc for sm_100a into ``oracle/_ref/cuda_<config>``.
That program speaks the wire protocol and has the reference's own
``--benchmark N --warmup W`` timing mode (backends/cuda/cli.cu:877-1060),
which is how the "existing Blackwell-capable kernel" is timed beside this
repository's kernels. Nothing from the reference is written outside
``oracle/_ref/`` (git-ignored).

Usage: python oracle/build_ref_cuda.py [--reference DIR] [config ...]
(the reference sources' location as in build_ref.py: ``reference_dir()``)
"""

from __future__ import annotations

import argparse
import hashlib
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_ref")
sys.path.insert(0, REPO)

from oracle.build_ref import CONFIGS, reference_dir  # noqa: E402

# B200: opt-in shared memory per block and the SM architecture number, the
# values the emitter bakes in after probing the device (Cuda/Generator.hs:70-92)
SHARED_MEMORY = 232448
SM_ARCH = 100


def _u(bits: int) -> str:
    return "uint%d_t" % bits


def _list(xs) -> str:
    return "{" + ", ".join(xs) + "}"


def _ints(a) -> str:
    return _list([str(int(x)) for x in np.asarray(a).reshape(-1)])


def _bools(a) -> str:
    return _list(["true" if bool(x) else "false" for x in np.asarray(a).reshape(-1)])


def terminals_section(t) -> str:
    """``generateTerminals`` (Cuda/Generator.hs:24-39)."""
    return "\n".join([
        "#ifndef ALPACC_TERMINAL_T",
        "#define ALPACC_TERMINAL_T %s" % _u(t.terminal_bits),
        "#endif",
        "enum terminal_t : ALPACC_TERMINAL_T {%s};" % ",".join(t.terminal_names),
    ]) + "\n"


def index_section(t) -> str:
    """``indexTypeAlias`` (Cuda/Generator.hs:41-66), with the length type
    written out (the generated tables carry its width)."""
    lines = (["#define INDEX32"] if t.index32 else []) + [
        "#ifndef ALPACC_INDEX_T", "#ifdef INDEX32", "using index_t = int32_t;", "#else",
        "using index_t = int64_t;", "#endif", "#else", "using index_t = ALPACC_INDEX_T;", "#endif",
        "#ifndef ALPACC_LENGTH_T", "using length_t = %s;" % _u(t.length_bits), "#else",
        "using length_t = ALPACC_LENGTH_T;", "#endif",
    ]
    return "\n".join(lines) + "\n"


def device_section() -> str:
    return "\n".join([
        "#ifndef ALPACC_SHARED_MEMORY", "#define ALPACC_SHARED_MEMORY %d" % SHARED_MEMORY, "#endif",
        "#ifndef ALPACC_SM_ARCH", "#define ALPACC_SM_ARCH %d" % SM_ARCH, "#endif",
    ]) + "\n"


def lexer_section(t) -> str:
    """The constants of ``generateLexer`` (Cuda/Lexer.hs:22-70)."""
    L = t.lexer
    ign = "#define IGNORE_TOKEN %d" % t.ignore_token if t.ignore_token is not None else ""
    return "\n".join([
        "using state_t = %s;" % _u(L.state_bits),
        "using endo_t = state_t;",
        "const size_t NUM_STATES     = %d;" % L.num_states,
        "const size_t NUM_TRANS      = 256;",
        "const state_t ENDO_MASK     = %d;" % L.index_mask,
        "const state_t ENDO_OFFSET   = %d;" % L.index_offset,
        "const state_t TERMINAL_MASK = %d;" % L.token_mask,
        "const state_t TERMINAL_OFFSET = %d;" % L.token_offset,
        "const state_t PRODUCE_MASK  = %d;" % L.produce_mask,
        "const state_t PRODUCE_OFFSET = %d;" % L.produce_offset,
        "const state_t IDENTITY      = %d;" % L.identity,
        ign,
        "const state_t h_to_state[NUM_TRANS] =",
        "  %s;" % _ints(L.to_state),
        "",
        "const state_t h_compose[NUM_STATES * NUM_STATES] =",
        "  %s;" % _ints(L.compose),
        "",
        "const bool h_accept[NUM_STATES] =",
        "  %s;" % _bools(L.accept),
    ]) + "\n"


def parser_section(t) -> str:
    """The constants of ``generateParser`` (Cuda/Parser.hs:27-105): spans
    narrowed to u16 when both tables are shorter than 65535 (the all-ones value
    marks an empty slot)."""
    fits16 = len(t.stacks) < 65535 and len(t.productions) < 65535
    span_bits, none = (16, 65535) if fits16 else (32, 4294967295)
    recs = []
    for v, key, (ss, se), (ps, pe) in zip(t.ht_valid, t.ht_keys, t.ht_stack_span, t.ht_prod_span):
        if v:
            keys = _list(["(terminal_t) %d" % int(k) for k in key])
            recs.append("{%s, %d, %d, %d, %d}" % (keys, ss, se, ps, pe))
        else:
            keys = _list(["(terminal_t) 0"] * len(key))
            recs.append("{%s, %d, %d, %d, %d}" % (keys, none, none, none, none))
    return "\n".join([
        "using production_t = %s;" % _u(t.production_bits),
        "using bracket_t = %s;" % _u(t.bracket_bits),
        "const int64_t Q = %d;" % t.q,
        "const int64_t K = %d;" % t.k,
        "const terminal_t EMPTY_TERMINAL = (terminal_t) %d;" % t.empty_terminal,
        "const terminal_t START_TERMINAL = (terminal_t) %d;" % t.start_terminal,
        "const terminal_t END_TERMINAL = (terminal_t) %d;" % t.end_terminal,
        "const int64_t NUMBER_OF_PRODUCTIONS = %d;" % t.num_productions,
        "__device__ const bool PRODUCTION_TO_TERMINAL_IS_VALID[NUMBER_OF_PRODUCTIONS] =",
        "  %s;" % _bools(t.prod_is_terminal),
        "__device__ const uint8_t PRODUCTION_TO_ARITY[NUMBER_OF_PRODUCTIONS] =",
        "  %s;" % _ints(t.arity),
        "const int64_t HASH_TABLE_SIZE = %d;" % t.hash_size,
        "const int64_t MAX_ITERS = %d;" % t.max_iters,
        "const int64_t PRODUCTIONS_SIZE = %d;" % len(t.productions),
        "const int64_t STACKS_SIZE = %d;" % len(t.stacks),
        "const int64_t MAX_BRACKETS_PER_POSITION = %d;" % t.max_brackets_per_pos,
        "const int64_t MAX_PRODS_PER_POSITION = %d;" % t.max_prods_per_pos,
        "__device__ const bracket_t STACKS[STACKS_SIZE] =",
        "  %s;" % _ints(t.stacks),
        "__device__ const production_t PRODUCTIONS[PRODUCTIONS_SIZE] =",
        "  %s;" % _ints(t.productions),
        "using span_t = %s;" % _u(span_bits),
        "struct alignas(16) HashRecord {",
        "    terminal_t key[Q + K];",
        "    span_t ss, se, ps, pe;",
        "};",
        "__device__ const HashRecord HASH_TABLE[HASH_TABLE_SIZE] =",
        "  %s;" % _list(recs),
    ]) + "\n"


def assemble(reference: str, t) -> str:
    def rd(p):
        with open(os.path.join(reference, p), "r", encoding="utf-8") as f:
            return f.read()

    parts = [
        "// alpacc CUDA backend (reference templates) for grammar %s" % t.name,
        "#define HAS_LEXER", "#define HAS_PARSER", "#define HAS_RAW_INPUT",
        device_section(),
        rd("backends/cuda/common.cu"), rd("backends/cuda/scan.cu"),
        index_section(t),
        terminals_section(t),
        lexer_section(t), rd("backends/cuda/lexer.cu"),
        rd("backends/cuda/pse.cu"), parser_section(t), rd("backends/cuda/parser.cu"),
        rd("backends/cuda/cli.cu"),
    ]
    return "".join(p + "\n" for p in parts)


def build(config: str, reference: str, force: bool = False) -> str:
    from alpacc_b200.grammar.cache import load_tables

    gfile, index32 = CONFIGS[config]
    os.makedirs(OUT, exist_ok=True)
    name = "cuda_" + config
    src = os.path.join(OUT, name + ".cu")
    exe = os.path.join(OUT, name)
    stamp = os.path.join(OUT, name + ".stamp")
    t = load_tables(os.path.join(REPO, "grammars", gfile), index32=index32)
    text = assemble(reference, t)
    key = hashlib.sha256(text.encode()).hexdigest()[:16]
    if not force and os.path.exists(exe) and os.path.exists(stamp) and open(stamp).read().strip() == key:
        return exe
    with open(src, "w", encoding="utf-8") as f:
        f.write(text)
    subprocess.check_call(["nvcc", "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                           "-o", exe, src])
    with open(stamp, "w") as f:
        f.write(key)
    return exe


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("configs", nargs="*", default=["json_i32"])
    a = ap.parse_args(argv)
    a.reference = a.reference or reference_dir() or ""
    if not os.path.isdir(a.reference):
        print("reference sources not present; not built")
        return 0
    for c in a.configs:
        print("building", c, "->", build(c, a.reference, a.force))
    return 0


if __name__ == "__main__":
    sys.exit(main())
