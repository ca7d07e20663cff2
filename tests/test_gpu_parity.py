"""GPU path vs the reference C backend (oracle/_ref), byte for byte.

Every case compares the response record of ``run_case`` (valid byte, tokens,
spans, production tree, parents, token parents) from the CUDA path, called
through the C ABI, with the record the reference's own C program writes for
the same tables and input.
"""

import pytest

from oracle.ref import RefOracle, available
from tests import cases

pytestmark = pytest.mark.gpu

_PARSERS = {}


def parser(config):
    from alpacc_b200.native import Parser
    if config not in _PARSERS:
        _PARSERS[config] = Parser(cases.tables(config))
    return _PARSERS[config]


def check(config, data):
    ref = RefOracle(config).run_case(data)
    got = parser(config).run_case(data)
    assert got == ref, "mismatch for %r (len %d): ref valid=%d got valid=%d" % (
        data[:60], len(data), ref[0], got[0])


@pytest.mark.parametrize("config", sorted(cases.CONFIGS))
def test_parity_cases(gpu, config):
    if not available(config):
        pytest.skip("oracle/_ref/%s not built" % config)
    for data in cases.case_inputs(config):
        check(config, data)


GOLDEN = None


def golden():
    global GOLDEN
    if GOLDEN is None:
        import json
        import os
        GOLDEN = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "records.json")))
    return GOLDEN


@pytest.mark.parametrize("config", sorted(cases.CONFIGS))
def test_parity_golden_records(gpu, config):
    """Committed records of the reference's C backend (travel without oracle/_ref)."""
    items = golden().get(config, [])
    for it in items:
        data = bytes.fromhex(it["input"])
        assert parser(config).run_case(data).hex() == it["record"], data[:60]


@pytest.mark.parametrize("config,n", [("json_ext_i32", 8 << 20), ("json_ext_i64", 3 << 20),
                                      ("sexp_i64", 4 << 20), ("arithmetic_i32", 2 << 20),
                                      ("json_ext_i32", 40 << 20)])
def test_parity_large_vs_port(gpu, config, n):
    """Multi-tile inputs (thousands of lexer tiles, deep nesting; 40 MiB spans
    three host-to-device pieces) against the C restatement oracle."""
    from oracle.port import PortOracle
    data = cases.generated(config, n, 99)
    if config.startswith("sexp"):
        from alpacc_b200 import workloads as W
        data = W.sexp_doc(n, 99, max_depth=3000)
    want = PortOracle(cases.tables(config)).run_case(data)
    got = parser(config).run_case(data)
    assert got[0] == want[0] and got == want


def test_reject_unbalanced_sexp(gpu):
    from alpacc_b200 import workloads as W
    data = W.sexp_doc(1 << 20, 5, unbalanced_frac=0.05, max_depth=500)
    assert parser("sexp_i64").run_case(data) == b"\x00"


def test_repeated_calls_reuse_scratch(gpu):
    """The same handle parses inputs of decreasing and increasing size."""
    from oracle.port import PortOracle
    po = PortOracle(cases.tables("json_ext_i32"))
    for n in (1 << 20, 1000, 3 << 20, 17):
        data = cases.generated("json_ext_i32", n, n)
        assert parser("json_ext_i32").run_case(data) == po.run_case(data)
