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
