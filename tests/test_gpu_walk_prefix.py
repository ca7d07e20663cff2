"""The depth walks' tile prefixes on the GPU, both ways.

By default the walk kernels find their tiles' prefixes by decoupled look-back.
With ALPACC_WALK_PREFIX=pairs (single-document path) the pair kernel instead
adds each element's depth step (and terminal flag) to its walk tile's
aggregate as it writes the element, walk_prefix_kernel scans them, and the
walk kernels read their prefixes. Both must give records byte-identical to the reference's C
backend (oracle/_ref), on inputs spanning many walk tiles, deep nesting and
rejects.
"""

import pytest

from oracle.ref import RefOracle, available
from tests import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["lookback", "pairs"])
@pytest.mark.parametrize("config", ["json_ext_i32", "sexp_i64", "arithmetic_i64"])
def test_walk_prefix_modes(gpu, config, mode, monkeypatch):
    from alpacc_b200 import workloads as W
    from alpacc_b200.native import Parser
    if mode == "pairs":
        monkeypatch.setenv("ALPACC_WALK_PREFIX", "pairs")
    if not available(config):
        pytest.skip("oracle/_ref/lib%s.so is not built" % config)
    ref = RefOracle(config)
    p = Parser(cases.tables(config))
    try:
        extra = []
        if config.startswith("json"):
            extra = [W.json_doc(3 << 20, 41)]
        elif config.startswith("sexp"):
            extra = [W.sexp_doc(3 << 20, 42, max_depth=5000), W.sexp_doc(2 << 20, 43, unbalanced_frac=0.05, max_depth=3000)]
        for data in cases.case_inputs(config)[:40] + extra:
            assert p.run_case(data) == ref.run_case(data), data[:60]
    finally:
        p.close()
