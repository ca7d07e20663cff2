"""The launch-geometry autotuner on the GPU.

alpacc_gpu_autotune times a device-resident sample under each candidate
geometry (lexer window 16/24/32 bytes x resident CTAs per SM, then the pair
kernel's and the walks' CTAs per SM), keeps the fastest and caches it per
(grammar digest, device): a handle loaded afterwards for the same tables
starts with that geometry. Whatever the geometry, every record must still
equal the reference's own C backend's.
"""

import pytest

from oracle.ref import RefOracle, available
from tests import cases

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("config", ["json_ext_i32", "sexp_i64"])
def test_autotune_geometry_cached_and_exact(gpu, config):
    import torch

    from alpacc_b200 import workloads as W
    from alpacc_b200.native import Parser

    t = cases.tables(config)
    doc = W.json_doc(8 << 20, 31) if config.startswith("json") else W.sexp_doc(8 << 20, 31)
    p = Parser(t, max_input=len(doc))
    try:
        d = torch.frombuffer(bytearray(doc), dtype=torch.uint8).cuda()
        before = p.run_case(doc)
        p.autotune(d.data_ptr(), len(doc))
        geo = p.geometry()
        assert geo["lex_window_bytes"] in (16, 24, 32) and not geo["from_cache"], geo
        assert min(geo["lex_ctas_per_sm"], geo["pair_ctas_per_sm"], geo["walk_ctas_per_sm"]) >= 1, geo
        assert p.run_case(doc) == before
        q = Parser(t)
        try:
            g2 = q.geometry()
            assert g2["from_cache"] and g2["grammar_digest"] == geo["grammar_digest"], (g2, geo)
            assert all(g2[k] == geo[k] for k in ("lex_window_bytes", "lex_ctas_per_sm", "pair_ctas_per_sm",
                                                 "walk_ctas_per_sm"))
            if available(config):
                ref = RefOracle(config)
                for data in cases.case_inputs(config)[:40]:
                    assert q.run_case(data) == ref.run_case(data), data[:60]
        finally:
            q.close()
    finally:
        p.close()
