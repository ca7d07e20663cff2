"""The request server (alpacc_server_*): requests submitted concurrently are
coalesced into batches while others are on the GPU; every result must be the
same as parsing that input alone, whatever else was in its batch."""

import threading

import numpy as np
import pytest

from alpacc_b200 import native, wire
from tests import cases

pytestmark = pytest.mark.gpu


def _docs(config, seed):
    rng = np.random.default_rng(seed)
    docs = [cases.generated(config, int(n), seed * 1000 + i)
            for i, n in enumerate(rng.integers(2, 60000, 40))]
    docs += [cases.mutate(d, rng) for d in docs[:10]]
    docs += [b"", cases.generated(config, 300000, seed)] + list(cases.FIXED.get(cases.family(config), []))
    return [docs[i] for i in rng.permutation(len(docs))]


@pytest.mark.parametrize("config", ["json_ext_i32", "sexp_i64"])
def test_server_results_equal_alone(gpu, config):
    tables = cases.tables(config)
    alone = native.Parser(tables, device=0)
    srv = native.Server(tables, device=0, workers=2, budget=1 << 30)
    try:
        docs = _docs(config, 3)
        ids = [None] * len(docs)

        def submit(part):
            for i in part:
                ids[i] = srv.submit(docs[i])

        threads = [threading.Thread(target=submit, args=(range(k, len(docs), 2),)) for k in range(2)]
        for th in threads:
            th.start()
        for th in threads:
            th.join()
        got = [srv.wait(ids[i]) for i in range(len(docs))]
        for d, (r, ms) in zip(docs, got):
            assert ms >= 0
            assert wire.encode_record(r, srv.layout) == alone.run_case(d), d[:60]
        st = srv.stats()
        assert st["served"] == len(docs) and st["batches"] <= len(docs) and st["queued"] == 0
        # the same inputs one at a time: identical results
        for d in docs[:5]:
            r, _ = srv.wait(srv.submit(d))
            assert wire.encode_record(r, srv.layout) == alone.run_case(d)
    finally:
        srv.close()


def test_server_scratch_within_share(gpu):
    """Admission by the batch path's exact scratch: with a share far below
    what all requests together need, batches split and no worker's handle
    ever holds more batch scratch than its share."""
    config = "json_ext_i32"
    tables = cases.tables(config)
    alone = native.Parser(tables, device=0)
    srv = native.Server(tables, device=0, workers=2, budget=96 << 20)
    try:
        rng = np.random.default_rng(11)
        docs = [cases.generated(config, int(n), 500 + i) for i, n in enumerate(rng.integers(20000, 60000, 48))]
        ids = [srv.submit(d) for d in docs]
        got = [srv.wait(i) for i in ids]
        for d, (r, _) in zip(docs, got):
            assert wire.encode_record(r, srv.layout) == alone.run_case(d)
        st = srv.stats()
        assert st["scratch_share"] == 48 << 20
        assert 0 < st["max_scratch_held"] <= st["scratch_share"], st
        assert st["batches"] > 2, st
    finally:
        srv.close()
