"""Synthetic workload generators produce inputs the reference accepts (and
the unbalanced s-expression variant is rejected)."""

from alpacc_b200 import workloads as W
from oracle.port import PortOracle
from tests import cases


def test_json_doc_exact_size_and_accepted():
    po = PortOracle(cases.tables("json_ext_i32"))
    for n in (2, 100, 5000, 200000):
        d = W.json_doc(n, 11)
        assert len(d) == n
        assert po.run_case(d)[0] == 1


def test_arithmetic_accepted():
    po = PortOracle(cases.tables("arithmetic_i64"))
    for n in (10, 4000, 100000):
        d = W.arithmetic(n, 3)
        assert len(d) == n and po.run_case(d)[0] == 1


def test_sexp_balanced_and_unbalanced():
    po = PortOracle(cases.tables("sexp_i64"))
    d = W.sexp_doc(200000, 3, max_depth=300)
    assert len(d) == 200000 and po.run_case(d)[0] == 1
    bad = W.sexp_doc(200000, 3, unbalanced_frac=0.05, max_depth=300)
    assert po.run_case(bad) == b"\x00"


def test_deterministic():
    assert W.json_doc(10000, 5) == W.json_doc(10000, 5)
    assert W.json_doc(10000, 5) != W.json_doc(10000, 6)
