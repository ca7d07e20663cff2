"""The C restatement oracle (oracle/oracle.c) pinned to the reference.

* against the committed golden records written by the reference's C backend
  (tests/golden/records.json), for every grammar configuration;
* against the reference's C backend itself (oracle/_ref) on the shared case
  families, when that library has been built here.
"""

import json
import os

import pytest

from oracle.port import PortOracle
from oracle.ref import RefOracle, available
from tests import cases

HERE = os.path.dirname(os.path.abspath(__file__))
RECORDS = json.load(open(os.path.join(HERE, "golden", "records.json")))


@pytest.mark.parametrize("config", sorted(RECORDS))
def test_port_matches_golden_records(config):
    po = PortOracle(cases.tables(config))
    for item in RECORDS[config]:
        data = bytes.fromhex(item["input"])
        assert po.run_case(data).hex() == item["record"], data[:60]


@pytest.mark.parametrize("config", sorted(cases.CONFIGS))
def test_port_matches_reference_c(config):
    if not available(config):
        pytest.skip("oracle/_ref not built")
    po = PortOracle(cases.tables(config))
    ro = RefOracle(config)
    for data in cases.case_inputs(config, sizes=(1, 64, 1000, 20000), seeds=(0,)):
        assert po.run_case(data) == ro.run_case(data), data[:60]


def test_golden_records_cover_accept_and_reject():
    for config, items in RECORDS.items():
        valid = [bytes.fromhex(i["record"])[0] for i in items]
        assert 1 in valid and 0 in valid, config
