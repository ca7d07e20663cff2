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


MODE_RECORDS = json.load(open(os.path.join(HERE, "golden", "records_modes.json")))


def _mode_of(name):
    for parts in ("lexer", "parser"):
        if name.endswith("_" + parts):
            return name[: -len(parts) - 1], parts
    raise ValueError(name)


@pytest.mark.parametrize("name", sorted(MODE_RECORDS))
def test_port_modes_match_golden_records(name):
    """Lexer-mode and parser-mode records of the reference's programs."""
    config, parts = _mode_of(name)
    po = PortOracle(cases.tables(config, parts))
    for item in MODE_RECORDS[name]:
        data = bytes.fromhex(item["input"])
        assert po.run_case(data).hex() == item["record"], data[:60]


@pytest.mark.parametrize("parts", ["lexer", "parser"])
@pytest.mark.parametrize("config", cases.MODE_CONFIGS)
def test_port_modes_match_reference_c(config, parts):
    name = cases.mode_name(config, parts)
    if not available(name):
        pytest.skip("oracle/_ref not built")
    po = PortOracle(cases.tables(config, parts))
    ro = RefOracle(name)
    ins = (cases.case_inputs(config, sizes=(1, 64, 1000, 20000), seeds=(0,)) if parts == "lexer"
           else cases.token_inputs(config))
    valid = 0
    for data in ins:
        rec = po.run_case(data)
        assert rec == ro.run_case(data), data[:60]
        valid += rec[0]
    assert 0 < valid < len(ins)  # both accepts and rejects


def test_mode_records_cover_accept_and_reject():
    for name, items in MODE_RECORDS.items():
        valid = [bytes.fromhex(i["record"])[0] for i in items]
        assert 1 in valid and 0 in valid, name


def test_lexer_mode_numbers_terminals_in_order():
    """The lexer-mode program numbers the lexer's terminals in sorted order
    (ignore, then the dead token last); the combined program in declaration
    order. json.alp declares string before number, so the two differ."""
    both, lex = cases.tables("json_i32"), cases.tables("json_i32", "lexer")
    assert both.terminal_names[:2] == ["string", "number"]
    assert lex.terminal_names[:2] == ["number", "string"]
    assert lex.ignore_token == lex.dead_token - 1


def test_reference_cuda_backend_builds():
    """The reference's CUDA backend (the baseline kernels) assembles with the
    restated constants and compiles for sm_100a; its --layout, printed before
    any device call, agrees with the C program's type sizes."""
    import shutil
    import subprocess
    from oracle.build_ref import reference_dir
    if reference_dir() is None or shutil.which("nvcc") is None:
        pytest.skip("reference sources or nvcc not present")
    from oracle.build_ref_cuda import build
    exe = build("json_i32", reference_dir())
    out = subprocess.run([exe, "--layout"], capture_output=True, text=True, timeout=60).stdout
    assert out.startswith("terminal_t=1\nproduction_t=1\nindex_t=4\n"), out
