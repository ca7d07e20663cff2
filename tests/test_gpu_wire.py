"""The wire-protocol program on the B200 path against the reference's own
program (oracle/_ref/<config>): batch mode, server mode fed the batch twice
(tests/testc.sh:102-112 of the reference), --layout."""

import os
import subprocess

import pytest

from alpacc_b200 import wire
from oracle.ref import REF_DIR
from tests import cases

pytestmark = pytest.mark.gpu

CONFIGS = ["arithmetic_i64", "sexp_i64"]


def program(config):
    from alpacc_b200.wire_program import build_program
    return build_program(cases.tables(config), config)


def ref_program(config):
    p = os.path.join(REF_DIR, config)
    if not os.path.exists(p):
        pytest.skip("reference program not built")
    return p


def batch(config):
    return wire.encode_batch(cases.case_inputs(config, sizes=(1, 64, 2000), seeds=(0,)))


@pytest.mark.parametrize("config", CONFIGS)
def test_batch_matches_reference_program(gpu, config):
    data = batch(config)
    ref = subprocess.run([ref_program(config)], input=data, capture_output=True, check=True).stdout
    got = subprocess.run([program(config)], input=data, capture_output=True, check=True).stdout
    assert got == ref


@pytest.mark.parametrize("config", CONFIGS)
def test_server_mode_twice(gpu, config):
    data = batch(config)
    single = subprocess.run([program(config)], input=data, capture_output=True, check=True).stdout
    twice = subprocess.run([program(config), "--server"], input=data + data, capture_output=True, check=True).stdout
    assert twice == single + single


@pytest.mark.parametrize("config", CONFIGS)
def test_layout_and_frame_errors(gpu, config):
    lay = subprocess.run([program(config), "--layout"], capture_output=True, check=True).stdout
    ref = subprocess.run([ref_program(config), "--layout"], capture_output=True, check=True).stdout
    assert lay == ref
    bad = (1).to_bytes(8, "little") + (100).to_bytes(8, "little") + b"\x05" * 10
    r = subprocess.run([program(config)], input=bad, capture_output=True)
    assert r.returncode == 1
