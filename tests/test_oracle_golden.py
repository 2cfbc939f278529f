"""Pins the CPU oracle to the reference: the oracle must reproduce, bit for bit,
the outputs the reference's own kernels produced on a B200 (digests in
tests/golden/reference_decoder.json, made by tests/golden/make_golden.py)."""
import json
import os

import numpy as np
import pytest

import llr_gen
from oracle import oracle
from fast_ldpc_decoder_for_gpu_fixed_b200 import load_table

FIXTURE = os.path.join(os.path.dirname(__file__), "golden", "reference_decoder.json")
CASES = json.load(open(FIXTURE))["cases"] if os.path.exists(FIXTURE) else []


def _sha(a):
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def test_fixture_present():
    assert CASES, "tests/golden/reference_decoder.json missing"
    kinds = {c["kind"] for c in CASES}
    assert kinds == {"MS", "OMS", "NMS", "2NMS", "XMS"}


@pytest.mark.parametrize("idx", range(len(CASES)))
def test_oracle_matches_reference(idx):
    case = CASES[idx]
    code = load_table(case["code"])
    inp = case["input"]
    llr = llr_gen.case_llr(case, code.n)
    o = oracle.decode(code, case["kind"], llr, case["iters"], want_state=True)
    got = {"hard": _sha(o["hard"]), "app": _sha(o["app"]), "msg": _sha(o["msg"])}
    assert got == case["sha256"]
