"""GPU decoder against the golden fixtures recorded from the reference's own kernels.

tests/golden/reference_decoder.json holds SHA-256 digests of what the
reference kernels (built unmodified from the reference sources, run on a
B200 by tests/golden/make_golden.py) returned for deterministic inputs: hard
decisions, final APP and final messages in the reference's device layouts.
The sm_100a decoder must reproduce every digest, for every frame packing.
"""
import json
import os

import pytest

from gpu_helpers import gpu_decode, sha, table
import llr_gen

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(__file__), "golden", "reference_decoder.json")


def _cases():
    if not os.path.exists(FIXTURE):
        return []
    return json.load(open(FIXTURE))["cases"]


CASES = _cases()


def _llr(case, n):
    return llr_gen.case_llr(case, n)


@pytest.mark.parametrize("pack", ["SIMD4", "F16X2", "I8"])
def test_gpu_matches_reference_kernels(cuda, pack):
    assert CASES, "golden fixture missing"
    bad, done = [], 0
    for case in CASES:
        code = table(case["code"])
        try:
            out = gpu_decode(code, case["kind"], _llr(case, code.n), case["iters"], case["W"], pack=pack)
        except pytest.skip.Exception:
            continue  # state too large for one CTA with this packing (LDPC_ERR_UNSUPPORTED)
        done += 1
        got = {"hard": sha(out["hard"]), "app": sha(out["app"]), "msg": sha(out["msg"])}
        if got != case["sha256"]:
            bad.append((case["code"], case["kind"], case["iters"], case["input"]["type"],
                        [k for k in got if got[k] != case["sha256"][k]]))
    assert not bad, "%d of %d cases differ from the reference: %s" % (len(bad), done, bad[:10])
    assert done >= len(CASES) * 3 // 4
