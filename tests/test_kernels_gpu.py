"""Per-kernel parity on the GPU: every launcher of libtti_b200.so against the
C oracle, against the reference's own kernels (oracle/_ref, when built) and
against the committed golden vectors of those reference kernels."""
import os

import numpy as np
import pytest

from oracle import REF_LIB_PATH
from tests.golden.make_golden import CASES, oracle_outputs, product_outputs, reference_outputs
from tests.helpers import rel_l2

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_kernels.npz")
IDS = [c["name"] for c in CASES]


def tol(case):
    # one kernel: FP32 rounding only; 24 forward + 24 adjoint steps: accumulated
    return 2e-5 if case["name"] == "steps" else 2e-6


def _compare(got, want, t):
    assert set(want) <= set(got)
    for k in want:
        assert np.all(np.isfinite(got[k])), k
        err = rel_l2(got[k], want[k])
        assert err < t, (k, err)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_product_kernels_match_oracle(case):
    _compare(product_outputs(case), oracle_outputs(case), tol(case))


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(REF_LIB_PATH), reason="reference kernels not built")
@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_product_kernels_match_reference_kernels(case):
    _compare(product_outputs(case), reference_outputs(case), tol(case))


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(GOLDEN), reason="golden vectors not generated yet")
@pytest.mark.parametrize("case", CASES, ids=IDS)
def test_product_kernels_match_golden(case):
    gold = np.load(GOLDEN)
    want = {k.split("/", 1)[1]: gold[k] for k in gold.files if k.startswith(case["name"] + "/")}
    _compare(product_outputs(case), want, tol(case))
