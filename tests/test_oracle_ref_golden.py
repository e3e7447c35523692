"""The CPU oracle against the reference CUDA engine's recorded probe series.

tests/golden/ref_cuda_probes.npz holds the probe series that the reference's
own rfnetwork/core/src/solver.cu produced for the models of
tests/test_ref_cuda.py (written by tests/golden/make_ref_cuda_golden.py on a
GPU). The oracle restates the reference's CPU engine; both engines must agree
to a relative L2 of 1e-5 (the reference GPU build contracts multiply-adds).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from helpers import rel_l2, run_oracle
from test_ref_cuda import _models

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_cuda_probes.npz"

pytestmark = pytest.mark.skipif(not GOLDEN.exists(), reason="reference CUDA golden fixture not recorded")


@pytest.mark.parametrize("name", ["microstrip", "boxes"])
def test_oracle_matches_reference_cuda_golden(name):
    ref = np.load(GOLDEN)[name]
    _, ora = run_oracle(_models()[name])
    assert ora.shape == ref.shape
    err = rel_l2(ora, ref)
    assert err <= 1e-5, f"{name}: oracle vs reference CUDA relative L2 {err:.3e}"
