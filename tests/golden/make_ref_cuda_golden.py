"""Record the reference CUDA engine's probe series as golden fixtures.

Runs rfnetwork/core/src/solver.cu (built from the reference sources by
oracle/ref_cuda.py into oracle/_ref/libref_cuda.so) on the models of
tests/test_ref_cuda.py and stores every probe's recorded series. The CPU
suite (tests/test_oracle_ref_golden.py) pins the oracle to these numbers
without a GPU.

Usage (on a machine with a GPU and the built library):
    python tests/golden/make_ref_cuda_golden.py [output.npz]
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

sys.path.insert(0, str(HERE.parent))
from test_ref_cuda import _models, run_reference_cuda  # noqa: E402


def main():
    out = Path(sys.argv[1]) if len(sys.argv) > 1 else HERE / "ref_cuda_probes.npz"
    data = {}
    for name, s in _models().items():
        data[name] = run_reference_cuda(s).astype(np.float32)
        print(name, data[name].shape, float(np.abs(data[name]).max()))
    out.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(out, **data)
    print("wrote", out)


if __name__ == "__main__":
    main()
