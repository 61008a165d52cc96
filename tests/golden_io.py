"""Loading of the golden vectors recorded from the reference's own code
(tests/golden/make_golden.py writes them)."""
from __future__ import annotations

import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def names(prefix: str):
    return sorted(os.path.basename(p)[len(prefix) + 1:-4] for p in glob.glob(os.path.join(GOLDEN, prefix + "_*.npz")))


def load(name: str):
    with np.load(os.path.join(GOLDEN, name + ".npz")) as f:
        return {k: f[k] for k in f.files}
