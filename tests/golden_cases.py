"""Loads the golden fixtures (tests/golden/*.npz) made by
tests/golden/make_golden.py from the reference GASAL2 library built for
sm_100a and run on a B200."""
import glob
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

import make_golden  # noqa: E402
from gasal_b200.capi import Batch  # noqa: E402


def cases():
    """Yields (case_name, Params, Batch, {field: expected array}) for every
    launch configuration stored in the fixtures."""
    for f in sorted(glob.glob(os.path.join(HERE, "golden", "*.npz"))):
        name = os.path.basename(f)[:-4]
        z = np.load(f)
        b = Batch.from_arrays({k[4:]: z[k] for k in z.files if k.startswith("in__")})
        for p in make_golden.configs_for(name):
            key = p.key()
            idx = z["idx__" + key]
            sb = b if len(idx) == b.n else b.subset(idx)
            exp = {k.split("__")[2]: z[k] for k in z.files if k.startswith(f"out__{key}__")}
            yield name, p, sb, exp


def case_ids():
    return [f"{n}-{p.key()}" for n, p, _, _ in cases()]
