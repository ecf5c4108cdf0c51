"""The oracle against golden vectors produced by the reference's own CUDA
library (tests/golden/make_golden.py): field, fixed-dt Heun and adaptive
RK23 runs on a 2D film and a 3D grid.  Tolerances are those of float32
FFTs (the reference's transforms are cuFFT, the oracle's are float64)."""
import json
import os

import numpy as np
import pytest

import oracle as O
from test_golden_cases import CASES_FOR_TESTS

HERE = os.path.dirname(os.path.abspath(__file__))
NPZ = os.path.join(HERE, "golden", "reference_vectors.npz")
META = os.path.join(HERE, "golden", "reference_vectors.json")

pytestmark = pytest.mark.skipif(not os.path.exists(NPZ), reason="golden vectors not generated yet")


@pytest.fixture(scope="module")
def golden():
    return np.load(NPZ), json.load(open(META))


@pytest.mark.parametrize("name", sorted(CASES_FOR_TESTS))
def test_oracle_field_matches_reference(golden, name):
    g, meta = golden
    c = meta["cases"][name]
    cfg = O.make_cfg(**{k: tuple(v) if isinstance(v, list) else v for k, v in c["config"].items()},
                     solver="heun", dt=1e-14)
    m0 = g[name + "/m0"]
    for bits in (32, 64):
        o = O.OracleSim(cfg, m0, bits=bits)
        h = o.heff(m0.astype(np.float64 if bits == 64 else np.float32))
        ref = g[name + "/heff"]
        assert np.abs(h - ref).max() / np.abs(ref).max() < 5e-6, bits


@pytest.mark.parametrize("name", sorted(CASES_FOR_TESTS))
def test_oracle_runs_match_reference(golden, name):
    g, meta = golden
    c = meta["cases"][name]
    conf = {k: tuple(v) if isinstance(v, list) else v for k, v in c["config"].items()}
    m0 = g[name + "/m0"]
    for rname, run in c["runs"].items():
        kw = dict(run["solver"])
        o = O.OracleSim(O.make_cfg(**conf, **kw), m0, bits=64)
        o.steps(run["steps"])
        ref = g["%s/%s/m" % (name, rname)]
        tol = 1e-5 if rname == "heun" else 1e-4
        assert np.abs(o.m() - ref).max() < tol, (name, rname, np.abs(o.m() - ref).max())
        assert abs(o.time() - run["time"]) <= 1e-3 * run["time"], (o.time(), run["time"])
