"""The batched form: every instance of a mixed-size batch evolves exactly
as the same instance stepping alone (same kernels, same arithmetic), and
RK4 / Heun batches track the FP64 oracle."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def seeded_unit(grid, seed):
    return O.seeded_m(grid, seed, "random")


@pytest.mark.parametrize("solver", ["rk4", "heun"])
def test_batch_equals_alone(eng, cuda, solver):
    cfgs = eng.batch_config(6, seed=4, solver=solver, dt=5e-15)
    # keep the test small: shrink the large instances
    for c in cfgs:
        c["grid"] = tuple(min(g, 64) if i < 2 else g for i, g in enumerate(c["grid"]))
    params = [eng.mmx_params(**c) for c in cfgs]
    ms = [seeded_unit(c["grid"], 100 + i) for i, c in enumerate(cfgs)]
    b = eng.Batch(params)
    for inst, m in zip(b.instances, ms):
        inst.set_m(m)
        inst.normalize()
    b.use_graph(True)
    b.step(5)
    for i, (c, m) in enumerate(zip(cfgs, ms)):
        s = eng.Solver(eng.mmx_params(**c))
        s.set_m(m)
        s.normalize()
        s.step(5)
        alone = s.get_m()
        mixed = b.instances[i].get_m()
        assert np.array_equal(alone, mixed), (i, c["grid"], np.abs(alone - mixed).max())
        s.close()
    b.close()


def test_batch_rk4_vs_oracle(eng, cuda):
    cfgs = eng.batch_config(3, seed=7, solver="rk4", dt=5e-15)
    for c in cfgs:
        c["grid"] = tuple(min(g, 32) if i < 2 else g for i, g in enumerate(c["grid"]))
    b = eng.Batch([eng.mmx_params(**c) for c in cfgs])
    ms = [seeded_unit(c["grid"], 200 + i) for i, c in enumerate(cfgs)]
    for inst, m in zip(b.instances, ms):
        inst.set_m(m)
        inst.normalize()
    b.step(10)
    for i, (c, m) in enumerate(zip(cfgs, ms)):
        o = O.OracleSim(O.make_cfg(**c), m, bits=64)
        o.steps(10)
        assert np.abs(b.instances[i].get_m() - o.m()).max() < 1e-5
    b.close()


def test_autotuner_times_both_column_tiles(eng, cuda):
    cfgs = eng.batch_config(4, seed=9, solver="rk4", dt=5e-15)
    b = eng.Batch([eng.mmx_params(**c) for c in cfgs])
    tune = eng.batch_tuning()
    b.close()
    P1 = {2 * c["grid"][1] for c in cfgs if c["grid"][2] > 1}  # user y -> internal Y, padded (3D instances)
    seen = {(t["L"], t["inverse"]) for t in tune}
    for L in P1:
        assert (L, False) in seen and (L, True) in seen
    for t in tune:
        assert t["ms"][0] > 0 and t["ms"][1] > 0
        assert t["chosen"] in t["widths"]
        faster = t["widths"][1] if t["ms"][1] < t["ms"][0] else t["widths"][0]
        assert t["chosen"] == faster
