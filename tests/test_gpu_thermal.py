"""Thermal field (src/go/sim/temperature.go:21-55): each RK step adds
sigma N(0,1) per cell and component to the field of all its stages,
sigma = sqrt(2 alpha kB T / (gamma0 mu0 Ms V dt)) / Ms, the noise fixed for
the step's trials (rk.go:289-292) and the stage-0 dt bounds skipped
(rk.go:347-348).  The reference draws the numbers with cuRAND; this engine
with a counter-based Philox-4x32-10 stream (cell, step, seed), which the
oracle restates, so a thermal run is compared with the FP64 oracle on the
same noise."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

FILM = dict(grid=(32, 16, 1), cell=(3.90625e-9, 3.90625e-9, 3e-9), msat=8.0e5, aexch=1.3e-11, alpha=0.1,
            solver="rk12", maxerror=1e-4)


@pytest.mark.parametrize("temperature", [300.0, 3000.0])
def test_thermal_rk12_vs_fp64_oracle(eng, cuda, temperature):
    c = dict(FILM, temperature=temperature, thermal_seed=7)
    m0 = O.seeded_m(c["grid"], 1, "tilted")
    o = O.OracleSim(O.make_cfg(**c), m0, bits=64)
    s = eng.Solver(eng.mmx_params(**c))
    s.set_m(m0)
    s.normalize()
    s.step(60)
    o.steps(60)
    st = s.state()
    d = float(np.abs(s.get_m() - o.m()).max())
    cold = O.OracleSim(O.make_cfg(**dict(FILM)), m0, bits=64)
    cold.steps(60)
    d_cold = float(np.abs(o.m() - cold.m()).max())
    print("\nthermal %g K: max|dm| vs FP64 oracle %.3g; the noise moved m by %.3g; time %.6g vs %.6g" %
          (temperature, d, d_cold, st["time"], o.time()))
    s.close()
    assert d_cold > 1e-3  # the field acted
    assert d <= 1e-4
    assert abs(st["time"] - o.time()) <= 1e-3 * o.time()


def test_thermal_noise_depends_on_seed_and_refuses_device_control(eng, cuda):
    m0 = O.seeded_m(FILM["grid"], 2, "tilted")
    out = []
    for seed in (1, 1, 2):
        s = eng.Solver(eng.mmx_params(**dict(FILM, temperature=300.0, thermal_seed=seed)))
        s.set_m(m0)
        s.normalize()
        s.step(10)
        out.append(s.get_m())
        if seed == 2:
            with pytest.raises(eng.MmxError):
                s.device_control(True)
        s.close()
    assert np.array_equal(out[0], out[1])
    assert np.abs(out[0] - out[2]).max() > 1e-5
    with pytest.raises(eng.MmxError):
        eng.Solver(eng.mmx_params(**dict(FILM, solver="heun", maxerror=0.0, dt=1e-14, temperature=300.0)))
