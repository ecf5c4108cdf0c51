"""Parity of the fused solver (mmx_*), the GPU demag kernel and the C++
driver over the drop-in ABI with the CPU oracle and, where its library was
built, with the reference's own libgpukern on identical inputs."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
from conftest import REF_LIB

pytestmark = pytest.mark.gpu


def P(t):
    return ctypes.c_void_p(t.data_ptr())


# internal sizes, internal cell sizes, periodic flags
KERNEL_CASES = [
    ((1, 8, 16), (0.7, 0.6, 0.6), (0, 0, 0)),
    ((4, 6, 8), (0.8, 0.9, 1.1), (0, 0, 0)),
    ((2, 4, 6), (1.0, 1.0, 1.0), (0, 1, 0)),
]


@pytest.mark.parametrize("N,cs,per", KERNEL_CASES)
def test_face_kernel_bitexact(eng, cuda, N, cs, per):
    """GPU FaceKernel6 + Exch6 == the oracle's float32 restatement of
    demag.go:26-84 / exchange.go:44-71, bit for bit."""
    Pd = tuple(2 * n if (n > 1 and p == 0) else n for n, p in zip(N, per))
    csf = np.array(cs, np.float32)
    ref = O.face_kernel6(Pd, csf, periodic=per)
    O.add_exch6_kernel(Pd, csf, ref)
    out = cuda.zeros((6,) + Pd, device="cuda")
    eng.face_kernel6_device(Pd, per, csf, exch6=True, out_ptr=P(out))
    cuda.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), ref)


def thin_film_like(grid=(32, 16, 1)):
    return dict(grid=grid, cell=(3.90625e-9, 3.90625e-9, 3e-9), msat=8.0e5, aexch=1.3e-11, alpha=0.02,
                bext=(-24.6e-3, 4.3e-3, 0.0))


def anis_cube_like(grid=(16, 16, 8)):
    return dict(grid=grid, cell=(4e-9, 4e-9, 4e-9), msat=1.1e6, aexch=1.5e-11, alpha=0.5, anis=1, k1=5e5,
                axis=(0, 0, 1))


@pytest.mark.parametrize("kind", ["2d", "3d"])
def test_fused_field_vs_oracle(eng, cuda, kind):
    """h = demag + exchange + Zeeman + anisotropy of the fused pipeline vs
    the oracle's FP64 run of the same field evaluation."""
    c = thin_film_like() if kind == "2d" else anis_cube_like()
    m = O.seeded_m(c["grid"], 1, "random")
    ocfg = O.make_cfg(**c, solver="heun", dt=1e-14)
    o64 = O.OracleSim(ocfg, m, bits=64)
    o32 = O.OracleSim(ocfg, m, bits=32)
    mm = o32.m()  # normalised by the oracle as Sim.Run does
    h64 = o64.heff(mm.astype(np.float64))
    h32 = o32.heff(mm)
    s = eng.Solver(eng.mmx_params(**c, solver="heun", dt=1e-14))
    dm = cuda.from_numpy(mm.copy()).cuda()
    dh = cuda.zeros_like(dm)
    s.field(P(dm), P(dh))
    cuda.cuda.synchronize()
    h = dh.cpu().numpy()
    scale = np.abs(h64).max()
    err_gpu = np.abs(h - h64).max() / scale
    err_o32 = np.abs(h32 - h64).max() / scale
    assert err_gpu < 2e-6, (err_gpu, err_o32)


def test_driver_heff_vs_oracle(eng, cuda):
    """The Go-driver restatement over the drop-in ABI (primitive path)."""
    c = anis_cube_like((8, 12, 4))
    m = O.seeded_m(c["grid"], 2, "random")
    ocfg = O.make_cfg(**c, solver="heun", dt=1e-14)
    o64 = O.OracleSim(ocfg, m, bits=64)
    o32 = O.OracleSim(ocfg, m, bits=32)
    N = o32.N
    Pd = tuple(2 * n if n > 1 else n for n in N)
    k6 = O.face_kernel6(Pd, o32.internal_params()["cellsize"])
    O.add_exch6_kernel(Pd, o32.internal_params()["cellsize"], k6)
    d = eng.DriverSim(eng.driver_config(**c, solver="heun", dt=1e-14), o32.m(), k6)
    h = d.heff(o32.m())
    h64 = o64.heff(o32.m().astype(np.float64))
    assert np.abs(h - h64).max() / np.abs(h64).max() < 2e-6


@pytest.mark.parametrize("solver,steps", [("heun", 20), ("rk23", 8), ("rk4", 8)])
def test_fused_steps_vs_oracle(eng, cuda, solver, steps):
    c = thin_film_like((32, 8, 1)) if solver != "rk4" else anis_cube_like((8, 8, 4))
    kw = dict(solver=solver, dt=1e-14 if solver != "rk23" else 0.0, maxerror=1e-5 if solver == "rk23" else 0.0)
    m = O.seeded_m(c["grid"], 3, "tilted")
    o = O.OracleSim(O.make_cfg(**c, **kw), m, bits=64)
    s = eng.Solver(eng.mmx_params(**c, **kw))
    s.set_m(m)
    s.normalize()
    o.steps(steps)
    s.step(steps)
    dm = np.abs(s.get_m() - o.m()).max()
    assert dm < 1e-5, dm
    st = s.state()
    assert abs(st["time"] - o.time()) <= 1e-6 * abs(o.time())


@pytest.mark.parametrize("grid", [(64, 8, 2), (256, 4, 2)])
def test_fused_heun_two_stage_z_vs_oracle(eng, cuda, grid):
    """Z lines of two equal-radix stages (the user's x = 64 -> 8 x 8 and
    256 -> 16 x 16 complex points after the real-to-complex packing) keep
    their twiddles in [q][k] order in the Z passes: the field and 10 fused
    Heun steps still match the FP64 oracle."""
    c = anis_cube_like(grid)
    kw = dict(solver="heun", dt=1e-14)
    m = O.seeded_m(grid, 6, "random")
    o = O.OracleSim(O.make_cfg(**c, **kw), m, bits=64)
    s = eng.Solver(eng.mmx_params(**c, **kw))
    mm = o.m().astype(np.float32)
    dm = cuda.from_numpy(mm.copy()).cuda()
    dh = cuda.zeros_like(dm)
    s.field(P(dm), P(dh))
    cuda.cuda.synchronize()
    h64 = o.heff(mm.astype(np.float64))
    assert np.abs(dh.cpu().numpy() - h64).max() / np.abs(h64).max() < 2e-6
    s.set_m(mm)
    o.steps(10)
    s.step(10)
    assert np.abs(s.get_m() - o.m()).max() < 1e-5


def test_fused_vs_primitive_heun(eng, cuda):
    """Fused Heun (mmx_solver_step) and the drop-in primitive sequence the Go
    driver issues agree to rounding."""
    c = anis_cube_like((16, 8, 4))
    m = O.seeded_m(c["grid"], 4, "random")
    kw = dict(solver="heun", dt=1e-14)
    o32 = O.OracleSim(O.make_cfg(**c, **kw), m, bits=32)
    N = o32.N
    Pd = tuple(2 * n if n > 1 else n for n in N)
    cs = o32.internal_params()["cellsize"]
    k6 = O.face_kernel6(Pd, cs)
    O.add_exch6_kernel(Pd, cs, k6)
    d = eng.DriverSim(eng.driver_config(**c, **kw), o32.m(), k6)
    s = eng.Solver(eng.mmx_params(**c, **kw))
    s.set_m(o32.m())
    d.steps(30)
    s.step(30)
    assert np.abs(s.get_m() - d.m()).max() < 2e-6


@pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference library not built here")
@pytest.mark.parametrize("kind", ["2d", "3d"])
def test_reference_library_parity(eng, cuda, kind):
    """The reference's own libgpukern (cuFFT path) and the B200 engine, both
    driven by the same Go-driver restatement on identical seeded inputs:
    max |dm| per cell after a fixed-dt run."""
    c = thin_film_like((64, 16, 1)) if kind == "2d" else anis_cube_like((16, 16, 8))
    kw = dict(solver="heun", dt=1e-14 if kind == "3d" else 2e-13)
    m = O.seeded_m(c["grid"], 5, "tilted" if kind == "2d" else "random")
    o32 = O.OracleSim(O.make_cfg(**c, **kw), m, bits=32)
    N = o32.N
    Pd = tuple(2 * n if n > 1 else n for n in N)
    cs = o32.internal_params()["cellsize"]
    k6 = O.face_kernel6(Pd, cs)
    O.add_exch6_kernel(Pd, cs, k6)
    ref = eng.DriverSim(eng.driver_config(**c, **kw), o32.m(), k6, libpath=REF_LIB)
    mine = eng.DriverSim(eng.driver_config(**c, **kw), o32.m(), k6)
    h_ref = ref.heff(o32.m())
    h_mine = mine.heff(o32.m())
    assert np.abs(h_ref - h_mine).max() / np.abs(h_ref).max() < 5e-6
    ref.steps(100)
    mine.steps(100)
    fused = eng.Solver(eng.mmx_params(**c, **kw))
    fused.set_m(o32.m())
    fused.step(100)
    assert np.abs(ref.m() - mine.m()).max() <= 1e-5
    assert np.abs(ref.m() - fused.get_m()).max() <= 1e-5


def test_rk23_device_controller_matches_host(eng, cuda):
    """The device-side dt controller (graph-replayed trials, no host sync)
    takes the same accepted steps as the host controller of rk.go."""
    cfg = dict(grid=(128, 32, 1), cell=(3.90625e-9, 3.90625e-9, 3e-9), msat=8.0e5, aexch=1.3e-11, alpha=0.02,
               bext=(-24.6e-3, 4.3e-3, 0.0), solver="rk23", maxerror=1e-5)
    m0 = O.seeded_m(cfg["grid"], 1, "tilted")
    host = eng.Solver(eng.mmx_params(**cfg))
    host.set_m(m0)
    host.normalize()
    host.step(30)
    sh = host.state()
    dev = eng.Solver(eng.mmx_params(**cfg))
    dev.set_m(m0)
    dev.normalize()
    dev.device_control(True)
    sd = dev.state()
    for _ in range(300):
        dev.step(1)
        sd = dev.state()
        if sd["steps"] >= 30:
            break
    assert sd["steps"] == 30
    assert abs(sd["time"] - sh["time"]) <= 1e-9 * sh["time"], (sd["time"], sh["time"])
    assert np.abs(dev.get_m() - host.get_m()).max() < 1e-6
    # and runs on without host synchronisation: many trials, one read-back
    dev.step(200)
    s2 = dev.state()
    assert s2["steps"] > 30 and s2["time"] > sd["time"]
    host.close()
    dev.close()


def test_fused_heun_spectrum_reuse(eng, cuda):
    """Fixed-step Heun runs its inverse-Z epilogue and the next forward Z in
    one pass (the spectrum buffer carries zfwd(m) between steps).  Setting m
    between steps, stepping through the graph or directly, and the primitive
    path all agree."""
    cfg = dict(grid=(32, 16, 8), cell=(4e-9, 4e-9, 4e-9), msat=1.1e6, aexch=1.5e-11, alpha=0.5, anis=1, k1=5e5,
               axis=(0, 0, 1), solver="heun", dt=1e-14)
    m0 = O.seeded_m(cfg["grid"], 2, "random")
    a = eng.Solver(eng.mmx_params(**cfg))
    a.set_m(m0)
    a.normalize()
    a.use_graph(True)
    a.step(4)
    mid = a.get_m()
    a.set_m(mid)  # invalidates the carried spectrum
    a.step(4)
    b = eng.Solver(eng.mmx_params(**cfg))
    b.set_m(m0)
    b.normalize()
    b.step(8)  # direct launches
    assert np.abs(a.get_m() - b.get_m()).max() < 1e-6
    o = O.OracleSim(O.make_cfg(**cfg), m0, bits=64)
    o.steps(8)
    assert np.abs(b.get_m() - o.m()).max() < 1e-5
    a.close()
    b.close()


def test_avg_m_host_pinned_device_vs_oracle(eng, cuda):
    """<m> (mmx_solver_avg_m) into pageable host memory, page-locked host
    memory (written by the reducing kernel itself) and device memory, called
    several times in a row (the accumulators clear themselves), against the
    FP64 oracle's <m> after the same Heun steps."""
    torch = cuda
    c = anis_cube_like((64, 32, 4))
    kw = dict(solver="heun", dt=1e-14)
    m = O.seeded_m(c["grid"], 8, "random")
    o = O.OracleSim(O.make_cfg(**c, **kw), m, bits=64)
    s = eng.Solver(eng.mmx_params(**c, **kw))
    s.set_m(m)
    s.normalize()
    s.step(5)
    o.steps(5)
    ref = o.m().reshape(3, -1).mean(axis=1)
    pinned = torch.zeros((4, 3), dtype=torch.float32).pin_memory()
    dev = torch.zeros((4, 3), dtype=torch.float32, device="cuda")
    got = []
    for k in range(4):
        got.append(s.avg_m())  # pageable: staged copy
        s.avg_m(P(pinned[k]), True)
        s.avg_m(P(dev[k]), False)
    torch.cuda.synchronize()
    got = np.array(got)
    assert np.array_equal(got, pinned.numpy()) and np.array_equal(got, dev.cpu().numpy())
    assert (got == got[0]).all()
    assert np.abs(got[0] - ref).max() < 1e-6, (got[0], ref)
    s.close()


_SYNC_CHILD = r"""
import os, sys, importlib
import numpy as np
sys.path.insert(0, sys.argv[1])
import oracle as O
sys.path.insert(0, os.path.join(sys.argv[1], "tests"))
from test_gpu_solver import anis_cube_like
eng = importlib.import_module("1_b200")
c = anis_cube_like((16, 8, 4))
kw = dict(solver="heun", dt=1e-14)
o32 = O.OracleSim(O.make_cfg(**c, **kw), O.seeded_m(c["grid"], 4, "random"), bits=32)
Pd = tuple(2 * n if n > 1 else n for n in o32.N)
cs = o32.internal_params()["cellsize"]
k6 = O.face_kernel6(Pd, cs)
O.add_exch6_kernel(Pd, cs, k6)
d = eng.DriverSim(eng.driver_config(**c, **kw), o32.m(), k6)
d.steps(10)
np.save(sys.argv[2], d.m())
"""


def test_drop_in_sync_env_gives_identical_results(tmp_path):
    """The drop-in primitives return once queued on the default stream;
    MMX_GPUKERN_SYNC=1 restores a device synchronisation after every
    primitive (the reference's behaviour).  The Go-driver call sequence
    gives the same m bit for bit either way (each run in its own process,
    since the setting is read once)."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = {}
    for flag in ("0", "1"):
        env = dict(os.environ, MMX_GPUKERN_SYNC=flag)
        f = str(tmp_path / ("m%s.npy" % flag))
        r = subprocess.run([sys.executable, "-c", _SYNC_CHILD, root, f], env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        out[flag] = np.load(f)
    assert np.array_equal(out["0"], out["1"])
