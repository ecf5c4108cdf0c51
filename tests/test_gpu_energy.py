"""Energy: the drop-in energy-density primitives against the FP32 oracle
(bit for bit) and against the reference's own library, and the fused
solver's total energy against the FP64 oracle and the reference library
driven by the Go-driver restatement (calcHeffEnergy + sumEdens,
src/go/sim/field.go:64-71, energy.go:38-52)."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O
from conftest import REF_LIB

pytestmark = pytest.mark.gpu
need_ref = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference library not built here")


def P(t):
    return ctypes.c_void_p(t.data_ptr())


def fa(*v):
    return (ctypes.c_float * len(v))(*[float(x) for x in v])


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def ulps(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return int(np.abs(a - b).max())


@pytest.fixture(scope="module")
def ref_lib():
    if not os.path.exists(REF_LIB):
        pytest.skip("reference library not built here")
    L = ctypes.CDLL(REF_LIB)
    L.gpu_scale_dot_product.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_float, ctypes.c_int]
    L.gpu_add_local_fields_H_and_phi.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int] + [ctypes.c_void_p] * 2 + \
        [ctypes.c_int] + [ctypes.c_void_p] * 2
    return L


def case(n, seed):
    g = np.random.default_rng(seed)
    m = O.normalize(g.standard_normal((3, n)).astype(np.float32))
    h = (g.standard_normal((3, n)) * 2).astype(np.float32)
    return m, h


def test_scale_dot_product_bitexact(eng, cuda):
    L = eng.lib()
    n = 7001
    m, h = case(n, 11)
    phi = cuda.zeros(n, device="cuda")
    dm, dh = dev(cuda, m), dev(cuda, h)
    L.gpu_scale_dot_product(P(phi), P(dm), P(dh), np.float32(-0.5), n)
    assert np.array_equal(phi.cpu().numpy(), O.scale_dot_product(m, h, np.float32(-0.5)))


@pytest.mark.parametrize("anis", [0, 1])
def test_local_fields_phi_bitexact(eng, cuda, anis):
    L = eng.lib()
    n = 6007
    m, h = case(n, 12)
    phi0 = O.scale_dot_product(m, h, np.float32(-0.5))
    hext = np.array([-0.0244, 0.0043, 0.011], np.float32)
    K, u = np.float32(0.63), np.array([0.6, 0.0, 0.8], np.float32)
    dm, dh, dp = dev(cuda, m), dev(cuda, h), dev(cuda, phi0)
    L.gpu_add_local_fields_H_and_phi(P(dm), P(dh), P(dp), n, fa(*hext), None, anis, fa(K, 0, 0), fa(*u))
    h_ref, phi_ref = O.add_local_fields_phi(m, h, phi0, hext, anis, K, u)
    assert np.array_equal(dh.cpu().numpy(), h_ref)
    assert np.array_equal(dp.cpu().numpy(), phi_ref)


@pytest.mark.parametrize("anis", [0, 1])
def test_energy_primitives_vs_reference_library(eng, cuda, ref_lib, anis):
    """The same symbols of the reference's libgpukern (compiled with fast
    math, so products may fuse into FMAs) on identical inputs: within 4 ulp
    of the value, or 1e-6 of the largest |phi| where terms cancel."""
    L = eng.lib()
    n = 5003
    m, h = case(n, 13)
    hext = fa(0.02, -0.01, 0.005)
    K, u = fa(0.7, 0, 0), fa(0.0, 0.6, 0.8)
    outs = []
    for lib in (L, ref_lib):
        dm, dh = dev(cuda, m), dev(cuda, h)
        dp = cuda.zeros(n, device="cuda")
        lib.gpu_scale_dot_product(P(dp), P(dm), P(dh), ctypes.c_float(-0.5), n)
        lib.gpu_add_local_fields_H_and_phi(P(dm), P(dh), P(dp), n, hext, None, anis, K, u)
        cuda.cuda.synchronize()
        outs.append((dh.cpu().numpy(), dp.cpu().numpy()))
    (h1, p1), (h2, p2) = outs
    # per value: within 4 ulp, or within 1e-6 of the largest magnitude
    # where terms cancel (fused multiply-adds round differently near zero)
    for a, b in ((h1, h2), (p1, p2)):
        ia = a.view(np.int32).astype(np.int64)
        ib = b.view(np.int32).astype(np.int64)
        ok = (np.abs(ia - ib) <= 4) | (np.abs(a - b) <= 1e-6 * np.abs(b).max())
        assert np.all(ok)


FILM = dict(grid=(64, 16, 1), cell=(3.90625e-9, 3.90625e-9, 3e-9), msat=8.0e5, aexch=1.3e-11, alpha=0.02,
            bext=(-24.6e-3, 4.3e-3, 0.0))
CUBE = dict(grid=(16, 16, 8), cell=(4e-9, 4e-9, 4e-9), msat=1.1e6, aexch=1.5e-11, alpha=0.5, anis=1, k1=5e5,
            axis=(0, 0, 1), bext=(0.0, 0.01, 0.02))


@pytest.mark.parametrize("kind", ["2d", "3d"])
def test_fused_energy_vs_fp64_oracle(eng, cuda, kind):
    c = FILM if kind == "2d" else CUBE
    for mode, seed in (("tilted", 1), ("random", 2)):
        m = O.seeded_m(c["grid"], seed, mode)
        o64 = O.OracleSim(O.make_cfg(**c, solver="heun", dt=1e-14), m, bits=64)
        o32 = O.OracleSim(O.make_cfg(**c, solver="heun", dt=1e-14), m, bits=32)
        mm = o32.m()
        e64 = o64.energy(mm.astype(np.float64))
        e32 = o32.energy(mm)
        s = eng.Solver(eng.mmx_params(**c, solver="heun", dt=1e-14))
        s.set_m(mm)
        e = s.energy()
        s.close()
        print("\n%s %s: energy fused %.9g, FP64 oracle %.9g, FP32 oracle %.9g" % (kind, mode, e, e64, e32))
        # per-cell terms are float32: compare with the sum of their magnitudes
        assert abs(e - e64) <= 2e-6 * max(abs(e64), 1.0) * 8


@need_ref
@pytest.mark.parametrize("kind", ["2d", "3d"])
def test_energy_reference_library_vs_fused(eng, cuda, kind):
    """calcHeffEnergy through the driver restatement on the reference's own
    library and on this library's drop-in primitives, and the fused
    solver's energy, on the same m."""
    c = FILM if kind == "2d" else CUBE
    m = O.seeded_m(c["grid"], 3, "random")
    o32 = O.OracleSim(O.make_cfg(**c, solver="heun", dt=1e-14), m, bits=32)
    mm = o32.m()
    cs = o32.internal_params()["cellsize"]
    N = o32.N
    Pd = tuple(2 * n if n > 1 else n for n in N)
    k6 = O.face_kernel6(Pd, cs)
    O.add_exch6_kernel(Pd, cs, k6)
    ref = eng.DriverSim(eng.driver_config(**c, solver="heun", dt=1e-14), mm, k6, libpath=REF_LIB)
    mine = eng.DriverSim(eng.driver_config(**c, solver="heun", dt=1e-14), mm, k6)
    e_ref, e_mine = ref.energy(mm), mine.energy(mm)
    s = eng.Solver(eng.mmx_params(**c, solver="heun", dt=1e-14))
    s.set_m(mm)
    e_f = s.energy()
    s.close()
    e32 = o32.energy(mm)
    print("\n%s: energy reference library %.9g, drop-in %.9g, fused %.9g, FP32 oracle %.9g" %
          (kind, e_ref, e_mine, e_f, e32))
    assert abs(e_mine - e_ref) <= 1e-5 * abs(e_ref)
    assert abs(e_f - e_ref) <= 1e-5 * abs(e_ref)
    assert abs(e32 - e_ref) <= 1e-5 * abs(e_ref)
