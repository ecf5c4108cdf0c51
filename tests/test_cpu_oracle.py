"""CPU checks of the oracle and of the host-side logic (no GPU needed)."""
import os
import re
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, engine


def test_oracle_fft_matches_numpy():
    for N, Pd in [((2, 6, 10), (4, 12, 20)), ((1, 6, 10), (1, 12, 20)), ((3, 5, 7), (6, 10, 14))]:
        a = np.random.default_rng(0).standard_normal(N)
        pad = np.zeros(Pd)
        pad[:N[0], :N[1], :N[2]] = a
        ref = np.fft.rfftn(pad)
        out = O.fft_forward_padded(N, Pd, a, bits=64)
        c = out[..., 0::2] + 1j * out[..., 1::2]
        assert np.abs(c - ref).max() < 1e-12 * max(1, np.abs(ref).max())
        back = O.fft_inverse_padded(N, Pd, out, bits=64)
        assert np.abs(back / np.prod(Pd) - a).max() < 1e-13


def test_oracle_convolution_matches_direct_sum():
    N, Pd = (3, 4, 5), (6, 8, 10)
    cs = np.array([0.7, 0.9, 1.1])
    k = O.face_kernel6(Pd, cs, bits=64)
    O.add_exch6_kernel(Pd, cs, k, bits=64)
    m = np.random.default_rng(1).standard_normal((3,) + N)
    h = O.convolve(N, cs, m, bits=64)
    KI = [[0, 5, 4], [5, 1, 3], [4, 3, 2]]
    hd = np.zeros_like(m)
    X, Y, Z = np.meshgrid(range(N[0]), range(N[1]), range(N[2]), indexing="ij")
    for x in range(N[0]):
        for y in range(N[1]):
            for z in range(N[2]):
                for d in range(3):
                    for s in range(3):
                        kk = k[KI[s][d]][(x - X) % Pd[0], (y - Y) % Pd[1], (z - Z) % Pd[2]]
                        hd[d, x, y, z] += (kk * m[s]).sum()
    assert np.abs(h - hd).max() < 1e-12 * np.abs(hd).max()


def test_face_kernel_self_term_cube():
    # the self demag factors of a cube are -1/3 each (point-charge faces at
    # accuracy 8 approximate the exact value to a few 1e-3)
    k = O.face_kernel6((4, 4, 4), np.array([1.0, 1.0, 1.0]), bits=64)
    diag = [k[c, 0, 0, 0] for c in range(3)]
    assert np.allclose(diag, diag[0])
    assert abs(diag[0] + 1 / 3) < 5e-3
    # symmetry: K(x) = K(-x) for the diagonal components
    assert abs(k[0, 1, 0, 0] - k[0, 3, 0, 0]) < 1e-12


def test_face_kernel_2d_exchange_centre_overwrite():
    """In 2D (P0 = 1) the +-x exchange writes overwrite the centre value
    (exchange.go:58-65): centre = demag + 1/hx."""
    Pd = (1, 8, 8)
    cs = np.array([0.5, 0.7, 0.7], np.float32)
    k = O.face_kernel6(Pd, cs)
    k0 = k.copy()
    O.add_exch6_kernel(Pd, cs, k)
    hx = np.float32(cs[0] * cs[0])
    assert k[0, 0, 0, 0] == np.float32(k0[0, 0, 0, 0] + np.float32(np.float32(1.0) / hx))
    hy = np.float32(cs[1] * cs[1])
    assert k[0, 0, 1, 0] == np.float32(k0[0, 0, 1, 0] + np.float32(np.float32(1.0) / hy))


def test_units_match_reference_values():
    eng = engine()
    u = eng.units(8.0e5, 1.3e-11)
    assert abs(u["length"] - 5.6858e-9) / 5.6858e-9 < 1e-4
    assert abs(u["time"] - 5.6536e-12) / 5.6536e-12 < 1e-4
    assert abs(u["field"] - 1.00531) < 1e-5
    cfg = O.make_cfg((16, 8, 1), (3.90625e-9, 3.90625e-9, 3e-9), 8e5, 1.3e-11, 0.02, bext=(-24.6e-3, 4.3e-3, 0))
    o = O.OracleSim(cfg, O.seeded_m((16, 8, 1), 1), bits=32)
    assert np.float32(o.unit("length")) == u["length"]
    assert np.float32(o.unit("time")) == u["time"]
    p = eng.mmx_params((16, 8, 1), (3.90625e-9, 3.90625e-9, 3e-9), 8e5, 1.3e-11, 0.02, bext=(-24.6e-3, 4.3e-3, 0))
    ip = o.internal_params()
    assert list(p.cellsize) == [float(x) for x in ip["cellsize"]]
    assert list(p.hext) == [float(x) for x in ip["hext"]]
    # axis swap: user x field lands in internal component Z
    assert p.hext[2] < 0 and p.hext[0] == 0.0


def test_oracle_fp32_tracks_fp64():
    c = dict(grid=(32, 8, 1), cell=(3.90625e-9, 3.90625e-9, 3e-9), msat=8e5, aexch=1.3e-11, alpha=0.02,
             bext=(-24.6e-3, 4.3e-3, 0.0))
    m = O.seeded_m(c["grid"], 1)
    cfg = O.make_cfg(**c, solver="rk23", maxerror=1e-5)
    o32, o64 = O.OracleSim(cfg, m, 32), O.OracleSim(cfg, m, 64)
    o32.steps(20)
    o64.steps(20)
    assert np.abs(o32.m() - o64.m()).max() < 1e-5
    assert abs(o32.time() - o64.time()) / o64.time() < 1e-4


def test_oracle_heun_fixed_step_advances_time():
    c = dict(grid=(8, 8, 4), cell=(4e-9, 4e-9, 4e-9), msat=1.1e6, aexch=1.5e-11, alpha=0.5, anis=1, k1=5e5,
             axis=(0, 0, 1))
    cfg = O.make_cfg(**c, solver="heun", dt=1e-14)
    o = O.OracleSim(cfg, O.seeded_m(c["grid"], 2, "random"), 32)
    o.steps(5)
    assert abs(o.time() - 5 * o.dt()) < 1e-12
    m = o.m()
    assert np.abs((m * m).sum(0) - 1).max() < 1e-6


def test_reference_sum_order():
    a = np.random.default_rng(3).standard_normal(20000).astype(np.float32)
    s = O.ref_sum(a)
    assert abs(s - a.astype(np.float64).sum()) < 1e-3
    assert O.ref_sum(np.ones(1025, np.float32)) == 1025.0


def header_symbols():
    names = []
    for h in ("gpukern.h", "mmx.h"):
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for mm in re.finditer(r"^[A-Za-z_][\w\s\*]*?\b([a-zA-Z_]\w*)\s*\(", txt, flags=re.M):
            name = mm.group(1)
            if name not in ("if", "defined"):
                names.append(name)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = os.path.join(ROOT, "1_b200", "libgpukern.so")
    if not os.path.exists(lib):
        pytest.skip("libgpukern.so not built")
    out = subprocess.check_output(["nm", "-D", "--defined-only", lib]).decode()
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [s for s in header_symbols() if s not in exported]
    assert not missing, missing
    eng = engine()
    for s in eng.exported_symbols():
        assert s in exported


def test_library_loads_without_gpu():
    eng = engine()
    L = eng.lib()
    assert L.gpu_reduce is not None
    D = eng.driver()
    assert D.mmxd_open is not None


def test_driver_exports():
    lib = os.path.join(ROOT, "1_b200", "libmmxdriver.so")
    out = subprocess.check_output(["nm", "-D", "--defined-only", lib]).decode()
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    txt = open(os.path.join(ROOT, "include", "mmx_driver.h")).read()
    for name in re.findall(r"\b(mmxd_\w+)\s*\(", txt):
        assert name in exported, name


def test_energy_zeeman_and_anisotropy_terms():
    """Energy of a uniform state: switching on a field adds -N (m.B) V and a
    uniaxial term adds -1/2 K (m.u)^2 N V (gpu_local_contr3.cu:230-247,
    362-374, energy.go:38-52), in both oracle builds."""
    base = dict(grid=(16, 8, 2), cell=(5e-9, 5e-9, 5e-9), msat=8e5, aexch=1.3e-11, alpha=0.1)
    m = np.zeros((3, 2, 8, 16), np.float32)
    m[2] = 1.0  # internal Z = the user's x
    for bits in (32, 64):
        e0 = O.OracleSim(O.make_cfg(**base), m, bits=bits)
        eb = O.OracleSim(O.make_cfg(**base, bext=(0.05, 0.0, 0.0)), m, bits=bits)
        ek = O.OracleSim(O.make_cfg(**base, anis=1, k1=4e5, axis=(1, 0, 0)), m, bits=bits)
        cs = e0.internal_params()["cellsize"]
        vol = float(cs[0]) * float(cs[1]) * float(cs[2])
        n = 16 * 8 * 2
        hx = 0.05 / e0.unit("field")
        dz = eb.energy() - e0.energy()
        assert abs(dz - (-n * hx * vol)) <= 2e-5 * abs(n * hx * vol)
        K = ek.internal_params()["K"]
        da = ek.energy() - e0.energy()
        assert abs(da - (-0.5 * float(K) * n * vol)) <= 2e-5 * abs(0.5 * float(K) * n * vol)
        # demag self-energy of the uniform state is positive
        assert e0.energy() > 0


def test_run_table_schedule():
    """Sim.Run's table: the first row at t = 0, each later row at the first
    step boundary at or past 'period' after the previous one; a second call
    continues the schedule."""
    c = dict(grid=(32, 8, 1), cell=(3.90625e-9, 3.90625e-9, 3e-9), msat=8e5, aexch=1.3e-11, alpha=0.02,
             bext=(-24.6e-3, 4.3e-3, 0.0), solver="rk23", maxerror=1e-5)
    o = O.OracleSim(O.make_cfg(**c), O.seeded_m(c["grid"], 1, "tilted"), bits=32)
    r1 = o.run_table(3e-11, 1e-11)
    r2 = o.run_table(3e-11, 1e-11)
    r = np.concatenate([r1, r2])
    assert r[0, 0] == 0 and len(r) == 6
    gaps = np.diff(r[:, 0])
    assert np.all(gaps >= np.float32(1e-11) * (1 - 1e-6))
    assert np.all(gaps <= 1e-11 + 2 * o.dt() * o.unit("time"))
    assert np.allclose(np.linalg.norm(r[:, 1:4], axis=1) <= 1.0 + 1e-6, True)
    assert np.all(r[:, 5] <= r[:, 6])
