"""Precision form: length-32 DFTs as split-BF16 tensor-core GEMMs (tcgen05),
checked against a float64 DFT.  The split keeps about 16 significant bits
per operand, so the error bound is stated relative to the largest output."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("inverse", [0, 1])
@pytest.mark.parametrize("nvec", [1, 300, 1024])
def test_dft_tc_vs_fp64(eng, cuda, inverse, nvec):
    torch = cuda
    rng = np.random.default_rng(11 + nvec + inverse)
    x = (rng.standard_normal((nvec, 32)) + 1j * rng.standard_normal((nvec, 32))).astype(np.complex64)
    xin = torch.from_numpy(x.view(np.float32).reshape(nvec, 64)).cuda()
    out = torch.zeros_like(xin)
    rc = eng.lib().mmx_dft_tc(ctypes.c_void_p(xin.data_ptr()), ctypes.c_void_p(out.data_ptr()), nvec, inverse, None)
    assert rc == 0, eng.lib().mmx_last_error()
    got = out.cpu().numpy().reshape(nvec, 32, 2)
    got = got[..., 0].astype(np.float64) + 1j * got[..., 1]
    xd = x.astype(np.complex128)
    ref = np.fft.ifft(xd, axis=1) * 32 if inverse else np.fft.fft(xd, axis=1)
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 4e-5, err


def vortex_m(nx, ny, seed=3, core=2.5, noise=0.02):
    """The 512 x 512 film's vortex-like state, user (x,y,z) -> internal [3][1][ny][nx]:
    in-plane curl about the centre, +z within `core` cells of it, plus
    noise * N(0,1) per component (default_rng(seed)), normalised."""
    y, x = np.mgrid[0:ny, 0:nx].astype(np.float64)
    x -= (nx - 1) / 2.0
    y -= (ny - 1) / 2.0
    r = np.hypot(x, y)
    u = np.zeros((3, 1, ny, nx))
    u[0, 0] = -y / np.maximum(r, 1e-12)
    u[1, 0] = x / np.maximum(r, 1e-12)
    inner = r <= core
    u[0, 0][inner] = 0.0
    u[1, 0][inner] = 0.0
    u[2, 0][inner] = 1.0
    u += noise * np.random.default_rng(seed).standard_normal(u.shape)
    u /= np.sqrt((u * u).sum(axis=0, keepdims=True))
    return np.ascontiguousarray(u[::-1]).astype(np.float32)


FILM512 = dict(grid=(512, 512, 1), cell=(2e-9, 2e-9, 2e-9), msat=8.6e5, aexch=1.3e-11, alpha=0.1)


def test_precision_field_vs_fp64(eng, cuda):
    import oracle as O
    torch = cuda
    m = vortex_m(512, 512)
    h = {}
    for prec in (0, 1):
        s = eng.Solver(eng.mmx_params(**FILM512, solver="rk23", maxerror=1e-5, precision=prec))
        mt = torch.from_numpy(m).cuda().contiguous()
        ht = torch.zeros_like(mt)
        s.field(ctypes.c_void_p(mt.data_ptr()), ctypes.c_void_p(ht.data_ptr()))
        torch.cuda.synchronize()
        s.state()  # raises if the tensor-core waits timed out
        h[prec] = ht.cpu().numpy()
        s.close()
    o = O.OracleSim(O.make_cfg(**FILM512, solver="rk23", maxerror=1e-5), m, bits=64)
    h64 = o.heff(m.astype(np.float64))
    scale = np.abs(h64).max()
    e32 = np.abs(h[0] - h64).max() / scale
    etc = np.abs(h[1] - h64).max() / scale
    assert e32 < 2e-6, e32
    assert etc < 1e-4, etc


def test_precision_steps_vs_fp64(eng, cuda):
    import oracle as O
    m = vortex_m(512, 512)
    s = eng.Solver(eng.mmx_params(**FILM512, solver="rk4", dt=1e-13, precision=1))
    s.set_m(m)
    s.normalize()
    s.step(10)
    s.state()
    got = s.get_m()
    s.close()
    o = O.OracleSim(O.make_cfg(**FILM512, solver="rk4", dt=1e-13), m, bits=64)
    o.steps(10)
    assert np.abs(got - o.m()).max() < 1e-4
