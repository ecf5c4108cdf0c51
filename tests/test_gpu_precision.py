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
