"""Parity of the drop-in libgpukern C ABI primitives (CUDA, sm_100a) with the
CPU oracle, called through the C ABI exactly as the reference's Go driver
calls them (src/go/sim/gpu.go).

Element-wise primitives are bit-exact against the oracle's FP32 build (same
float32 operations in the same order); transforms are compared with the
oracle's FP64 build within the reference's own FFT tolerance (1e-4,
src/go/sim/fft_test.go:160,224) scaled to the data."""
import ctypes

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def host(t):
    return t.detach().cpu().numpy()


def P(t):
    return ctypes.c_void_p(t.data_ptr())


def ints(*v):
    return (ctypes.c_int * len(v))(*v)


def fa(*v):
    return (ctypes.c_float * len(v))(*[float(x) for x in v])


@pytest.fixture(scope="module")
def L(eng, cuda):
    lib = eng.lib()
    lib.gpu_init(0, 0)
    return lib


def rand_m(n, seed, unit=True):
    m = np.random.default_rng(seed).standard_normal((3, n)).astype(np.float32)
    if unit:
        m = O.normalize(m)
    return m


def test_deltaM_bitexact(L, cuda):
    n = 10007
    m = rand_m(n, 1)
    h = np.random.default_rng(2).standard_normal((3, n)).astype(np.float32) * 3
    alpha, dtg = np.float32(0.02), np.float32(0.00123)
    dm, dh = dev(cuda, m), dev(cuda, h)
    L.gpu_deltaM(P(dm), P(dh), alpha, None, dtg, n)
    ref = O.delta_m(m, h, alpha, dtg)
    assert np.array_equal(host(dh), ref)


def test_normalize_bitexact(L, cuda):
    n = 4099
    m = rand_m(n, 3, unit=False) * 1.7
    d = dev(cuda, m)
    L.gpu_normalize_uniform(P(d), n)
    assert np.array_equal(host(d), O.normalize(m))


@pytest.mark.parametrize("anis", [0, 1])
def test_local_fields_bitexact(L, cuda, anis):
    n = 5000
    m = rand_m(n, 4)
    h = np.random.default_rng(5).standard_normal((3, n)).astype(np.float32)
    hext = np.array([-0.0244, 0.0043, 0.0], np.float32)
    K, u = np.float32(0.63), np.array([0.6, 0.0, 0.8], np.float32)
    dm, dh = dev(cuda, m), dev(cuda, h)
    L.gpu_add_local_fields(P(dm), P(dh), n, fa(*hext), None, anis, fa(K, 0, 0), fa(*u))
    ref = O.add_local_fields(m, h, hext, anis, K, u)
    assert np.array_equal(host(dh), ref)


def test_linalg_bitexact(L, cuda):
    n = 3 * 7001
    rng = np.random.default_rng(6)
    a, b = rng.standard_normal(n).astype(np.float32), rng.standard_normal(n).astype(np.float32)
    da, db = dev(cuda, a), dev(cuda, b)
    L.gpu_madd(P(da), np.float32(-0.37), P(db), n)
    ref = (a + np.float32(-0.37) * b).astype(np.float32)
    assert np.array_equal(host(da), ref)
    da = dev(cuda, a)
    L.gpu_linear_combination(P(da), P(db), np.float32(0.5), np.float32(0.5), n)
    assert np.array_equal(host(da), (np.float32(0.5) * a + np.float32(0.5) * b).astype(np.float32))
    da = dev(cuda, a)
    L.gpu_add(P(da), P(db), n)
    assert np.array_equal(host(da), a + b)


# redux_test.go:13-102 sizes and expectations
NS = [2, 8, 16, 31, 33, 128, 255, 511, 1023, 1024, 1025, 20000]


def reductor(L, n):
    threads = L.gpu_maxthreads() // 2
    while n <= threads:
        threads //= 2
    blocks = (n - 1) // (threads * 2) + 1
    return threads, blocks


@pytest.mark.parametrize("n", NS)
def test_reductions_reference_cases(L, cuda, n):
    threads, blocks = reductor(L, n)
    dev2 = cuda.zeros(blocks, device="cuda")
    host2 = (ctypes.c_float * blocks)()
    ones = dev(cuda, np.ones(n))
    assert L.gpu_reduce(1, P(ones), P(dev2), host2, blocks, threads, n) == float(n)
    neg = dev(cuda, -np.ones(n))
    assert L.gpu_reduce(5, P(neg), P(dev2), host2, blocks, threads, n) == float(n)
    v = np.ones(n, np.float32)
    v[12349 % n] = 10.0
    assert L.gpu_reduce(2, P(dev(cuda, v)), P(dev2), host2, blocks, threads, n) == 10.0
    v[12349 % n] = -10.0
    assert L.gpu_reduce(3, P(dev(cuda, v)), P(dev2), host2, blocks, threads, n) == 10.0
    assert L.gpu_reduce(4, P(dev(cuda, v)), P(dev2), host2, blocks, threads, n) == -10.0


FFT_CASES = [
    # (N, P): internal sizes; 2D, 3D, mixed radix, periodic (P == N)
    ((1, 16, 16), (1, 32, 32)),
    ((1, 32, 128), (1, 64, 256)),
    ((4, 8, 16), (8, 16, 32)),
    ((3, 12, 10), (6, 24, 20)),
    ((2, 24, 48), (4, 48, 96)),
    ((5, 7, 9), (10, 14, 18)),
    ((4, 16, 16), (4, 32, 32)),
    ((8, 64, 64), (16, 128, 128)),
]


@pytest.mark.parametrize("N,Pd", FFT_CASES)
def test_fft_forward_inverse(L, cuda, N, Pd):
    rng = np.random.default_rng(7)
    a = rng.random(N).astype(np.float32)
    plan = L.new_gpuFFT3dPlan_padded(ints(*N), ints(*Pd))
    assert L.gpuFFT3dPlan_normalization(plan) == Pd[0] * Pd[1] * Pd[2]
    din = dev(cuda, a)
    dout = cuda.zeros(Pd[0] * Pd[1] * (Pd[2] + 2), device="cuda")
    L.gpuFFT3dPlan_forward(plan, P(din), P(dout))
    spec = host(dout).reshape(Pd[0], Pd[1], Pd[2] + 2)
    ref = O.fft_forward_padded(N, Pd, a.astype(np.float64), bits=64)
    scale = np.abs(ref).max()
    assert np.abs(spec - ref).max() <= 1e-5 * scale
    # inverse (unnormalised), compare with the oracle and the round trip
    back = cuda.zeros(N, device="cuda")
    L.gpuFFT3dPlan_inverse(plan, P(dout), P(back))
    rt = host(back) / np.float32(np.prod(Pd))
    assert np.abs(rt - a).max() <= 1e-4 * max(1.0, np.abs(a).max())
    L.delete_gpuFFT3dPlan(plan)


def test_fft_matches_oracle_inverse(L, cuda):
    N, Pd = (3, 20, 24), (6, 40, 48)
    rng = np.random.default_rng(8)
    spec = rng.standard_normal((Pd[0], Pd[1], Pd[2] + 2)).astype(np.float32)
    # a spectrum of a real field: take the forward transform of a real array
    a = rng.standard_normal(N).astype(np.float32)
    spec = O.fft_forward_padded(N, Pd, a.astype(np.float64), bits=64).astype(np.float32)
    plan = L.new_gpuFFT3dPlan_padded(ints(*N), ints(*Pd))
    d = dev(cuda, spec)
    out = cuda.zeros(N, device="cuda")
    L.gpuFFT3dPlan_inverse(plan, P(d), P(out))
    ref = O.fft_inverse_padded(N, Pd, spec.astype(np.float64), bits=64)
    assert np.abs(host(out) - ref).max() <= 2e-5 * np.abs(ref).max()
    L.delete_gpuFFT3dPlan(plan)


def test_kernelmul6_bitexact(L, cuda):
    n = 3000
    rng = np.random.default_rng(9)
    M = [rng.standard_normal(2 * n).astype(np.float32) for _ in range(3)]
    K = [rng.standard_normal(n).astype(np.float32) for _ in range(6)]
    dM = [dev(cuda, x) for x in M]
    dK = [dev(cuda, x) for x in K]
    L.gpu_kernelmul6(*[P(t) for t in dM], *[P(t) for t in dK], 2 * n)
    Kxx, Kyy, Kzz, Kyz, Kxz, Kxy = K
    re = [x[0::2] for x in M]
    im = [x[1::2] for x in M]
    f = np.float32

    def row(a, b, c, p, q, r):
        return ((a * p).astype(f) + (b * q).astype(f)).astype(f) + (c * r).astype(f)

    hx = (row(re[0], re[1], re[2], Kxx, Kxy, Kxz), row(im[0], im[1], im[2], Kxx, Kxy, Kxz))
    out = host(dM[0])
    assert np.array_equal(out[0::2], hx[0]) and np.array_equal(out[1::2], hx[1])


def test_copy_pad_unpad(L, cuda):
    S = (3, 5, 7)
    D = (6, 10, 16)
    a = np.arange(np.prod(S), dtype=np.float32).reshape(S)
    src = dev(cuda, a)
    dst = cuda.zeros(D, device="cuda")
    L.gpu_copy_pad(P(src), P(dst), *S, *D)
    ref = np.zeros(D, np.float32)
    ref[:3, :5, :7] = a
    assert np.array_equal(host(dst), ref)
    back = cuda.zeros(S, device="cuda")
    L.gpu_copy_unpad(P(dst), P(back), *D, *S)
    assert np.array_equal(host(back), a)


def test_zeropad_reference_case(L, cuda):
    # zeropad_test.cpp: 129 x 255 into 258 x 510 and back
    S1, S2, D1, D2 = 129, 255, 258, 510
    a = np.random.default_rng(10).random((S1, S2)).astype(np.float32)
    src = dev(cuda, a)
    dst = cuda.zeros((D1, D2), device="cuda")
    L.gpu_copy_pad2D(P(src), P(dst), S1, S2, D1, D2)
    assert np.array_equal(host(dst)[:S1, :S2], a) and host(dst)[S1:].sum() == 0
    back = cuda.zeros((S1, S2), device="cuda")
    L.gpu_copy_unpad2D(P(dst), P(back), D1, D2, S1, S2)
    assert np.array_equal(host(back), a)


def test_exchange_stencil(L, cuda):
    N = (4, 6, 8)
    cs = np.array([0.8, 0.9, 1.1], np.float32)
    m = rand_m(int(np.prod(N)), 11).reshape((3,) + N)
    h = np.zeros_like(m)
    dm, dh = dev(cuda, m), dev(cuda, h)
    L.gpu_add_exch(P(dm), P(dh), ints(*N), ints(0, 0, 0), ints(0, 0, 0), fa(*cs), 6)
    # direct 7-point Laplacian with zero outside
    pad = np.zeros((3, N[0] + 2, N[1] + 2, N[2] + 2), np.float64)
    pad[:, 1:-1, 1:-1, 1:-1] = m
    lap = (-2 / cs[0] ** 2 - 2 / cs[1] ** 2 - 2 / cs[2] ** 2) * m.astype(np.float64)
    lap += (pad[:, :-2, 1:-1, 1:-1] + pad[:, 2:, 1:-1, 1:-1]) / cs[0] ** 2
    lap += (pad[:, 1:-1, :-2, 1:-1] + pad[:, 1:-1, 2:, 1:-1]) / cs[1] ** 2
    lap += (pad[:, 1:-1, 1:-1, :-2] + pad[:, 1:-1, 1:-1, 2:]) / cs[2] ** 2
    assert np.abs(host(dh) - lap).max() < 1e-5 * np.abs(lap).max()


def test_memory_and_properties(L, cuda):
    p = L.new_gpu_array(1000)
    assert L.gpu_array_get(p, 999) == 0.0
    L.gpu_array_set(p, 5, 3.5)
    assert L.gpu_array_get(p, 5) == 3.5
    buf = (ctypes.c_float * 10)(*range(10))
    L.memcpy_gpu_dir(buf, p, 10, 1)
    out = (ctypes.c_float * 10)()
    L.memcpy_gpu_dir(p, out, 10, 3)
    assert list(out) == list(range(10))
    L.free_gpu_array(p)
    assert L.gpu_maxthreads() >= 256
    assert L.gpu_stride_float() >= 1


GENERIC_SIZES = [((3, 11, 13), (6, 22, 26)), ((1, 17, 19), (1, 34, 38)), ((2, 5, 23), (4, 10, 46)),
                 ((4, 7, 11), (4, 14, 22)), ((1, 6, 9), (1, 12, 9)), ((2, 3, 4), (2, 3, 4))]


@pytest.mark.parametrize("N,Pd", GENERIC_SIZES)
def test_fft_plan_any_size_vs_numpy(L, cuda, N, Pd):
    """gpuFFT3dPlan_* for padded sizes with prime factors above 7 (and an
    odd padded Z): the plan takes the generic path (Bluestein lines) where
    cufftPlan3d takes any size (gpu_fft0.cu:57-68).  Forward against numpy's
    real FFT in float64 (the reference's (P0,P1,P2+2)-float rows), inverse
    as the unnormalised complex-to-real transform."""
    n = int(np.prod(N))
    a = np.random.default_rng(40).standard_normal(N).astype(np.float32)
    box = np.zeros(Pd)
    box[:N[0], :N[1], :N[2]] = a
    want = np.fft.rfftn(box)
    H = Pd[2] // 2 + 1
    plan = L.new_gpuFFT3dPlan_padded(ints(*N), ints(*Pd))
    din = dev(cuda, a)
    spec = cuda.zeros(Pd[0] * Pd[1] * (Pd[2] + 2), device="cuda")
    L.gpuFFT3dPlan_forward(plan, P(din), P(spec))
    s = host(spec).reshape(Pd[0], Pd[1], Pd[2] + 2)[:, :, :2 * H]
    got = s[..., 0::2] + 1j * s[..., 1::2]
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= 2e-6 * scale * np.log2(np.prod(Pd))
    back = cuda.zeros(n + (Pd[0] - N[0]) * N[1] * N[2], device="cuda")
    L.gpuFFT3dPlan_inverse(plan, P(spec), P(back))
    b = host(back)[:n].reshape(N)
    nrm = L.gpuFFT3dPlan_normalization(plan)
    assert nrm == np.prod(Pd)
    assert np.abs(b / nrm - a).max() <= 2e-6 * np.abs(a).max() * np.log2(np.prod(Pd))
    L.delete_gpuFFT3dPlan(plan)
