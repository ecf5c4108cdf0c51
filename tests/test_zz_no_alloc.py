"""The allocation-free reduction, mmx_reduce_static, called through the C ABI.

Callers that may not call cudaMalloc (a thread running while another captures
a CUDA graph in global mode, host callbacks, embedders that budget all device
memory up front) use this variant of gpu_reduce; its per-block partials live
in an array compiled into the library.  Checked against the existing entry
point gpu_reduce on two calls in a row, so that the second call runs on the
array as the first call left it.  Collected last so a stop-at-first-failure
run has already run every other test."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

OPS = {1: "add", 2: "max", 3: "maxabs", 4: "min", 5: "sumabs"}


def reference_reduce(L, torch, op, dev_in, n):
    threads = L.gpu_maxthreads() // 2
    while n <= threads:
        threads //= 2
    blocks = (n - 1) // (threads * 2) + 1
    dev2 = torch.zeros(blocks, device="cuda")
    host2 = (ctypes.c_float * blocks)()
    return L.gpu_reduce(op, ctypes.c_void_p(dev_in.data_ptr()), ctypes.c_void_p(dev2.data_ptr()), host2, blocks,
                        threads, n)


def test_reduce_static_matches_gpu_reduce_twice(eng, cuda):
    L = eng.lib()
    L.gpu_init(0, 0)
    rng = np.random.default_rng(11)
    out = cuda.zeros(1, device="cuda")
    sizes = [4_194_304, 37_001]  # the maximum, then a smaller call on the same array
    for call, n in enumerate(sizes):
        a = cuda.from_numpy(rng.standard_normal(n).astype(np.float32)).cuda()
        for op in OPS:
            rc = L.mmx_reduce_static(op, ctypes.c_void_p(a.data_ptr()), n, ctypes.c_void_p(out.data_ptr()), None)
            assert rc == 0, L.mmx_last_error()
            cuda.cuda.synchronize()
            got = float(out.item())
            want = reference_reduce(L, cuda, op, a, n)
            tol = 1e-6 * max(1.0, abs(want)) if op in (1, 5) else 0.0
            assert abs(got - want) <= tol, (call, OPS[op], got, want)


def test_reduce_static_rejects_oversize(eng, cuda):
    L = eng.lib()
    a = cuda.zeros(8, device="cuda")
    out = cuda.zeros(1, device="cuda")
    rc = L.mmx_reduce_static(1, ctypes.c_void_p(a.data_ptr()), 4_194_305, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == 3  # MMX_ERR_SIZE, nothing launched
    assert b"MMX_REDUCE_STATIC_MAX_N" in L.mmx_last_error()


def test_reduce_static_beside_a_global_mode_capture(eng, cuda):
    """The case the entry point exists for: while one thread captures a CUDA
    graph in global mode (where cudaMalloc from any thread is an error),
    another thread reduces on a non-blocking stream of its own.  The first
    call, which looks the array's address up, comes before the capture."""
    import threading

    L = eng.lib()
    n = 100_003
    a = cuda.from_numpy(np.random.default_rng(12).standard_normal(n).astype(np.float32)).cuda()
    out = cuda.zeros(1, device="cuda")
    assert L.mmx_reduce_static(1, ctypes.c_void_p(a.data_ptr()), n, ctypes.c_void_p(out.data_ptr()), None) == 0
    cuda.cuda.synchronize()
    want = {op: reference_reduce(L, cuda, op, a, n) for op in OPS}
    side = cuda.cuda.Stream()  # torch streams are created non-blocking
    results = cuda.zeros(len(OPS), device="cuda")
    started, reduced = threading.Event(), threading.Event()
    rcs = []

    def reducer():
        started.wait(30)
        for k, op in enumerate(OPS):
            rcs.append(L.mmx_reduce_static(op, ctypes.c_void_p(a.data_ptr()), n,
                                           ctypes.c_void_p(results.data_ptr() + 4 * k),
                                           ctypes.c_void_p(side.cuda_stream)))
        reduced.set()

    t = threading.Thread(target=reducer)
    t.start()
    g = cuda.cuda.CUDAGraph()
    x = cuda.zeros(16, device="cuda")
    with cuda.cuda.graph(g, capture_error_mode="global"):
        x.add_(1.0)
        started.set()
        assert reduced.wait(30)
    t.join(30)
    side.synchronize()
    g.replay()
    cuda.cuda.synchronize()
    assert rcs == [0] * len(OPS), [L.mmx_last_error()]
    got = results.cpu().numpy()
    for k, op in enumerate(OPS):
        tol = 1e-6 * max(1.0, abs(want[op])) if op in (1, 5) else 0.0
        assert abs(float(got[k]) - want[op]) <= tol, (OPS[op], got[k], want[op])
    assert float(x[0].item()) == 1.0
