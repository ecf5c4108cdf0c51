"""Host side of the serving form (no GPU): the seeded request stream, the
sweep fields' float32 arithmetic (simhysteresis.go:18-24 then the
ApplyStatic conversion, simfield.go:87-98), the footprint the admission
control budgets with, and the submission checks."""
import numpy as np
import pytest


def test_stream_is_seeded_and_poisson(eng):
    a = eng.serve_stream(400, seed=5)
    b = eng.serve_stream(400, seed=5)
    assert [r["arrival"] for r in a] == [r["arrival"] for r in b]
    assert [r["cfg"]["grid"] for r in a] == [r["cfg"]["grid"] for r in b]
    gaps = np.diff([0.0] + [r["arrival"] for r in a])
    assert abs(gaps.mean() - 1 / 200.0) < 0.25 / 200.0  # rate 200 req/s
    kinds = [r["kind"] for r in a]
    assert 0.35 < kinds.count("sweep") / len(kinds) < 0.65
    for r in a:
        nx, ny, nz = r["cfg"]["grid"]
        assert nx in (32, 48, 64, 96, 128, 192, 256) and ny in (32, 48, 64, 96, 128, 192, 256) and nz in (1, 2, 4)
        assert 4e5 <= r["cfg"]["msat"] <= 1.4e6 and 5e-12 <= r["cfg"]["aexch"] <= 2e-11
        assert r["cfg"]["alpha"] == 1.0 and r["cfg"]["solver"] == "rk4"
        if r["kind"] == "relax":
            assert r["fields"] is None and np.linalg.norm(r["cfg"]["bext"]) <= 0.1 + 1e-12
        else:
            assert r["fields"].shape == (21, 3)


def test_stream_m0_is_unit_and_internal_layout(eng):
    r = eng.serve_stream(3, seed=5)[2]
    m = eng.stream_m0(r)
    nx, ny, nz = r["cfg"]["grid"]
    assert m.shape == (3, nz, ny, nx) and m.dtype == np.float32
    assert np.allclose((m.astype(np.float64) ** 2).sum(0), 1.0, atol=1e-6)


def test_sweep_fields_follow_reference_float32(eng):
    ms, a = 8.6e5, 1.3e-11
    f = eng.sweep_fields(ms, a, (-0.1, 0.0, 0.0), (0.1, 0.0, 0.0), 21)
    B = eng.units(ms, a)["field"]
    for i in range(21):
        frac = np.float32(np.float32(i) / np.float32(20))
        bx = np.float32(np.float32(-0.1) + np.float32(np.float32(np.float32(0.1) - np.float32(-0.1)) * frac))
        # user x is internal component 2
        assert f[i, 2] == np.float32(bx / B) and f[i, 0] == 0 and f[i, 1] == 0
    assert f[10, 2] == 0.0 and f[0, 2] == -f[20, 2]


def test_footprint_counts_resident_buffers(eng):
    # 256 x 256 x 4 RK4 instance: spectrum 3*N0*P1*HZ complex, 7 vectors of
    # 3N floats, the kernel octant, plus the transient kernel build buffers.
    p = eng.mmx_params(grid=(256, 256, 4), cell=(3e-9,) * 3, msat=8e5, aexch=1.3e-11, alpha=1.0, solver="rk4",
                       dt=1e-13)
    N0, N1, N2 = 4, 256, 256
    P0, P1, P2 = 8, 512, 512
    HZ = P2 // 2 + 1
    n3 = 3 * N0 * N1 * N2
    want = 3 * N0 * P1 * HZ * 8 + n3 * 4 * 7 + 64 + 6 * (P0 // 2 + 1) * (P1 // 2 + 1) * HZ * 4
    want += 6 * P0 * P1 * P2 * 4 + P0 * P1 * HZ * 8
    assert eng.footprint(p) == want
    small = eng.mmx_params(grid=(32, 32, 1), cell=(3e-9,) * 3, msat=8e5, aexch=1.3e-11, alpha=1.0, solver="rk4",
                           dt=1e-13)
    assert eng.footprint(small) < eng.footprint(p) / 50


def test_server_admission_checks_on_the_host(eng):
    """Submission is pure host logic: requests whose footprint exceeds the
    device budget, non-RK4 solves and malformed sweeps are refused with a
    status, before anything reaches a GPU."""
    sv = eng.Server(batched=True, check_every=10, hbm_budget=1 << 20)  # 1 MiB: nothing fits
    r = eng.serve_stream(1, seed=5)[0]
    m0 = eng.stream_m0(r)
    with pytest.raises(eng.MmxError, match="out of memory|budget"):
        sv.submit(eng.mmx_params(**r["cfg"]), m0, r["fields"])
    sv.close()
    sv = eng.Server(batched=True, check_every=10, hbm_budget=1 << 40)
    heun = dict(r["cfg"], solver="heun")
    with pytest.raises(eng.MmxError, match="bad argument|RK4"):
        sv.submit(eng.mmx_params(**heun), m0, r["fields"])
    with pytest.raises(eng.MmxError):
        sv.submit(eng.mmx_params(**r["cfg"]), m0, None, max_torque=0.0)
    rid = sv.submit(eng.mmx_params(**r["cfg"]), m0, r["fields"])
    res = sv.result(rid)
    assert res["state"] == "queued" and res["points_done"] == 0 and res["t_admit"] < 0
    assert res["footprint"] == eng.footprint(eng.mmx_params(**r["cfg"]))
    with pytest.raises(eng.MmxError):
        sv.release(rid)  # still in flight
    sv.close()
