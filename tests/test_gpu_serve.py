"""The serving form on the GPU: each request's result is the same alone and
in the mix (bit for bit: admission at chunk boundaries, stop checks on the
solve's own step count, batched instances compute what they compute alone),
the batched loop equals the one-at-a-time loop, admission respects the
device budget, and a served relaxation tracks the FP64 oracle."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

CHECK = 50
CAP = 1500


def small_stream(eng, count, seed=5):
    reqs = eng.serve_stream(count, seed=seed, sweep_points=3)
    for r in reqs:
        r["cfg"]["grid"] = tuple(min(g, 48) if i < 2 else g for i, g in enumerate(r["cfg"]["grid"]))
    return reqs


def serve(eng, reqs, batched=True, stagger=False, budget=0, max_active=0):
    sv = eng.Server(batched=batched, check_every=CHECK, hbm_budget=budget, max_active=max_active, keep_m=True)
    ids = []
    peak_used = 0
    for k, r in enumerate(reqs):
        ids.append(sv.submit(eng.mmx_params(**r["cfg"]), eng.stream_m0(r), r["fields"], 1e-4, CAP))
        if stagger:  # later requests join while the earlier ones run
            sv.pump()
            peak_used = max(peak_used, sv.stats()["used_bytes"])
    while True:
        a, q = sv.pump()
        peak_used = max(peak_used, sv.stats()["used_bytes"])
        if max_active:
            assert a <= max_active
        if a == 0 and q == 0:
            break
    out = []
    for rid in ids:
        res = sv.result(rid)
        assert res["state"] == "done", res
        res["m"] = sv.result_m(rid)
        out.append(res)
    stats = sv.stats()
    sv.close()
    return out, peak_used, stats


def test_served_result_is_the_same_alone_and_in_the_mix(eng, cuda):
    reqs = small_stream(eng, 5)
    mixed, _, stats = serve(eng, reqs, stagger=True)
    assert stats["regroups"] >= 1  # the mix ran batched (solves also ran on their own graphs)
    for r, got in zip(reqs, mixed):
        alone, _, _ = serve(eng, [r])
        a = alone[0]
        assert np.array_equal(a["m"], got["m"]), r["index"]
        assert np.array_equal(a["avg_m"], got["avg_m"])
        assert list(a["point_steps"]) == list(got["point_steps"])


def test_batched_loop_equals_one_at_a_time(eng, cuda):
    reqs = small_stream(eng, 4, seed=11)
    b, _, _ = serve(eng, reqs, batched=True)
    p, _, _ = serve(eng, reqs, batched=False)
    for x, y in zip(b, p):
        assert np.array_equal(x["m"], y["m"])
        assert list(x["point_steps"]) == list(y["point_steps"])


def test_admission_respects_device_budget(eng, cuda):
    reqs = small_stream(eng, 6, seed=12)
    fps = [eng.footprint(eng.mmx_params(**r["cfg"])) for r in reqs]
    budget = sorted(fps)[-1] + sorted(fps)[-2]  # room for about two solves
    got, peak, _ = serve(eng, reqs, budget=budget)
    assert peak <= budget
    ref, _, _ = serve(eng, reqs)
    for x, y in zip(got, ref):
        assert np.array_equal(x["m"], y["m"])


def test_served_relaxation_tracks_fp64_oracle(eng, cuda):
    r = small_stream(eng, 1, seed=13)[0]
    r["kind"], r["fields"] = "relax", None
    r["cfg"]["grid"] = (32, 32, 1)
    r["cfg"]["bext"] = (0.01, 0.0, 0.0)
    res, _, _ = serve(eng, [r])
    steps = int(res[0]["point_steps"][0])
    o = O.OracleSim(O.make_cfg(**{k: v for k, v in r["cfg"].items()}), eng.stream_m0(r), bits=64)
    o.steps(steps)
    assert np.abs(res[0]["m"] - o.m()).max() < 1e-4
