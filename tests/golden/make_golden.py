"""Generates golden vectors from the REFERENCE's own CUDA library.

Runs on a machine with a GPU, after `make -f oracle/Makefile.ref` has built
oracle/_ref/libgpukern_ref.so from the reference's sources (MuMax 1.1
src/gpukern, cuFFT-based).  The reference library is driven through the
C++ restatement of its Go driver (1_b200/libmmxdriver.so) exactly as
src/go/sim drives it; the real-space demag + exchange kernel fed to it is the
oracle's float32 restatement of FaceKernel6 + Exch6NgbrKernel (the Go
subprocess mumaxkern-go cannot be built here).

Writes tests/golden/reference_vectors.npz (+ .json with provenance).  The
CPU tests compare the oracle with these vectors (tests/test_cpu_golden.py);
the GPU tests compare the B200 engine with the reference library directly.

usage: python tests/golden/make_golden.py
"""
import importlib
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402

REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libgpukern_ref.so")

CASES = {
    # 2D film: the 128 x 32 x 1 thin-film materials on a 64 x 16 x 1 grid
    "film2d": dict(cfg=dict(grid=(64, 16, 1), cell=(3.90625e-9, 3.90625e-9, 3e-9), msat=8.0e5, aexch=1.3e-11,
                            alpha=0.02, bext=(-24.6e-3, 4.3e-3, 0.0)),
                   seed=1, init="tilted",
                   runs=[("heun", dict(solver="heun", dt=2e-13), 50),
                         ("rk23", dict(solver="rk23", maxerror=1e-5), 20)]),
    # 3D grid: the 256 x 256 x 32 workload's materials on a 16 x 16 x 8 grid
    "cube3d": dict(cfg=dict(grid=(16, 16, 8), cell=(4e-9, 4e-9, 4e-9), msat=1.1e6, aexch=1.5e-11, alpha=0.5,
                            anis=1, k1=5e5, axis=(0, 0, 1)),
                   seed=2, init="random",
                   runs=[("heun", dict(solver="heun", dt=1e-14), 50),
                         ("rk23", dict(solver="rk23", maxerror=1e-5), 10)]),
}


def kernel_for(o32):
    N = o32.N
    P = tuple(2 * n if n > 1 else n for n in N)
    cs = o32.internal_params()["cellsize"]
    k6 = O.face_kernel6(P, cs)
    O.add_exch6_kernel(P, cs, k6)
    return k6


def main():
    eng = importlib.import_module("1_b200")
    if not os.path.exists(REF_LIB):
        raise SystemExit("build the reference library first: make -f oracle/Makefile.ref")
    out = {}
    meta = {"library": "oracle/_ref/libgpukern_ref.so (reference src/gpukern, nvcc sm_100a, cuFFT)",
            "driver": "1_b200/libmmxdriver.so (restatement of src/go/sim)", "cases": {}}
    try:
        import torch
        meta["gpu"] = torch.cuda.get_device_name(0)
    except Exception:
        pass
    try:
        meta["nvcc"] = subprocess.check_output(["nvcc", "--version"]).decode().strip().splitlines()[-1]
    except Exception:
        pass
    for name, case in CASES.items():
        m = O.seeded_m(case["cfg"]["grid"], case["seed"], case["init"])
        o32 = O.OracleSim(O.make_cfg(**case["cfg"], solver="heun", dt=1e-14), m, bits=32)
        m0 = o32.m()
        k6 = kernel_for(o32)
        out[name + "/m0"] = m0
        d = eng.DriverSim(eng.driver_config(**case["cfg"], solver="heun", dt=1e-14), m0, k6, libpath=REF_LIB)
        out[name + "/heff"] = d.heff(m0)
        d.close()
        meta["cases"][name] = {"config": case["cfg"], "seed": case["seed"], "init": case["init"], "runs": {}}
        for rname, kw, steps in case["runs"]:
            d = eng.DriverSim(eng.driver_config(**case["cfg"], **kw), m0, k6, libpath=REF_LIB)
            d.steps(steps)
            out["%s/%s/m" % (name, rname)] = d.m()
            out["%s/%s/avg_m" % (name, rname)] = d.avg_m()
            meta["cases"][name]["runs"][rname] = {"solver": kw, "steps": steps, "time": d.time(), "dt": float(d.dt()),
                                                  "torque": float(d.torque())}
            d.close()
    np.savez_compressed(os.path.join(HERE, "reference_vectors.npz"), **out)
    with open(os.path.join(HERE, "reference_vectors.json"), "w") as f:
        json.dump(meta, f, indent=1, default=str)
    print("wrote", sorted(out))


if __name__ == "__main__":
    main()
