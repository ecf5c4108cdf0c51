"""B200 LLG engine: the drop-in libgpukern C ABI, its fused extended ABI and
the C++ restatement of the reference's Go driver, loaded through ctypes.

Modules of this package:
  * ``libgpukern.so``   -- CUDA kernels for sm_100a behind the reference's
    libgpukern C ABI (include/gpukern.h) plus the fused ``mmx_*`` entry
    points (include/mmx.h);
  * ``libmmxdriver.so`` -- C++ host driver restating the Go driver over
    any libgpukern implementation (include/mmx_driver.h).

Nothing here falls back to a CPU path: if the CUDA library is missing the
import fails with a message naming the build step.
"""
import ctypes
import time
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
# MMX_LIBGPUKERN selects another build of the library (e.g. one compiled with
# different tile shapes); the default is the in-tree build.
LIB_PATH = os.environ.get("MMX_LIBGPUKERN", os.path.join(HERE, "libgpukern.so"))
DRIVER_PATH = os.path.join(HERE, "libmmxdriver.so")

SOLVERS = {"heun": 0, "rk12": 1, "rk23": 2, "rk4": 3, "rkck": 4, "rkdp": 5, "rk2": 6}
ERRORS = {0: "ok", 1: "bad argument", 2: "CUDA error", 3: "unsupported size", 4: "NaN", 5: "out of memory",
          6: "bad state"}


def build(jobs=8):
    """Compile libgpukern.so and libmmxdriver.so in-tree for sm_100a."""
    subprocess.check_call(["make", "-s", "-j%d" % jobs, "-f", os.path.join(HERE, "Makefile")], cwd=HERE)


class MmxError(RuntimeError):
    pass


# --------------------------------------------------------------------------
# ctypes prototypes
# --------------------------------------------------------------------------
c_float_p = ctypes.c_void_p
c_int_p = ctypes.POINTER(ctypes.c_int)


class MmxParams(ctypes.Structure):
    _fields_ = [
        ("size", ctypes.c_int * 3),
        ("periodic", ctypes.c_int * 3),
        ("cellsize", ctypes.c_float * 3),
        ("alpha", ctypes.c_float),
        ("hext", ctypes.c_float * 3),
        ("anis_type", ctypes.c_int),
        ("anis_k", ctypes.c_float),
        ("anis_axis", ctypes.c_float * 3),
        ("solver", ctypes.c_int),
        ("dt", ctypes.c_float),
        ("max_error", ctypes.c_float),
        ("min_dm", ctypes.c_float),
        ("max_dm", ctypes.c_float),
        ("min_dt", ctypes.c_float),
        ("max_dt", ctypes.c_float),
        ("unit_time", ctypes.c_float),
        ("exch_type", ctypes.c_int),
        ("faithful", ctypes.c_int),
        ("accuracy", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("thermal_k", ctypes.c_float),
        ("thermal_seed", ctypes.c_uint),
    ]


class MmxRequest(ctypes.Structure):
    _fields_ = [
        ("params", MmxParams),
        ("m0", ctypes.c_void_p),
        ("npoints", ctypes.c_int),
        ("hext_points", ctypes.c_void_p),
        ("max_torque", ctypes.c_float),
        ("max_steps", ctypes.c_longlong),
    ]


class MmxServerConfig(ctypes.Structure):
    _fields_ = [
        ("hbm_budget", ctypes.c_size_t),
        ("max_active", ctypes.c_int),
        ("check_every", ctypes.c_int),
        ("batched", ctypes.c_int),
        ("keep_m", ctypes.c_int),
    ]


class MmxResult(ctypes.Structure):
    _fields_ = [
        ("state", ctypes.c_int),
        ("converged", ctypes.c_int),
        ("steps", ctypes.c_longlong),
        ("points_done", ctypes.c_int),
        ("t_submit", ctypes.c_double),
        ("t_admit", ctypes.c_double),
        ("t_done", ctypes.c_double),
        ("footprint", ctypes.c_size_t),
    ]


class DriverConfig(ctypes.Structure):
    _fields_ = [
        ("grid", ctypes.c_int * 3),
        ("cell", ctypes.c_double * 3),
        ("periodic", ctypes.c_int * 3),
        ("msat", ctypes.c_double),
        ("aexch", ctypes.c_double),
        ("alpha", ctypes.c_double),
        ("bext", ctypes.c_double * 3),
        ("anis_type", ctypes.c_int),
        ("k1", ctypes.c_double),
        ("anis_axis", ctypes.c_double * 3),
        ("solver", ctypes.c_int),
        ("dt", ctypes.c_double),
        ("maxerror", ctypes.c_double),
        ("mindm", ctypes.c_double),
        ("maxdm", ctypes.c_double),
        ("mindt", ctypes.c_double),
        ("maxdt", ctypes.c_double),
        ("faithful", ctypes.c_int),
    ]


# name -> (restype, argtypes); the libgpukern C ABI (include/gpukern.h)
ABI = {
    "gpu_init": (None, [ctypes.c_int, ctypes.c_int]),
    "gpu_set_device": (None, [ctypes.c_int]),
    "gpu_maxthreads": (ctypes.c_int, []),
    "gpu_setmaxthreads": (None, [ctypes.c_int]),
    "gpu_getproperties": (ctypes.c_void_p, []),
    "gpu_print_properties_stdout": (None, []),
    "gpu_getstream": (ctypes.c_void_p, []),
    "gpu_init_stream": (None, []),
    "new_gpu_array": (ctypes.c_void_p, [ctypes.c_int]),
    "free_gpu_array": (None, [ctypes.c_void_p]),
    "gpu_usedmem": (ctypes.c_ulonglong, []),
    "gpu_stride_float": (ctypes.c_int, []),
    "gpu_override_stride": (None, [ctypes.c_int]),
    "memcpy_gpu_dir": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "memcpy_to_gpu": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "memcpy_from_gpu": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "memcpy_on_gpu": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "memcpy_on_gpu_async": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "gpu_array_get": (ctypes.c_float, [ctypes.c_void_p, ctypes.c_int]),
    "gpu_array_set": (None, [ctypes.c_void_p, ctypes.c_int, ctypes.c_float]),
    "gpu_zero": (None, [ctypes.c_void_p, ctypes.c_int]),
    "gpu_zero_async": (None, [ctypes.c_void_p, ctypes.c_int]),
    "assertHost": (None, [ctypes.c_void_p]),
    "assertDevice": (None, [ctypes.c_void_p]),
    "new_ram_array": (ctypes.c_void_p, [ctypes.c_int]),
    "gpu_add": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "gpu_madd": (None, [ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_int]),
    "gpu_madd2": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "gpu_add_constant": (None, [ctypes.c_void_p, ctypes.c_float, ctypes.c_int]),
    "gpu_linear_combination": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_float,
                                      ctypes.c_int]),
    "gpu_linear_combination_many": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                           ctypes.c_int]),
    "gpu_scale_dot_product": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float,
                                     ctypes.c_int]),
    "gpu_normalize_uniform": (None, [ctypes.c_void_p, ctypes.c_int]),
    "gpu_normalize_map": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "gpu_deltaM": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_float,
                          ctypes.c_int]),
    "gpu_add_local_fields": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "gpu_add_local_fields_H_and_phi": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                              ctypes.c_void_p]),
    "gpu_kernelmul6": (None, [ctypes.c_void_p] * 9 + [ctypes.c_int]),
    "gpu_kernelmul4": (None, [ctypes.c_void_p] * 7 + [ctypes.c_int]),
    "gpu_kernelmul3": (None, [ctypes.c_void_p] * 5 + [ctypes.c_int]),
    "gpu_kernelmul_biot_savart3D": (None, [ctypes.c_void_p] * 6 + [ctypes.c_int]),
    "gpu_kernelmul_biot_savart3DNx1": (None, [ctypes.c_void_p] * 5 + [ctypes.c_int]),
    "gpu_kernelmul_biot_savart2D": (None, [ctypes.c_void_p] * 5 + [ctypes.c_int]),
    "gpu_copy_pad": (None, [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 6),
    "gpu_copy_unpad": (None, [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 6),
    "gpu_copy_pad2D": (None, [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 4),
    "gpu_copy_unpad2D": (None, [ctypes.c_void_p, ctypes.c_void_p] + [ctypes.c_int] * 4),
    "new_gpuFFT3dPlan_padded": (ctypes.c_void_p, [c_int_p, c_int_p]),
    "new_gpuFFT3dPlan": (ctypes.c_void_p, [c_int_p]),
    "delete_gpuFFT3dPlan": (None, [ctypes.c_void_p]),
    "gpuFFT3dPlan_forward": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "gpuFFT3dPlan_inverse": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "gpuFFT3dPlan_normalization": (ctypes.c_int, [ctypes.c_void_p]),
    "gpu_reduce": (ctypes.c_float, [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_int]),
    "gpu_partial_sums": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "gpu_partial_maxabs": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "gpu_add_exch": (None, [ctypes.c_void_p, ctypes.c_void_p, c_int_p, c_int_p, c_int_p, ctypes.c_void_p,
                            ctypes.c_int]),
    "gpu_add_lin_anisotropy": (None, [ctypes.c_void_p] * 12 + [ctypes.c_int]),
    "gpu_anal_fw_step": (None, [ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_void_p]),
    "gpu_spintorque_deltaM": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_float,
                                     ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "gpu_gaussian_noise": (None, [ctypes.c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_int]),
    "gpu_transpose_complex_YZ": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int]),
    "gpu_transpose_complex_XZ": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int]),
}

MMX = {
    "mmx_last_error": (ctypes.c_char_p, []),
    "mmx_solver_create": (ctypes.c_int, [ctypes.POINTER(MmxParams), ctypes.POINTER(ctypes.c_void_p)]),
    "mmx_solver_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "mmx_solver_set_m": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "mmx_solver_get_m": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "mmx_solver_normalize": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "mmx_solver_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "mmx_solver_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "mmx_solver_avg_m": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "mmx_solver_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                        ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                                        ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_longlong)]),
    "mmx_solver_set_hext": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "mmx_solver_energy": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    "mmx_solver_relax": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.POINTER(ctypes.c_longlong),
                                        ctypes.POINTER(ctypes.c_float), ctypes.c_void_p]),
    "mmx_solver_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_float, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int), ctypes.c_longlong, ctypes.c_void_p]),
    "mmx_solver_m_device": (ctypes.c_void_p, [ctypes.c_void_p]),
    "mmx_solver_use_graph": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "mmx_solver_device_control": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "mmx_solver_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "mmx_solver_pass_times": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                             ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                                             ctypes.POINTER(ctypes.c_int)]),
    "mmx_batch_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "mmx_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "mmx_batch_instance": (ctypes.c_void_p, [ctypes.c_void_p, ctypes.c_int]),
    "mmx_batch_size": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong),
                                      ctypes.POINTER(ctypes.c_int)]),
    "mmx_batch_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "mmx_batch_use_graph": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "mmx_batch_create_from": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "mmx_batch_tuning": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int)]),
    "mmx_batch_torques": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "mmx_solver_torque_device": (ctypes.c_void_p, [ctypes.c_void_p]),
    "mmx_server_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "mmx_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "mmx_server_footprint": (ctypes.c_int, [ctypes.POINTER(MmxParams), ctypes.POINTER(ctypes.c_size_t)]),
    "mmx_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    "mmx_server_pump": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    "mmx_server_result": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    "mmx_server_result_m": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong, ctypes.c_void_p]),
    "mmx_server_release": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_longlong]),
    "mmx_server_clock": (ctypes.c_double, [ctypes.c_void_p]),
    "mmx_server_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t),
                                        ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong)]),
    "mmx_write_ovf": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, c_int_p, ctypes.POINTER(ctypes.c_double),
                                     ctypes.c_int, ctypes.c_int, ctypes.c_char_p, ctypes.c_double, ctypes.c_double,
                                     ctypes.c_double]),
    "mmx_write_odt": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p]),
    "mmx_dft_tc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "mmx_reduce_static": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                         ctypes.c_void_p]),
    "mmx_face_kernel6": (ctypes.c_int, [c_int_p, c_int_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int,
                                        ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
}

DRIVER = {
    "mmxd_last_error": (ctypes.c_char_p, []),
    "mmxd_open": (ctypes.c_void_p, [ctypes.c_char_p]),
    "mmxd_close": (None, [ctypes.c_void_p]),
    "mmxd_new": (ctypes.c_void_p, [ctypes.c_void_p, ctypes.POINTER(DriverConfig), ctypes.c_void_p,
                                   ctypes.c_void_p]),
    "mmxd_free": (None, [ctypes.c_void_p]),
    "mmxd_sizes": (None, [ctypes.c_void_p, c_int_p, c_int_p]),
    "mmxd_internal": (None, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                             ctypes.c_void_p]),
    "mmxd_steps": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "mmxd_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "mmxd_get_m": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "mmxd_set_m": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "mmxd_heff": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "mmxd_avg_m": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "mmxd_time": (ctypes.c_double, [ctypes.c_void_p]),
    "mmxd_dt": (ctypes.c_float, [ctypes.c_void_p]),
    "mmxd_torque": (ctypes.c_float, [ctypes.c_void_p]),
    "mmxd_step_count": (ctypes.c_longlong, [ctypes.c_void_p]),
    "mmxd_step_error": (ctypes.c_float, [ctypes.c_void_p]),
    "mmxd_energy": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_float)]),
    "mmxd_run_table": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_float, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_int)]),
}

_cache = {}


def _load(path, table, tag):
    if tag in _cache:
        return _cache[tag]
    if not os.path.exists(path):
        raise ImportError("%s is not built: run __graft_entry__.build() (make -C 1_b200)" % path)
    lib = ctypes.CDLL(path)
    for name, (res, args) in table.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _cache[tag] = lib
    return lib


def lib():
    """The B200 libgpukern (ABI + mmx_*) with prototypes."""
    t = dict(ABI)
    t.update(MMX)
    return _load(LIB_PATH, t, "gpukern")


def driver():
    return _load(DRIVER_PATH, DRIVER, "driver")


def exported_symbols():
    """Names the library must export (every declaration of include/*.h)."""
    return sorted(list(ABI) + list(MMX))


def _check(rc):
    if rc != 0:
        raise MmxError("%s: %s" % (ERRORS.get(rc, rc), lib().mmx_last_error().decode()))


# --------------------------------------------------------------------------
# Units and the user -> internal conversion (src/go/sim/material.go,
# init.go, simgeom.go); float32 rounding at each step, as the Go code.
# --------------------------------------------------------------------------
def f32(x):
    return np.float32(x)


def units(msat, aexch):
    mu0 = f32(4.0e-7 * np.pi)
    gamma0 = f32(2.211e5)
    ms, A = f32(msat), f32(aexch)
    t = f32(f32(mu0 * ms) * ms)
    L = f32(np.sqrt(2.0 * np.float64(f32(A / t))))
    T = f32(f32(1.0) / f32(gamma0 * ms))
    B = f32(mu0 * ms)
    vol = f32(f32(L * L) * L)
    E = f32(f32(A * L) / vol)
    return dict(length=L, time=T, field=B, edens=E)


def thermal_k(msat, aexch, alpha, cell, temperature):
    """sigma^2 dt (internal units) of the thermal field at 'temperature'
    kelvin: sigma = sqrt(2 alpha kB T / (gamma0 mu0 Ms V dt_SI)) / Ms
    (src/go/sim/temperature.go:27-36), dt_SI = dt * unit time."""
    u = units(msat, aexch)
    kB, gamma0, mu0 = 1.380650424e-23, 2.211e5, 4.0e-7 * np.pi
    V = float(cell[0]) * float(cell[1]) * float(cell[2])
    return float(2.0 * alpha * kB * temperature / (gamma0 * mu0 * msat * V * float(u["time"])) / (msat * msat))


def mmx_params(grid, cell, msat, aexch, alpha, bext=(0, 0, 0), solver="heun", dt=0.0, maxerror=0.0, anis=0,
               k1=0.0, axis=(0, 0, 1), periodic=(0, 0, 0), faithful=1, exch_type=6, precision=0, temperature=0.0,
               thermal_seed=0):
    """Builds mmx_params from the reference's user-level (SI, user x,y,z)
    inputs with the same float32 conversions as the Go driver."""
    u = units(msat, aexch)
    p = MmxParams()
    for d in range(3):
        p.size[d] = grid[2 - d]
        p.periodic[d] = periodic[2 - d]
        p.cellsize[d] = f32(f32(cell[2 - d]) / u["length"])
        p.hext[d] = f32(f32(bext[2 - d]) / u["field"])
    p.alpha = f32(alpha)
    p.anis_type = anis
    if anis == 1:
        p.anis_k = f32(f32(k1) / u["edens"])
        ux, uy, uz = f32(axis[2]), f32(axis[1]), f32(axis[0])
        nn = f32(np.sqrt(np.float64(f32(f32(f32(ux * ux) + f32(uy * uy)) + f32(uz * uz)))))
        p.anis_axis[0], p.anis_axis[1], p.anis_axis[2] = f32(ux / nn), f32(uy / nn), f32(uz / nn)
    p.solver = SOLVERS[solver]
    dti = f32(f32(dt) / u["time"])
    p.dt = dti if dti != 0 else f32(1e-4)
    p.max_error = maxerror
    p.unit_time = u["time"]
    p.exch_type = exch_type
    p.faithful = faithful
    p.accuracy = 8
    p.precision = precision
    p.thermal_k = thermal_k(msat, aexch, alpha, cell, temperature) if temperature else 0.0
    p.thermal_seed = thermal_seed
    return p


class Solver:
    """The fused solver (mmx_solver_*), state resident on the device."""

    def __init__(self, params):
        self.params = params
        self.h = ctypes.c_void_p()
        _check(lib().mmx_solver_create(ctypes.byref(params), ctypes.byref(self.h)))
        self.N = (params.size[0], params.size[1], params.size[2])
        self.n = self.N[0] * self.N[1] * self.N[2]

    def close(self):
        if self.h:
            lib().mmx_solver_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_m(self, m, stream=None):
        a = np.ascontiguousarray(m, dtype=np.float32)
        assert a.size == 3 * self.n
        _check(lib().mmx_solver_set_m(self.h, a.ctypes.data, 1, stream))

    def set_m_device(self, ptr, stream=None):
        _check(lib().mmx_solver_set_m(self.h, ptr, 0, stream))

    def get_m(self, stream=None):
        out = np.empty((3,) + self.N, dtype=np.float32)
        _check(lib().mmx_solver_get_m(self.h, out.ctypes.data, 1, stream))
        return out

    def normalize(self, stream=None):
        _check(lib().mmx_solver_normalize(self.h, stream))

    def step(self, n=1, stream=None):
        _check(lib().mmx_solver_step(self.h, n, stream))

    def field(self, m_ptr, h_ptr, stream=None):
        _check(lib().mmx_solver_field(self.h, m_ptr, h_ptr, stream))

    def avg_m(self, out_ptr=None, on_host=True, stream=None):
        """<m> per internal component; into out_ptr (host or device) or a
        new numpy array (synchronous)."""
        if out_ptr is None:
            out = np.zeros(3, np.float32)
            _check(lib().mmx_solver_avg_m(self.h, out.ctypes.data, 1, stream))
            import torch
            torch.cuda.synchronize()
            return out
        _check(lib().mmx_solver_avg_m(self.h, out_ptr, 1 if on_host else 0, stream))

    def state(self):
        t, dt, tq, er, st = ctypes.c_double(), ctypes.c_float(), ctypes.c_float(), ctypes.c_float(), ctypes.c_longlong()
        _check(lib().mmx_solver_state(self.h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(tq), ctypes.byref(er),
                                      ctypes.byref(st)))
        return dict(time=t.value, dt=dt.value, torque=tq.value, error=er.value, steps=st.value)

    def energy(self, stream=None):
        """Total energy of m, internal units (mmx_solver_energy)."""
        e = ctypes.c_double()
        _check(lib().mmx_solver_energy(self.h, ctypes.byref(e), stream))
        return e.value

    def relax(self, max_steps=1000000, stream=None):
        """Sim.Relax: returns (steps taken, last energy) (mmx_solver_relax)."""
        k, e = ctypes.c_longlong(), ctypes.c_float()
        _check(lib().mmx_solver_relax(self.h, max_steps, ctypes.byref(k), ctypes.byref(e), stream))
        return k.value, e.value

    def run(self, seconds, period, max_rows=100000, max_steps=0, stream=None):
        """Sim.Run for 'seconds' with a table row every 'period' seconds:
        returns an (nrows, 7) array {t, <m> (user x,y,z), torque, min m_z,
        max m_z} (mmx_solver_run)."""
        rows = np.zeros((max(max_rows, 1), 7), np.float32)
        n = ctypes.c_int()
        _check(lib().mmx_solver_run(self.h, seconds, period, rows.ctypes.data, max_rows, ctypes.byref(n), max_steps,
                                    stream))
        return rows[:n.value]

    def m_device(self):
        return lib().mmx_solver_m_device(self.h)

    def use_graph(self, on=True):
        _check(lib().mmx_solver_use_graph(self.h, 1 if on else 0))

    def device_control(self, on=True):
        """Adaptive RK: dt controller on the device; step(n) = n trials."""
        _check(lib().mmx_solver_device_control(self.h, 1 if on else 0))

    def profile(self, on=True):
        _check(lib().mmx_solver_profile(self.h, 1 if on else 0))

    def pass_times(self):
        names = (ctypes.c_char * 32 * 32)()
        ms = (ctypes.c_double * 32)()
        la = (ctypes.c_longlong * 32)()
        n = ctypes.c_int()
        _check(lib().mmx_solver_pass_times(self.h, 32, names, ms, la, ctypes.byref(n)))
        return {names[i].value.decode(): (ms[i], la[i]) for i in range(n.value)}


class _InstanceView(Solver):
    """A solver owned by a batch (not destroyed on its own)."""

    def __init__(self, handle, params):
        self.params = params
        self.h = ctypes.c_void_p(handle)
        self.N = (params.size[0], params.size[1], params.size[2])
        self.n = self.N[0] * self.N[1] * self.N[2]

    def close(self):
        self.h = ctypes.c_void_p()


class Batch:
    """Many independent instances advanced together (mmx_batch_*)."""

    def __init__(self, params_list):
        arr = (MmxParams * len(params_list))(*params_list)
        self.h = ctypes.c_void_p()
        _check(lib().mmx_batch_create(arr, len(params_list), ctypes.byref(self.h)))
        self.params = list(params_list)
        self.instances = [_InstanceView(lib().mmx_batch_instance(self.h, i), p) for i, p in enumerate(params_list)]

    def close(self):
        if self.h:
            for v in self.instances:
                v.close()
            lib().mmx_batch_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def size(self):
        c, cells, la = ctypes.c_int(), ctypes.c_longlong(), ctypes.c_int()
        _check(lib().mmx_batch_size(self.h, ctypes.byref(c), ctypes.byref(cells), ctypes.byref(la)))
        return dict(count=c.value, cells=cells.value, launches_per_step=la.value)

    def step(self, n=1, stream=None):
        _check(lib().mmx_batch_step(self.h, n, stream))

    def use_graph(self, on=True):
        _check(lib().mmx_batch_use_graph(self.h, 1 if on else 0))


def batch_tuning():
    """The autotuner's decisions for the batched Y passes: one dict per
    (line length, direction) with both tile widths, their measured launch
    times (ms) and the width kept."""
    n = ctypes.c_int()
    _check(lib().mmx_batch_tuning(0, None, None, ctypes.byref(n)))
    rows = np.zeros((max(n.value, 1), 5), np.int32)
    ms = np.zeros((max(n.value, 1), 2), np.float32)
    _check(lib().mmx_batch_tuning(n.value, rows.ctypes.data, ms.ctypes.data, ctypes.byref(n)))
    return [dict(L=int(r[0]), inverse=bool(r[1]), widths=(int(r[2]), int(r[3])), ms=(float(m[0]), float(m[1])),
                 chosen=int(r[3] if r[4] else r[2]))
            for r, m in zip(rows[:n.value], ms[:n.value])]


def batch_config(count, seed=4, cell=3e-9, solver="rk4", dt=5e-15):
    """The batch configuration: count instances with Nx, Ny drawn from
    {32,48,64,96,128,192,256}, Nz from {1,2,4}, Ms ~ U[4e5,1.4e6] A/m,
    A ~ U[5e-12,2e-11] J/m, alpha ~ U[0.01,0.5], a uniform field of random
    direction and |B| ~ U[0,100] mT, cubic cells of 3 nm; returns the user
    level descriptions (per-instance draw order: Nx, Ny, Nz, Ms, A, alpha,
    field direction (3 normals), |B|)."""
    rng = np.random.default_rng(seed)
    sizes = [32, 48, 64, 96, 128, 192, 256]
    out = []
    for _ in range(count):
        nx = int(rng.choice(sizes))
        ny = int(rng.choice(sizes))
        nz = int(rng.choice([1, 2, 4]))
        ms = float(rng.uniform(4e5, 1.4e6))
        a = float(rng.uniform(5e-12, 2e-11))
        alpha = float(rng.uniform(0.01, 0.5))
        d = rng.standard_normal(3)
        d = d / np.linalg.norm(d)
        bmag = float(rng.uniform(0.0, 0.1))
        out.append(dict(grid=(nx, ny, nz), cell=(cell, cell, cell), msat=ms, aexch=a, alpha=alpha,
                        bext=tuple(float(x) for x in bmag * d), solver=solver, dt=dt))
    return out


def write_ovf(path, m, cell, version=2, binary=True, valueunit="A/m", multiplier=1.0, stage_time=0.0,
              total_time=0.0):
    """Writes m ([3][X][Y][Z], internal order) as an OVF file; cell is the
    internal (X, Y, Z) cell size in metres (mmx_write_ovf)."""
    a = np.ascontiguousarray(m, dtype=np.float32)
    size = (ctypes.c_int * 3)(*a.shape[1:])
    cs = (ctypes.c_double * 3)(*[float(c) for c in cell])
    _check(lib().mmx_write_ovf(os.fsencode(path), a.ctypes.data, size, cs, version, 1 if binary else 0,
                               valueunit.encode(), multiplier, stage_time, total_time))


def write_odt(path, rows, title="mumax data"):
    """Writes table rows of Solver.run as an ODT 1.0 file (mmx_write_odt)."""
    r = np.ascontiguousarray(rows, dtype=np.float32).reshape(-1, 7)
    _check(lib().mmx_write_odt(os.fsencode(path), r.ctypes.data, r.shape[0], title.encode()))


# --------------------------------------------------------------------------
# Serving form (mmx_server_*)
# --------------------------------------------------------------------------
REQ_STATES = {0: "queued", 1: "active", 2: "done", 3: "failed"}


def footprint(params):
    """Device bytes a resident solve with these parameters holds."""
    b = ctypes.c_size_t()
    _check(lib().mmx_server_footprint(ctypes.byref(params), ctypes.byref(b)))
    return b.value


class Server:
    """The request loop with continuous batching (batched=True) or one solve
    at a time on the single-instance solver (batched=False)."""

    def __init__(self, batched=True, check_every=100, hbm_budget=0, max_active=0, keep_m=False, stream=None):
        c = MmxServerConfig()
        c.hbm_budget, c.max_active, c.check_every = int(hbm_budget), int(max_active), int(check_every)
        c.batched, c.keep_m = 1 if batched else 0, 1 if keep_m else 0
        self.h = ctypes.c_void_p()
        _check(lib().mmx_server_create(ctypes.byref(c), stream, ctypes.byref(self.h)))
        self.npoints = {}
        self.sizes = {}

    def close(self):
        if self.h:
            lib().mmx_server_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, params, m0, fields=None, max_torque=1e-4, max_steps=0):
        """Queues one solve.  m0: internal [3][X][Y][Z] float32; fields: None
        (relax under params.hext) or an (npoints, 3) array of internal fields."""
        r = MmxRequest()
        r.params = params
        m0 = np.ascontiguousarray(m0, dtype=np.float32)
        r.m0 = m0.ctypes.data
        f = None
        if fields is None:
            r.npoints = 1
        else:
            f = np.ascontiguousarray(fields, dtype=np.float32).reshape(-1, 3)
            r.npoints = f.shape[0]
            r.hext_points = f.ctypes.data
        r.max_torque = max_torque
        r.max_steps = max_steps
        rid = ctypes.c_longlong()
        _check(lib().mmx_server_submit(self.h, ctypes.byref(r), ctypes.byref(rid)))
        self.npoints[rid.value] = r.npoints
        self.sizes[rid.value] = tuple(params.size)
        return rid.value

    def pump(self):
        a, q = ctypes.c_int(), ctypes.c_int()
        _check(lib().mmx_server_pump(self.h, ctypes.byref(a), ctypes.byref(q)))
        return a.value, q.value

    def result(self, rid):
        res = MmxResult()
        npts = self.npoints[rid]
        avg = np.zeros((npts, 3), np.float32)
        ps = np.zeros(npts, np.int64)
        _check(lib().mmx_server_result(self.h, rid, ctypes.byref(res), avg.ctypes.data, ps.ctypes.data))
        k = res.points_done
        return dict(state=REQ_STATES[res.state], converged=bool(res.converged), steps=res.steps, points_done=k,
                    t_submit=res.t_submit, t_admit=res.t_admit, t_done=res.t_done, footprint=res.footprint,
                    avg_m=avg[:k], point_steps=ps[:k])

    def result_m(self, rid):
        N = self.sizes[rid]
        m = np.empty((3,) + N, np.float32)
        _check(lib().mmx_server_result_m(self.h, rid, m.ctypes.data))
        return m

    def release(self, rid):
        _check(lib().mmx_server_release(self.h, rid))
        self.npoints.pop(rid, None)
        self.sizes.pop(rid, None)

    def clock(self):
        return lib().mmx_server_clock(self.h)

    def stats(self):
        u, c, g = ctypes.c_size_t(), ctypes.c_longlong(), ctypes.c_longlong()
        _check(lib().mmx_server_stats(self.h, ctypes.byref(u), ctypes.byref(c), ctypes.byref(g)))
        return dict(used_bytes=u.value, chunks=c.value, regroups=g.value)


def sweep_fields(msat, aexch, b0, b1, points):
    """Internal fields of a sweep from b0 to b1 (user x,y,z, tesla) in
    points-1 intervals: b = b0 + (b1-b0)*float32(i)/float32(points-1) in
    float32 (simhysteresis.go:18-24), then the ApplyStatic conversion to
    internal units and axes (simfield.go:87-98)."""
    u = units(msat, aexch)
    steps = f32(points - 1)
    out = np.zeros((points, 3), np.float32)
    for i in range(points):
        frac = f32(f32(i) / steps)
        for d in range(3):
            b = f32(f32(b0[d]) + f32(f32(f32(b1[d]) - f32(b0[d])) * frac))
            out[i, 2 - d] = f32(b / u["field"])
    return out


def stable_dt(grid, cell, msat, aexch, alpha, bmag=0.0, safety=2.0):
    """A fixed RK4 time step (s) inside the stability region of the
    linearised LLG operator: the six-neighbour exchange Laplacian's largest
    eigenvalue sum_d 4/c_d^2 (internal cell sizes, axes with more than one
    cell), plus 1 for the demagnetising field and |B| in internal units; the
    LLG eigenvalues have modulus lambda/sqrt(1+alpha^2), and RK4 is stable
    up to about 2.8 along the directions they take, so dt = safety *
    sqrt(1+alpha^2) / lambda internal time units."""
    u = units(msat, aexch)
    L = float(u["length"])
    lam = sum(4.0 / (c / L) ** 2 for c, n in zip(cell, grid) if n > 1)
    lam += 1.0 + bmag / float(u["field"])
    return safety * float(np.sqrt(1.0 + alpha * alpha)) / lam * float(u["time"])


def serve_stream(count, seed=5, rate=200.0, cell=3e-9, dt=None, sweep_points=21, sweep_fraction=0.5,
                 bmax=0.1):
    """The serving workload: a Poisson stream (rate requests/s) of
    relaxations (alpha = 1, under a uniform field drawn as in the batch
    configuration) and field sweeps (alpha = 1, B along user x from -bmax to
    +bmax tesla in sweep_points points), sizes and materials drawn as in
    batch_config, random unit m per cell.  dt: a fixed step in seconds, or
    None for each request's stable_dt (the relaxation is a steady state, so
    the step only sets how many steps it takes).  Per request, in order: the
    inter-arrival gap, the kind, then the batch_config draws; m comes from
    its own generator seeded (seed, index).  Returns dicts with 'arrival'
    (s), 'kind', 'cfg' (user-level) and 'fields' (None or internal)."""
    rng = np.random.default_rng(seed)
    sizes = [32, 48, 64, 96, 128, 192, 256]
    t = 0.0
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        sweep = bool(rng.uniform() < sweep_fraction)
        nx = int(rng.choice(sizes))
        ny = int(rng.choice(sizes))
        nz = int(rng.choice([1, 2, 4]))
        ms = float(rng.uniform(4e5, 1.4e6))
        a = float(rng.uniform(5e-12, 2e-11))
        float(rng.uniform(0.01, 0.5))  # the batch alpha draw, kept for the draw order; relaxations use alpha = 1
        d = rng.standard_normal(3)
        d = d / np.linalg.norm(d)
        bmag = float(rng.uniform(0.0, bmax))
        step = dt if dt is not None else stable_dt((nx, ny, nz), (cell, cell, cell), ms, a, 1.0,
                                                   bmax if sweep else bmag)
        cfg = dict(grid=(nx, ny, nz), cell=(cell, cell, cell), msat=ms, aexch=a, alpha=1.0,
                   bext=(0.0, 0.0, 0.0) if sweep else tuple(float(x) for x in bmag * d), solver="rk4", dt=step)
        fields = sweep_fields(ms, a, (-bmax, 0.0, 0.0), (bmax, 0.0, 0.0), sweep_points) if sweep else None
        if sweep:
            cfg["bext"] = (-bmax, 0.0, 0.0)
        out.append(dict(index=i, arrival=t, kind="sweep" if sweep else "relax", cfg=cfg, fields=fields,
                        m_seed=(seed, i)))
    return out


def stream_m0(req):
    """Random unit m per cell (internal layout) of a serve_stream request."""
    nx, ny, nz = req["cfg"]["grid"]
    g = np.random.default_rng(list(req["m_seed"]))
    u = g.standard_normal((3, nz, ny, nx))
    u /= np.sqrt((u * u).sum(axis=0, keepdims=True))
    return np.ascontiguousarray(u[::-1].astype(np.float32))


def partition_requests(reqs, world):
    """Rank of every request when the stream is spread over 'world' GPUs:
    in arrival order, each request goes to the rank with the least device
    bytes x field points assigned so far (ties to the lowest rank).  Every
    rank computes the same partition; there is no data exchange."""
    load = [0] * world
    out = []
    for r in sorted(reqs, key=lambda q: q["arrival"]):
        w = footprint(mmx_params(**r["cfg"])) * (1 if r["fields"] is None else len(r["fields"]))
        k = min(range(world), key=lambda i: (load[i], i))
        load[k] += w
        out.append((r["index"], k))
    ranks = dict(out)
    return [ranks[r["index"]] for r in reqs]


def serve_share(reqs, rank, world, make_server, gather=None, **run_kw):
    """The multi-GPU serving form: every rank computes the same partition
    (partition_requests), serves its share on its own server (make_server()
    builds it; run_stream drives it) and the results are gathered on rank 0
    by 'gather' (a torch.distributed gather_object to rank 0 when None and
    world > 1).  No collective touches the solves' data.  Returns the
    results of every request sorted by index on rank 0, None on the others."""
    part = partition_requests(reqs, world)
    mine = [r for r, k in zip(reqs, part) if k == rank]
    server = make_server()
    try:
        res = run_stream(server, mine, **run_kw)
    finally:
        close = getattr(server, "close", None)
        if close:
            close()
    for r in res:
        r["rank"] = rank
    if world == 1:
        return res
    if gather is None:
        import torch.distributed as dist
        got = [None] * world if rank == 0 else None
        dist.gather_object(res, got, dst=0)
    else:
        got = gather(res)
    if rank != 0:
        return None
    return sorted((r for part_res in got for r in part_res), key=lambda x: x["index"])


def run_stream(server, reqs, realtime=True, max_torque=1e-4, max_steps=0, poll=0.0005):
    """Drives a Server with the requests' arrival times: each request is
    submitted once the server clock passes its arrival (all at once when
    realtime is False) and the loop pumps while work is resident or queued.
    Returns per-request results with latency = completion - arrival."""
    t0 = server.clock()
    pending = sorted(reqs, key=lambda r: r["arrival"])
    ids = {}
    k = 0
    while True:
        now = server.clock() - t0
        while k < len(pending) and (not realtime or pending[k]["arrival"] <= now):
            r = pending[k]
            p = mmx_params(**r["cfg"])
            ids[server.submit(p, stream_m0(r), r["fields"], max_torque, max_steps)] = r
            k += 1
        active, queued = server.pump()
        if active == 0 and queued == 0:
            if k == len(pending):
                break
            wait = pending[k]["arrival"] - (server.clock() - t0)
            if wait > 0:
                time.sleep(min(wait, poll) if poll else wait)
    out = []
    for rid, r in ids.items():
        res = server.result(rid)
        res["id"] = rid
        res["index"] = r["index"]
        res["kind"] = r["kind"]
        res["arrival"] = r["arrival"] if realtime else 0.0
        res["latency"] = res["t_done"] - t0 - res["arrival"]
        out.append(res)
    return sorted(out, key=lambda x: x["index"])


def face_kernel6_device(P, periodic, cellsize, exch6=True, accuracy=8, out_ptr=None, stream=None):
    """Runs mmx_face_kernel6 into a device buffer of 6*P0*P1*P2 floats."""
    Pa = (ctypes.c_int * 3)(*P)
    pa = (ctypes.c_int * 3)(*periodic)
    ca = (ctypes.c_float * 3)(*[float(c) for c in cellsize])
    _check(lib().mmx_face_kernel6(Pa, pa, ca, accuracy, 1 if exch6 else 0, out_ptr, stream))


def driver_config(grid, cell, msat, aexch, alpha, bext=(0, 0, 0), solver="heun", dt=0.0, maxerror=0.0, anis=0,
                  k1=0.0, axis=(0, 0, 1), periodic=(0, 0, 0), faithful=1, mindm=0.0, maxdm=0.0, mindt=0.0,
                  maxdt=0.0):
    c = DriverConfig()
    c.grid[:] = list(grid)
    c.cell[:] = list(cell)
    c.periodic[:] = list(periodic)
    c.msat, c.aexch, c.alpha = msat, aexch, alpha
    c.bext[:] = list(bext)
    c.anis_type, c.k1 = anis, k1
    c.anis_axis[:] = list(axis)
    c.solver = SOLVERS[solver]
    c.dt, c.maxerror = dt, maxerror
    c.mindm, c.maxdm, c.mindt, c.maxdt = mindm, maxdm, mindt, maxdt
    c.faithful = faithful
    return c


class DriverSim:
    """The Go-driver restatement (libmmxdriver.so) over a libgpukern
    implementation given by path (the B200 engine by default)."""

    def __init__(self, cfg, m_internal, k6, libpath=LIB_PATH):
        D = driver()
        self.L = D.mmxd_open(libpath.encode())
        if not self.L:
            raise MmxError("mmxd_open(%s): %s" % (libpath, D.mmxd_last_error().decode()))
        self.m0 = np.ascontiguousarray(m_internal, dtype=np.float32)
        self.k6 = np.ascontiguousarray(k6, dtype=np.float32)
        self.h = D.mmxd_new(self.L, ctypes.byref(cfg), self.m0.ctypes.data, self.k6.ctypes.data)
        if not self.h:
            raise MmxError("mmxd_new: %s" % D.mmxd_last_error().decode())
        N = (ctypes.c_int * 3)()
        P = (ctypes.c_int * 3)()
        D.mmxd_sizes(self.h, N, P)
        self.N, self.P = tuple(N), tuple(P)

    def close(self):
        D = driver()
        if getattr(self, "h", None):
            D.mmxd_free(self.h)
            self.h = None
        if getattr(self, "L", None):
            D.mmxd_close(self.L)
            self.L = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def steps(self, n):
        rc = driver().mmxd_steps(self.h, n)
        if rc:
            raise MmxError(driver().mmxd_last_error().decode())

    def run(self, seconds):
        rc = driver().mmxd_run(self.h, seconds)
        if rc:
            raise MmxError(driver().mmxd_last_error().decode())

    def m(self):
        out = np.empty((3,) + self.N, dtype=np.float32)
        driver().mmxd_get_m(self.h, out.ctypes.data)
        return out

    def set_m(self, m):
        a = np.ascontiguousarray(m, dtype=np.float32)
        driver().mmxd_set_m(self.h, a.ctypes.data)

    def heff(self, m):
        a = np.ascontiguousarray(m, dtype=np.float32)
        out = np.empty_like(a)
        driver().mmxd_heff(self.h, a.ctypes.data, out.ctypes.data)
        return out

    def avg_m(self):
        out = np.zeros(3, np.float32)
        driver().mmxd_avg_m(self.h, out.ctypes.data)
        return out

    def time(self):
        return driver().mmxd_time(self.h)

    def dt(self):
        return driver().mmxd_dt(self.h)

    def torque(self):
        return driver().mmxd_torque(self.h)

    def step_error(self):
        return driver().mmxd_step_error(self.h)

    def steps_taken(self):
        return driver().mmxd_step_count(self.h)

    def energy(self, m=None):
        """Total energy (internal units) of m (default: the current m)."""
        a = np.ascontiguousarray(self.m() if m is None else m, dtype=np.float32)
        e = ctypes.c_float()
        rc = driver().mmxd_energy(self.h, a.ctypes.data, ctypes.byref(e))
        if rc:
            raise MmxError(driver().mmxd_last_error().decode())
        return e.value

    def run_table(self, seconds, period, max_rows=100000):
        """Sim.Run with a table row every 'period' seconds (7 floats per
        row, as Solver.run)."""
        rows = np.zeros((max(max_rows, 1), 7), np.float32)
        n = ctypes.c_int()
        rc = driver().mmxd_run_table(self.h, seconds, period, rows.ctypes.data, max_rows, ctypes.byref(n))
        if rc:
            raise MmxError(driver().mmxd_last_error().decode())
        return rows[:n.value]
