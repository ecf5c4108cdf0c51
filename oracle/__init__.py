"""CPU oracle for the LLG hot path -- TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``liboracle32.so`` (FP32 build: each float32 operation of
the reference, in the reference's order, one rounding per operation) and
``liboracle64.so`` (the same code in float64).  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may use
this module, and only as the checker.  The product library never imports it.

The C source ``oracle.c`` cites the reference file:line each function follows.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

SOLVERS = {"heun": 0, "rk12": 1, "rk23": 2, "rk4": 3, "rkck": 4, "rkdp": 5, "rk2": 6}


class OCfg(ctypes.Structure):
    _fields_ = [
        ("grid", ctypes.c_int * 3),
        ("cell", ctypes.c_double * 3),
        ("periodic", ctypes.c_int * 3),
        ("msat", ctypes.c_double),
        ("aexch", ctypes.c_double),
        ("alpha", ctypes.c_double),
        ("bext", ctypes.c_double * 3),
        ("anis", ctypes.c_int),
        ("k1", ctypes.c_double),
        ("axis", ctypes.c_double * 3),
        ("solver", ctypes.c_int),
        ("dt", ctypes.c_double),
        ("maxerror", ctypes.c_double),
        ("mindm", ctypes.c_double),
        ("maxdm", ctypes.c_double),
        ("mindt", ctypes.c_double),
        ("maxdt", ctypes.c_double),
        ("exch_type", ctypes.c_int),
        ("faithful", ctypes.c_int),
        ("accuracy", ctypes.c_int),
        ("maxthreads", ctypes.c_int),
        ("temperature", ctypes.c_double),
        ("thermal_seed", ctypes.c_int),
    ]


def build():
    subprocess.check_call(["make", "-s", "-f", os.path.join(HERE, "Makefile")], cwd=HERE)


_libs = {}


def lib(bits=32):
    if bits not in _libs:
        path = os.path.join(HERE, "liboracle%d.so" % bits)
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        _libs[bits] = L
    return _libs[bits]


def _dt(bits):
    return np.float32 if bits == 32 else np.float64


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _fn(bits, name, restype=None):
    L = lib(bits)
    f = getattr(L, ("o32_" if bits == 32 else "o64_") + name)
    f.restype = restype
    return f


def make_cfg(grid, cell, msat, aexch, alpha, bext=(0, 0, 0), solver="heun", dt=0.0, maxerror=0.0,
             anis=0, k1=0.0, axis=(0, 0, 1), periodic=(0, 0, 0), faithful=1, exch_type=6,
             mindm=0.0, maxdm=0.0, mindt=0.0, maxdt=0.0, maxthreads=1024, temperature=0.0, thermal_seed=0):
    c = OCfg()
    c.grid[:] = list(grid)
    c.cell[:] = list(cell)
    c.periodic[:] = list(periodic)
    c.msat, c.aexch, c.alpha = msat, aexch, alpha
    c.bext[:] = list(bext)
    c.anis, c.k1 = anis, k1
    c.axis[:] = list(axis)
    c.solver = SOLVERS[solver]
    c.dt, c.maxerror = dt, maxerror
    c.mindm, c.maxdm, c.mindt, c.maxdt = mindm, maxdm, mindt, maxdt
    c.exch_type, c.faithful, c.accuracy, c.maxthreads = exch_type, faithful, 8, maxthreads
    c.temperature, c.thermal_seed = temperature, thermal_seed
    return c


class OracleSim:
    """The oracle's restatement of Sim (init.go, field.go, solvers)."""

    def __init__(self, cfg, m_internal, bits=32):
        self.bits = bits
        self.cfg = cfg
        dt = _dt(bits)
        self.N = (cfg.grid[2], cfg.grid[1], cfg.grid[0])
        self.n = self.N[0] * self.N[1] * self.N[2]
        m = np.ascontiguousarray(m_internal, dtype=dt).reshape(3, *self.N)
        f = _fn(bits, "sim_new", ctypes.c_void_p)
        f.argtypes = [ctypes.POINTER(OCfg), ctypes.c_void_p]
        self.h = f(ctypes.byref(cfg), _ptr(m))

    def __del__(self):
        if getattr(self, "h", None):
            _fn(self.bits, "sim_free")(ctypes.c_void_p(self.h))
            self.h = None

    def steps(self, n):
        f = _fn(self.bits, "sim_steps", ctypes.c_int)
        return f(ctypes.c_void_p(self.h), ctypes.c_int(n))

    def m(self):
        out = np.empty((3,) + self.N, dtype=_dt(self.bits))
        _fn(self.bits, "sim_get_m")(ctypes.c_void_p(self.h), _ptr(out))
        return out

    def set_m(self, m):
        a = np.ascontiguousarray(m, dtype=_dt(self.bits))
        _fn(self.bits, "sim_set_m")(ctypes.c_void_p(self.h), _ptr(a))

    def heff(self, m):
        m = np.ascontiguousarray(m, dtype=_dt(self.bits))
        h = np.empty_like(m)
        _fn(self.bits, "sim_heff")(ctypes.c_void_p(self.h), _ptr(m), _ptr(h))
        return h

    def time(self):
        return _fn(self.bits, "sim_time", ctypes.c_double)(ctypes.c_void_p(self.h))

    def dt(self):
        return _fn(self.bits, "sim_dt", ctypes.c_double)(ctypes.c_void_p(self.h))

    def unit(self, which):
        idx = {"length": 0, "time": 1, "field": 2, "edens": 3, "k": 4}[which]
        return _fn(self.bits, "sim_unit", ctypes.c_double)(ctypes.c_void_p(self.h), ctypes.c_int(idx))

    def internal_params(self):
        dt = _dt(self.bits)
        cs, hx, u, ak = (np.zeros(3, dt), np.zeros(3, dt), np.zeros(3, dt), np.zeros(2, dt))
        _fn(self.bits, "sim_internal_params")(ctypes.c_void_p(self.h), _ptr(cs), _ptr(hx), _ptr(u), _ptr(ak))
        return dict(cellsize=cs, hext=hx, axis=u, alpha=ak[0], K=ak[1])

    def avg_m(self):
        out = np.zeros(3, _dt(self.bits))
        _fn(self.bits, "sim_avg_m")(ctypes.c_void_p(self.h), _ptr(out))
        return out

    def torque(self):
        rt = ctypes.c_float if self.bits == 32 else ctypes.c_double
        return _fn(self.bits, "sim_torque", rt)(ctypes.c_void_p(self.h))

    def energy(self, m=None):
        """Total energy (internal units) of m (default: the current m):
        calcHeffEnergy + sumEdens (field.go:64-71, energy.go:49-52)."""
        m = self.m() if m is None else np.ascontiguousarray(m, dtype=_dt(self.bits))
        out = np.zeros(1, _dt(self.bits))
        f = _fn(self.bits, "sim_energy")
        f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        f(ctypes.c_void_p(self.h), _ptr(m), _ptr(out))
        return float(out[0])

    def run_table(self, seconds, period, max_rows=100000):
        """Sim.Run for 'seconds' (SI) with a table row every 'period'
        seconds (simrun.go:19-57, simoutput.go:83-85,226-272).  Rows:
        t (s), <m> (user x, y, z), last maximum torque, min and max of the
        user's m_z.  Successive calls continue the schedule."""
        if not hasattr(self, "_since"):
            self._since = np.zeros(1, np.float32)
        rows = np.zeros((max_rows, 7), np.float32)
        f = _fn(self.bits, "sim_run_table", ctypes.c_int)
        f.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_float, ctypes.c_void_p, ctypes.c_int,
                      ctypes.c_void_p]
        k = f(ctypes.c_void_p(self.h), seconds / self.unit("time"), period, _ptr(rows), max_rows,
              _ptr(self._since))
        if k < 0:
            raise RuntimeError("oracle: dt is NaN")
        return rows[:k]

    def relax(self, max_steps=1000000):
        """Sim.Relax (relax.go:14-23); returns the steps taken."""
        f = _fn(self.bits, "sim_relax", ctypes.c_longlong)
        f.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
        k = f(ctypes.c_void_p(self.h), max_steps)
        if k < 0:
            raise RuntimeError("oracle: dt is NaN")
        return k

    def last_energy(self):
        """Sim.energy: the total energy the last RK step computed."""
        return _fn(self.bits, "sim_last_energy", ctypes.c_double)(ctypes.c_void_p(self.h))

    def step_error(self):
        rt = ctypes.c_float if self.bits == 32 else ctypes.c_double
        return _fn(self.bits, "sim_step_error", rt)(ctypes.c_void_p(self.h))


def face_kernel6(P, cs, periodic=(0, 0, 0), accuracy=8, bits=32):
    dt = _dt(bits)
    k = np.zeros((6,) + tuple(P), dtype=dt)
    Pa = (ctypes.c_int * 3)(*P)
    pa = (ctypes.c_int * 3)(*periodic)
    ca = np.asarray(cs, dtype=dt)
    _fn(bits, "face_kernel6")(Pa, _ptr(ca), ctypes.c_int(accuracy), pa, _ptr(k))
    return k


def add_exch6_kernel(P, cs, k, bits=32):
    Pa = (ctypes.c_int * 3)(*P)
    ca = np.asarray(cs, dtype=_dt(bits))
    _fn(bits, "add_exch6_kernel")(Pa, _ptr(ca), _ptr(k))
    return k


def convolve(N, cs, m, periodic=(0, 0, 0), exch=True, bits=32):
    dt = _dt(bits)
    m = np.ascontiguousarray(m, dtype=dt)
    h = np.empty_like(m)
    Na = (ctypes.c_int * 3)(*N)
    pa = (ctypes.c_int * 3)(*periodic)
    ca = np.asarray(cs, dtype=dt)
    _fn(bits, "convolve_standalone")(Na, pa, _ptr(ca), ctypes.c_int(1 if exch else 0), _ptr(m), _ptr(h))
    return h


def fft_forward_padded(N, P, a, bits=32):
    dt = _dt(bits)
    a = np.ascontiguousarray(a, dtype=dt)
    out = np.empty((P[0], P[1], P[2] + 2), dtype=dt)
    _fn(bits, "fft_forward_padded")((ctypes.c_int * 3)(*N), (ctypes.c_int * 3)(*P), _ptr(a), _ptr(out))
    return out


def fft_inverse_padded(N, P, spec, bits=32):
    dt = _dt(bits)
    spec = np.ascontiguousarray(spec, dtype=dt)
    out = np.empty(tuple(N), dtype=dt)
    _fn(bits, "fft_inverse_padded")((ctypes.c_int * 3)(*N), (ctypes.c_int * 3)(*P), _ptr(spec), _ptr(out))
    return out


def delta_m(m, h, alpha, dtg, bits=32):
    dt = _dt(bits)
    m = np.ascontiguousarray(m, dtype=dt)
    h = np.array(h, dtype=dt, copy=True)
    n = m.size // 3
    f = _fn(bits, "delta_m")
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                  ctypes.c_float if bits == 32 else ctypes.c_double,
                  ctypes.c_float if bits == 32 else ctypes.c_double]
    f(_ptr(m), _ptr(h), n, alpha, dtg)
    return h


def normalize(m, bits=32):
    m = np.array(m, dtype=_dt(bits), copy=True)
    f = _fn(bits, "normalize")
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64]
    f(_ptr(m), m.size // 3)
    return m


def add_local_fields(m, h, hext, anis=0, K=0.0, u=(0, 0, 0), bits=32):
    dt = _dt(bits)
    m = np.ascontiguousarray(m, dtype=dt)
    h = np.array(h, dtype=dt, copy=True)
    he = np.asarray(hext, dtype=dt)
    ua = np.asarray(u, dtype=dt)
    f = _fn(bits, "add_local_fields")
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int,
                  ctypes.c_float if bits == 32 else ctypes.c_double, ctypes.c_void_p]
    f(_ptr(m), _ptr(h), m.size // 3, _ptr(he), anis, K, _ptr(ua))
    return h


def scale_dot_product(a, b, sc, bits=32):
    """phi = sc (a . b) per cell of two [3][N] arrays (gpu_linalg.cu:125-140)."""
    dt = _dt(bits)
    a = np.ascontiguousarray(a, dtype=dt)
    b = np.ascontiguousarray(b, dtype=dt)
    n = a.size // 3
    phi = np.empty(n, dt)
    f = _fn(bits, "scale_dot_product")
    f.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_float if bits == 32 else ctypes.c_double, ctypes.c_int64]
    f(_ptr(phi), _ptr(a), _ptr(b), sc, n)
    return phi


def add_local_fields_phi(m, h, phi, hext, anis=0, K=0.0, u=(0, 0, 0), bits=32):
    """gpu_add_local_fields_H_and_phi (uniform field): returns (h', phi')."""
    dt = _dt(bits)
    m = np.ascontiguousarray(m, dtype=dt)
    h = np.array(h, dtype=dt, copy=True)
    phi = np.array(phi, dtype=dt, copy=True)
    n = m.size // 3
    f = _fn(bits, "add_local_fields_phi")
    f.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int64, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_float if bits == 32 else ctypes.c_double, ctypes.c_void_p]
    f(_ptr(m), _ptr(h), _ptr(phi), n, _ptr(np.asarray(hext, dt)), anis, K, _ptr(np.asarray(u, dt)))
    return h, phi


def ref_sum(a, maxthreads=1024, bits=32):
    a = np.ascontiguousarray(a, dtype=_dt(bits)).ravel()
    f = _fn(bits, "ref_sum", ctypes.c_float if bits == 32 else ctypes.c_double)
    f.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int]
    return f(_ptr(a), a.size, maxthreads)


def num_threads():
    return _fn(32, "num_threads", ctypes.c_int)()


def seeded_m(grid, seed, mode="tilted"):
    """Seeded initial magnetisation in INTERNAL order [3][X][Y][Z].

    grid is the user (nx, ny, nz).  ``u = default_rng(seed).standard_normal
    ((3, nz, ny, nx))`` holds user components (x, y, z) indexed [z][y][x];
    internal component C is user component 2-C (simgeom.go:19-38,
    simget.go:25-27).  mode "tilted": normalize((1,1,1) + 0.01 u);
    mode "random": normalize(u) (independent unit vectors)."""
    nx, ny, nz = grid
    u = np.random.default_rng(seed).standard_normal((3, nz, ny, nx))
    if mode == "tilted":
        v = 1.0 + 0.01 * u
    else:
        v = u
    v = v / np.sqrt((v * v).sum(axis=0, keepdims=True))
    return np.ascontiguousarray(v[::-1]).astype(np.float32)
