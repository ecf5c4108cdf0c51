"""The demag kernel restatement against an independent closed form.

FaceKernel6 (demag.go:26-84, faceIntegral demag.go:142-183) puts n x n point
charges on the two charged faces of a cell magnetised along s and sums their
Coulomb fields at the centre of the target cell.  As n grows this converges
to the field of two uniformly charged rectangles, which has a closed form
(the corner formulas of the rectangle's solid angle and of the integrals of
1/r^2 over it, as used for the demag tensor of a cuboid by Newell, Williams
and Dunlop, J. Geophys. Res. 98 (1993) 9551).  The oracle's FP64 restatement
(which the GPU kernel build matches bit for bit in FP32) must converge to it
at second order in 1/n, and the field at a cell's own centre must have trace
-1 (the charged faces of a closed surface subtend the full solid angle).
The reference's Go kernel generator cannot run here, so this pins the
restatement's physics rather than the reference's output."""
import numpy as np
import pytest

import oracle as O

KIDX = [[0, 5, 4], [5, 1, 3], [4, 3, 2]]  # XX, YY, ZZ, YZ, XZ, XY (kernel.go:95-98)


def plate_field(p, u, u0, lo, hi):
    """Field at p of the rectangle {x_u = u0, lo <= (x_v, x_w) <= hi},
    v = u + 1, w = u + 2 (mod 3), with unit surface charge and Coulomb law
    1 / (4 pi r^2): sums over the four corners."""
    v, w = (u + 1) % 3, (u + 2) % 3
    x = p[u] - u0
    e = np.zeros(3)
    for xv, sv in ((lo[0], -1.0), (hi[0], 1.0)):
        for xw, sw in ((lo[1], -1.0), (hi[1], 1.0)):
            xi, eta = xv - p[v], xw - p[w]
            r = np.sqrt(x * x + xi * xi + eta * eta)
            s = sv * sw
            if x != 0.0:
                e[u] += s * np.arctan(xi * eta / (x * r))
            e[v] += s * np.log(eta + r)
            e[w] += s * np.log(xi + r)
    return e / (4.0 * np.pi)


def cell_field(r, cs):
    """K[s][d]: component d of the field at r of a cell centred at the
    origin, uniformly magnetised with M = 1 along s (faces at +-cs[s]/2
    carrying charge +-1)."""
    k = np.zeros((3, 3))
    for s in range(3):
        v, w = (s + 1) % 3, (s + 2) % 3
        lo, hi = (-cs[v] / 2, -cs[w] / 2), (cs[v] / 2, cs[w] / 2)
        k[s] = plate_field(r, s, cs[s] / 2, lo, hi) - plate_field(r, s, -cs[s] / 2, lo, hi)
    return k


def test_plate_field_against_quadrature():
    """The closed form itself against a fine midpoint quadrature."""
    p = np.array([0.7, 0.3, -0.4])
    lo, hi = (-0.5, -0.25), (0.5, 0.6)
    n = 1500
    pv = lo[0] + (np.arange(n) + 0.5) * (hi[0] - lo[0]) / n
    pw = lo[1] + (np.arange(n) + 0.5) * (hi[1] - lo[1]) / n
    gv, gw = np.meshgrid(pv, pw, indexing="ij")
    d = np.stack([np.full_like(gv, p[0] - 0.2), p[1] - gv, p[2] - gw])
    r3 = np.sqrt((d * d).sum(0)) ** 3
    q = (d / r3).sum(axis=(1, 2)) * (hi[0] - lo[0]) * (hi[1] - lo[1]) / n / n / (4 * np.pi)
    assert np.abs(plate_field(p, 0, 0.2, lo, hi) - q).max() < 1e-6


OFFSETS = [(0, 0, 0), (1, 0, 0), (0, 1, 1), (2, 1, 0), (3, -2, 1), (7, 7, -7)]


@pytest.mark.parametrize("cs", [(1.0, 1.0, 1.0), (3.0, 3.90625, 3.90625), (4.0, 2.0, 1.0)])
def test_face_kernel_converges_to_cuboid_field(cs):
    P = (16, 16, 16)
    err = {}
    for acc in (8, 64):
        k = O.face_kernel6(P, cs, accuracy=acc, bits=64)
        worst = 0.0
        for off in OFFSETS:
            a = cell_field(np.array(off, dtype=np.float64) * np.array(cs), cs)
            g = np.array([[k[KIDX[s][d]][off[0] % 16][off[1] % 16][off[2] % 16] for d in range(3)]
                          for s in range(3)])
            worst = max(worst, float(np.abs(g - a).max() / np.abs(a).max()))
        err[acc] = worst
    # 8 x 8 charges per face (the reference's default accuracy): < 1%;
    # 64 x 64: < 2e-4; the error falls as 1/n^2 (64x for 8 -> 64)
    assert err[8] < 1e-2, err
    assert err[64] < 2e-4, err
    assert err[8] / err[64] > 30, err


@pytest.mark.parametrize("cs", [(1.0, 1.0, 1.0), (3.0, 3.90625, 3.90625), (4.0, 2.0, 1.0)])
def test_self_field_trace(cs):
    a = cell_field(np.zeros(3), cs)
    assert abs(np.trace(a) + 1.0) < 1e-12
    assert np.abs(a - np.diag(np.diag(a))).max() < 1e-12  # no off-diagonal self field
    k = O.face_kernel6((4, 4, 4), cs, accuracy=64, bits=64)
    tr = k[0][0][0][0] + k[1][0][0][0] + k[2][0][0][0]
    assert abs(tr + 1.0) < 1e-4, tr
