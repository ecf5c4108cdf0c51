"""OVF / ODT output (mmx_write_ovf, mmx_write_odt): host code, no GPU.

A small reader restates the OVF format the reference writes and reads
(src/go/mumax/omf/output.go:41-260, input.go): header lines '# key: value',
then 'Begin: Data Binary 4' with the control number 1234567.0 first
(big-endian in OVF 1.0, little-endian in 2.0) or 'Begin: Data Text'.
Files written by the library read back bit for bit; where the reference
tree is present, the same reader also reads the reference's own s-state
fixture (selftests/s-state.omf), so reader and writer follow one format."""
import os

import numpy as np
import pytest


def read_ovf(path):
    raw = open(path, "rb").read()
    hdr = {}
    pos = 0
    while True:
        end = raw.index(b"\n", pos)
        line = raw[pos:end].decode("latin-1")
        pos = end + 1
        if not line.startswith("#"):
            continue
        body = line[1:].strip()
        if ":" not in body:
            continue
        k, v = body.split(":", 1)
        k, v = k.strip(), v.strip()
        if k.lower() == "begin" and v.lower().startswith("data"):
            kind = v[5:].strip().lower()
            break
        hdr.setdefault(k.lower(), v)
    nx, ny, nz = int(hdr["xnodes"]), int(hdr["ynodes"]), int(hdr["znodes"])
    n = nx * ny * nz
    if kind == "binary 4":
        be = "rectangular mesh v1.0" in hdr.get("oommf", "") or hdr.get("oommf", "").endswith("v1.0")
        dt = np.dtype(">f4" if be else "<f4")
        ctl = np.frombuffer(raw[pos:pos + 4], dt)[0]
        assert ctl == np.float32(1234567.0)
        vals = np.frombuffer(raw[pos + 4:pos + 4 + 12 * n], dt).astype(np.float32)
    else:
        txt = raw[pos:].decode()
        txt = txt[:txt.index("# End: Data")]
        vals = np.array(txt.split(), np.float32)
    v = vals.reshape(nz, ny, nx, 3)  # x fastest, components x, y, z per cell
    m = np.ascontiguousarray(v.transpose(3, 0, 1, 2)[::-1])  # internal [3][X=z][Y=y][Z=x]
    return hdr, m


@pytest.mark.parametrize("version,binary", [(1, True), (2, True), (1, False), (2, False)])
def test_ovf_round_trip(eng, tmp_path, version, binary):
    g = np.random.default_rng(3)
    m = g.standard_normal((3, 2, 5, 7)).astype(np.float32)
    cell = (3e-9, 4e-9, 3.90625e-9)  # internal X, Y, Z
    p = str(tmp_path / "m.ovf")
    eng.write_ovf(p, m, cell, version=version, binary=binary, valueunit="A/m", multiplier=8e5, total_time=1e-9)
    hdr, back = read_ovf(p)
    assert np.array_equal(back, m)
    assert (int(hdr["xnodes"]), int(hdr["ynodes"]), int(hdr["znodes"])) == (7, 5, 2)
    assert float(hdr["xstepsize"]) == np.float32(3.90625e-9)
    assert float(hdr["zstepsize"]) == np.float32(3e-9)
    assert np.float32(float(hdr["xmax"])) == np.float32(np.float32(3.90625e-9) * np.float32(7))


def test_odt_table(eng, tmp_path):
    rows = np.arange(21, dtype=np.float32).reshape(3, 7) / 7
    p = str(tmp_path / "t.odt")
    eng.write_odt(p, rows, title="run")
    lines = open(p).read().splitlines()
    assert lines[0] == "# ODT 1.0" and lines[-1] == "# Table End"
    cols = [c.strip() for c in lines[4].split(":", 1)[1].split("\t") if c.strip()]
    assert cols == ["Time", "Mx/Ms", "My/Ms", "Mz/Ms", "max_dm/dt", "min_Mz/Ms", "max_Mz/Ms"]
    data = np.array([[float(x) for x in ln.split()] for ln in lines[5:-1]], np.float32)
    assert np.array_equal(data, rows)


REF_FIXTURE = "/root/reference/selftests/s-state.omf"


@pytest.mark.skipif(not os.path.exists(REF_FIXTURE), reason="reference tree not present")
def test_reader_reads_the_reference_fixture(eng, tmp_path):
    """The reference's own OVF 1.0 binary file (128 x 32 x 1 s-state):
    the reader accepts it; writing the field back in the same format and
    reading it again gives the same numbers."""
    hdr, m = read_ovf(REF_FIXTURE)
    assert m.shape == (3, 1, 32, 128)
    # values are m / Ms (unit vectors), valuemultiplier = Ms
    mag = np.sqrt((m.astype(np.float64) ** 2).sum(axis=0))
    assert abs(np.median(mag) - 1.0) <= 1e-3 and float(hdr["valuemultiplier"]) == 800000.0
    p = str(tmp_path / "s.omf")
    cell = (float(hdr["zstepsize"]), float(hdr["ystepsize"]), float(hdr["xstepsize"]))
    eng.write_ovf(p, m, cell, version=1, binary=True, valueunit=hdr["valueunit"],
                  multiplier=float(hdr["valuemultiplier"]))
    h2, m2 = read_ovf(p)
    assert np.array_equal(m2, m)
    for k in ("xnodes", "ynodes", "znodes", "meshunit", "valueunit"):
        assert h2[k] == hdr[k]
    for k in ("xstepsize", "ystepsize", "zstepsize", "xmax", "ymax", "zmax"):
        assert np.float32(float(h2[k])) == np.float32(float(hdr[k]))
