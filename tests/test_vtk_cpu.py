"""The headless VTK writer (no GPU): the .vts file parses back to the same
node coordinates, TimeValue and cell arrays."""
import re
import struct

import numpy as np

from curvilineardiffusionmanuscript_b200.mesh import wavy_mesh_2d, wavy_mesh_3d
from curvilineardiffusionmanuscript_b200.vtk import filename, write_vts


def read_vts(path):
    raw = open(path, "rb").read()
    head, _, rest = raw.partition(b'<AppendedData encoding="raw">')
    text = head.decode()
    data = rest[rest.index(b"_") + 1:]
    tv = float(re.search(r'Name="TimeValue"[^>]*>([^<]+)<', text).group(1))
    ext = [int(v) for v in re.search(r'WholeExtent="([^"]+)"', text).group(1).split()]
    arrays = {}
    for m in re.finditer(r'<DataArray type="(Float32|Float64)"(?: Name="([^"]+)")?[^>]*offset="(\d+)"', text):
        dt = np.float32 if m.group(1) == "Float32" else np.float64
        off = int(m.group(3))
        n = struct.unpack("<Q", data[off:off + 8])[0]
        arrays[m.group(2) or "Points"] = np.frombuffer(data[off + 8:off + 8 + n], dtype=dt)
    return tv, ext, arrays


def test_vts_roundtrip_2d(tmp_path):
    m = wavy_mesh_2d(12, 9, 0.05)
    rng = np.random.default_rng(0)
    u = rng.normal(size=(9, 12))
    q1 = rng.normal(size=(9, 12))
    p = write_vts(str(tmp_path / "a.vts"), m.nodes, {"u": u, "q1": q1}, 1.25e-5, dtype=np.float64)
    tv, ext, arr = read_vts(p)
    assert tv == 1.25e-5 and ext == [0, 12, 0, 9, 0, 0]
    pts = arr["Points"].reshape(-1, 3)
    assert np.array_equal(pts[:, 0], m.nodes[0].numpy().reshape(-1))
    assert np.array_equal(pts[:, 1], m.nodes[1].numpy().reshape(-1))
    assert np.array_equal(arr["u"], u.reshape(-1)) and np.array_equal(arr["q1"], q1.reshape(-1))


def test_vts_roundtrip_3d_float32(tmp_path):
    m = wavy_mesh_3d(5, 4, 3, 0.04)
    u = np.arange(60, dtype=np.float64).reshape(3, 4, 5)
    tv, ext, arr = read_vts(write_vts(str(tmp_path / "b.vts"), m.nodes, {"u": u}, 0.5))
    assert ext == [0, 5, 0, 4, 0, 3]
    assert arr["Points"].dtype == np.float32 and arr["Points"].size == 6 * 5 * 4 * 3
    assert np.array_equal(arr["u"], u.reshape(-1).astype(np.float32))


def test_reference_file_names():
    assert filename(12, "gaussian run") == "gaussian_run_0000012.vts"
    assert filename(0) == "diffusion_0000000.vts"
