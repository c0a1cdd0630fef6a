"""The CLI file formats (src/cpp/dc_cli.cpp:17-47) on the C ABI's native reader and writers:
the binary `.sdf` layout byte for byte, round trips, and the OBJ text line for line against
the reference writer's formatting (the C++ stream default: 6 significant digits, i.e. %g),
on one thread and on many."""
import os
import struct
import subprocess

import numpy as np
import pytest

from contouring_b200 import DenseSdfGrid
from contouring_b200 import io as dio


def _grid(seed=0, dims=(7, 5, 6)):
    from contouring_b200 import DenseSdfGrid
    rng = np.random.default_rng(seed)
    v = rng.normal(size=int(np.prod(dims))).astype(np.float32)
    return DenseSdfGrid(*dims, 0.125, 0.25, 0.5, -1.0, -0.75, 0.3, values=v)


def test_sdf_layout_and_round_trip(tmp_path):
    from contouring_b200 import io
    g = _grid()
    p = tmp_path / "g.sdf"
    io.write_sdf(p, g)
    raw = p.read_bytes()
    want = struct.pack("<3i6f", g.nx, g.ny, g.nz, g.vx, g.vy, g.vz, g.ox, g.oy, g.oz) + g.values.tobytes()
    assert raw == want
    h = io.read_sdf(p)
    assert (h.nx, h.ny, h.nz) == (g.nx, g.ny, g.nz)
    assert (h.vx, h.vy, h.vz, h.ox, h.oy, h.oz) == tuple(float(np.float32(x)) for x in (g.vx, g.vy, g.vz, g.ox, g.oy, g.oz))
    assert np.array_equal(h.values, g.values)


def test_sdf_errors(tmp_path):
    import ctypes
    from contouring_b200 import DcbError, _lib, io
    with pytest.raises(DcbError):
        io.read_sdf(tmp_path / "missing.sdf")
    p = tmp_path / "short.sdf"
    p.write_bytes(struct.pack("<3i6f", 4, 4, 4, 1, 1, 1, 0, 0, 0) + b"\0" * 8)
    with pytest.raises(DcbError):
        io.read_sdf(p)
    io.write_sdf(p, _grid())
    h = _lib.DcbGrid()
    buf = np.empty(10, np.float32)
    assert _lib.lib().dcb_read_sdf(bytes(p), ctypes.byref(h), buf.ctypes.data, 10) == _lib.DCB_ERR_TOO_LARGE


def _obj_text(V, F):
    lines = ["v %g %g %g" % tuple(float(x) for x in v) for v in V]
    lines += ["f " + " ".join(str(int(i) + 1) for i in f) for f in F]
    return "\n".join(lines) + "\n"


@pytest.mark.parametrize("threads", [1, 0])
@pytest.mark.parametrize("vpf", [4, 3])
def test_obj_text(tmp_path, threads, vpf):
    from contouring_b200 import io
    rng = np.random.default_rng(3)
    V = (rng.normal(size=(70000, 3)) * 10.0 ** rng.integers(-8, 6, size=(70000, 1))).astype(np.float32)
    V[:5] = [[0, -0.0, 1e-30], [1e7, -1e-7, 123456.7], [np.float32(0.1), 1 / 3, 2 / 3], [1, 2, 3], [-0.5, 0.25, 7e20]]
    F = rng.integers(0, len(V), size=(50000, vpf)).astype(np.int32)
    p = tmp_path / "m.obj"
    io.write_obj(p, V, F, verts_per_face=vpf, threads=threads)
    assert p.read_text() == _obj_text(V, F)


def test_obj_from_mesh_and_empty(tmp_path):
    from contouring_b200 import DualContouringMesh, io
    m = DualContouringMesh(np.array([0, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1, 0], np.float32), np.array([0, 1, 2, 3], np.int32))
    io.write_obj(tmp_path / "q.obj", m)
    assert (tmp_path / "q.obj").read_text() == "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n"
    io.write_obj(tmp_path / "e.obj", DualContouringMesh())
    assert (tmp_path / "e.obj").read_text() == ""


def _cli_harness():
    """oracle/_ref/ref_obj_to_sdf: the reference CLI's own file functions (dc_cli.cpp:17-47),
    compiled from dc_cli.cpp by `make -C oracle ref`; None when not built."""
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "ref_obj_to_sdf")
    return exe if os.path.exists(exe) else None


def test_obj_text_identical_to_the_reference_cli_writer(tmp_path):
    exe = _cli_harness()
    if exe is None:
        pytest.skip("oracle/_ref/ref_obj_to_sdf was not built (make -C oracle ref)")
    rng = np.random.default_rng(5)
    V = (rng.standard_normal((2000, 3)) * np.array([1e-6, 1.0, 3e5])).astype(np.float32)
    V[:20] = np.array([0.0, -0.0, 1e-38, -1e-45, 123456789.0, 1e20, 0.1, 2.5e-5, 7.0, -3.25] * 6, np.float32).reshape(20, 3)
    F = rng.integers(0, 2000, size=(1500, 4)).astype(np.int32)
    mesh_bin = tmp_path / "mesh.bin"
    with open(mesh_bin, "wb") as f:
        f.write(np.array([2000, 1500], np.int64).tobytes() + V.tobytes() + F.tobytes())
    subprocess.run([exe, "write_obj", str(mesh_bin), str(tmp_path / "ref.obj")], check=True)
    for threads in (1, 7):
        dio.write_obj(tmp_path / "ours.obj", V, F, verts_per_face=4, threads=threads)
        assert (tmp_path / "ours.obj").read_bytes() == (tmp_path / "ref.obj").read_bytes()


def test_sdf_reader_identical_to_the_reference_cli_reader(tmp_path):
    exe = _cli_harness()
    if exe is None:
        pytest.skip("oracle/_ref/ref_obj_to_sdf was not built (make -C oracle ref)")
    rng = np.random.default_rng(6)
    vals = rng.standard_normal(7 * 5 * 3).astype(np.float32)
    g = DenseSdfGrid(7, 5, 3, 0.5, 0.25, 0.125, -1.0, 2.0, 3.5, values=vals)
    path = tmp_path / "g.sdf"
    dio.write_sdf(path, g)
    subprocess.run([exe, "read_sdf", str(path), str(tmp_path / "rec.bin")], check=True)
    raw = (tmp_path / "rec.bin").read_bytes()
    ours = dio.read_sdf(path)
    assert tuple(np.frombuffer(raw[:12], np.int32)) == (ours.nx, ours.ny, ours.nz)
    assert np.array_equal(np.frombuffer(raw[12:36], np.float32),
                          np.array([ours.vx, ours.vy, ours.vz, ours.ox, ours.oy, ours.oz], np.float32))
    assert np.array_equal(np.frombuffer(raw[36:], np.float32), np.asarray(ours.values))


@pytest.mark.parametrize("shape", ["sphere", "box", "plane"])
@pytest.mark.parametrize("res", [9, 24, 33])
def test_cli_test_grids_identical_to_the_reference_generators(tmp_path, shape, res):
    """synth.cli_sphere / cli_box / cli_plane against the CLI's own generate_* (dc_cli.cpp:49-118)."""
    from contouring_b200 import synth
    exe = _cli_harness()
    if exe is None:
        pytest.skip("oracle/_ref/ref_obj_to_sdf was not built (make -C oracle ref)")
    out = tmp_path / ("%s.sdf" % shape)
    subprocess.run([exe, "generate", shape, str(res), str(out)], check=True)
    ref = dio.read_sdf(out)
    vals, dims, sp, org = getattr(synth, "cli_" + shape)(res)
    assert dims == (ref.nx, ref.ny, ref.nz)
    assert np.array_equal(np.array(sp, np.float32), np.array([ref.vx, ref.vy, ref.vz], np.float32))
    assert np.array_equal(np.array(org, np.float32), np.array([ref.ox, ref.oy, ref.oz], np.float32))
    assert np.array_equal(np.asarray(vals.numpy()).view(np.uint32), np.asarray(ref.values).view(np.uint32))
