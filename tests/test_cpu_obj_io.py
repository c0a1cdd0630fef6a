"""OBJ -> SDF ingestion of the reference CLI (read_obj_to_sdf, src/cpp/dc_cli.cpp:121-203): the
C ABI's OBJ reader against a plain-Python restatement of the reference's parsing rules on a file
full of edge cases, and the padded grid against the reference's float arithmetic restated in
numpy float32. No GPU needed; the conversion itself is the tested mesh -> SDF path."""
import re

import numpy as np
import pytest

from contouring_b200 import DcbError
from contouring_b200 import io as dio

TEXT = (
    "# comment\n"
    "v 0 0 0\n"
    "v 1.5 0 0\r\n"
    "v\t9 9 9\n"                 # second character is a tab: not a vertex line
    " v 8 8 8\n"                 # leading blank: not a vertex line
    "vn 0 0 1\n"
    "vt 0.5 0.5\n"
    "v 0 2.25 0\n"
    "v 1 2\n"                    # two floats: skipped
    "v  1e-3   1.0e1\t-2.5\n"
    "v 0.1 0.2 0.3 1.0\n"        # a fourth (weight) value is ignored
    "f 1 2 3\n"
    "f 1/1/1 2/1/1 4/1/1 5/1/1\n"
    "f -1 -2 -3\r\n"
    "f 1//1 3//1 4//1 5//1 2//1\n"
    "f 0 1 2 3\n"                # index 0 is dropped
    "f 1 2\n"                    # two indices: no triangle
    "f 3 4 5 \r\n"               # trailing blank + CR token reads as 0: dropped
    "o name\ns off\ng group\n"
    "f\t1 2 3\n"                 # not a face line
    "v 5 5 5"                    # last line without newline
)


def py_reference_parse(text):
    """The reference's rules (dc_cli.cpp:126-156), restated."""
    V, T = [], []
    for line in text.split("\n"):
        if len(line) < 2 or line[1] != " ":
            continue
        if line[0] == "v":
            nums = re.match(r"\s*([-+0-9.eE]+)\s*([-+0-9.eE]+)\s*([-+0-9.eE]+)", line[2:])
            if nums:
                V.append([float(x) for x in nums.groups()])
        elif line[0] == "f":
            idx = []
            for tok in re.split(r"[ \t]+", line[2:]):
                m = re.match(r"\s*([-+]?\d+)", tok)
                i = int(m.group(1)) if m else 0
                if i != 0:
                    if i < 0:
                        i = len(V) + i + 1
                    idx.append(i - 1)
            for k in range(1, len(idx) - 1):
                T.append([idx[0], idx[k], idx[k + 1]])
    return np.array(V, np.float32), np.array(T, np.int32)


def test_obj_reader_follows_reference_rules(tmp_path):
    p = tmp_path / "edge.obj"
    p.write_bytes(TEXT.encode())
    V, T = dio.read_obj(p)
    Vr, Tr = py_reference_parse(TEXT)
    assert V.shape == Vr.shape == (6, 3)
    assert np.array_equal(V, Vr)
    assert np.array_equal(T, Tr)
    assert T.shape[0] == 1 + 2 + 1 + 3 + 1 + 1


def test_obj_grid_matches_reference_float_arithmetic():
    rng = np.random.default_rng(3)
    V = (rng.standard_normal((500, 3)) * [1.0, 0.3, 2.0] + [5.0, -1.0, 0.25]).astype(np.float32)
    for res in (2, 17, 256):
        dims, sp, org = dio.obj_grid(V, res)
        f = np.float32
        lo, hi = V.min(0), V.max(0)
        d = hi - lo
        diag = np.sqrt(f(f(f(d[0] * d[0]) + f(d[1] * d[1])) + f(d[2] * d[2])))
        pad = f(diag * f(0.08))
        lo2, hi2 = lo - pad, hi + pad
        want_sp = [f((hi2[a] - lo2[a]) / f(res - 1)) for a in range(3)]
        assert dims == (res, res, res)
        assert np.array_equal(np.array(org, np.float32), lo2)
        assert np.array_equal(np.array(sp, np.float32), np.array(want_sp, np.float32))
    dims, sp, org = dio.obj_grid(np.zeros((1, 3), np.float32), 5)
    assert np.allclose(org, (-0.1, -0.1, -0.1)) and np.allclose(sp, (0.05, 0.05, 0.05))


def test_obj_errors(tmp_path):
    with pytest.raises(DcbError):
        dio.read_obj(tmp_path / "missing.obj")
    p = tmp_path / "nofaces.obj"
    p.write_text("v 0 0 0\nv 1 0 0\n")
    with pytest.raises(DcbError):
        dio.read_obj(p)
    p = tmp_path / "range.obj"
    p.write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n")
    with pytest.raises(DcbError):
        dio.read_obj(p)


def _reference_record(path, res):
    """The reference CLI's own read_obj_to_sdf run on `path` (oracle/_ref/ref_obj_to_sdf, built
    from dc_cli.cpp by `make -C oracle ref`): what it hands to the conversion. None when the
    harness was not built."""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref", "ref_obj_to_sdf")
    if not os.path.exists(exe):
        return None
    rec = str(path) + ".rec"
    subprocess.run([exe, "obj2sdf", str(path), str(res), rec], check=True)
    raw = open(rec, "rb").read()
    nv, nt = np.frombuffer(raw[:16], np.int64)
    at = 16
    V = np.frombuffer(raw[at:at + 12 * nv], np.float32).reshape(-1, 3)
    at += 12 * nv
    T = np.frombuffer(raw[at:at + 12 * nt], np.int32).reshape(-1, 3)
    at += 12 * nt
    dims = tuple(int(x) for x in np.frombuffer(raw[at:at + 12], np.int32))
    geo = np.frombuffer(raw[at + 12:at + 36], np.float32)
    return V, T, dims, geo[:3], geo[3:]


@pytest.mark.parametrize("res", [16, 97])
def test_ingestion_matches_the_reference_cli(tmp_path, res):
    from contouring_b200 import synth
    files = []
    p = tmp_path / "edge.obj"
    p.write_bytes(TEXT.encode())
    files.append(p)
    V, F = synth.icosphere(2)
    q = tmp_path / "ico.obj"
    dio.write_obj(q, (V * np.float32(3.7) + np.float32([1.0, -2.0, 0.5])).astype(np.float32), F, verts_per_face=3)
    files.append(q)
    for path in files:
        ref = _reference_record(path, res)
        if ref is None:
            pytest.skip("oracle/_ref/ref_obj_to_sdf was not built (make -C oracle ref)")
        Vr, Tr, dims_r, org_r, sp_r = ref
        Vo, To = dio.read_obj(path)
        dims, sp, org = dio.obj_grid(Vo, res)
        assert np.array_equal(Vo.view(np.uint32), Vr.view(np.uint32)) and np.array_equal(To, Tr), path
        assert dims == dims_r
        assert np.array_equal(np.array(org, np.float32), org_r) and np.array_equal(np.array(sp, np.float32), sp_r)
