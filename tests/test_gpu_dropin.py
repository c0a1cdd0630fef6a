"""include/dc_b200.h's B200DualContouringBackend, compiled against the reference's own headers
into oracle/_ref/ref_b200_drive and called the way dc_cli calls a backend (through
IDualContouringBackend::extract, and extract_device on a caller-owned device grid): both meshes
equal the oracle's (identical quads and vertex numbering, vertices within 1e-4 cell widths) and
DualContouringStats carries the counts."""
import os
import subprocess

import numpy as np
import pytest

from dc_compare import VERTEX_TOL, run_oracle
from dropin_io import read_drive_output

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVE = os.path.join(ROOT, "oracle", "_ref", "ref_b200_drive")


def _cases():
    from contouring_b200 import synth
    return {"sphere32": lambda: synth.cli_sphere(32), "csg96": lambda: synth.csg(96, seed=1),
            "noise_zeros": lambda: synth.noise((17, 23, 9), seed=2, zero_frac=0.3),
            "empty16": lambda: synth.constant(16, 1.0)}


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_dropin_class_matches_oracle(tmp_path, name):
    if not os.path.exists(DRIVE):
        pytest.skip("oracle/_ref/ref_b200_drive was not built")
    from contouring_b200 import DenseSdfGrid, io
    case = _cases()[name]()
    io.write_sdf(str(tmp_path / "g.sdf"), DenseSdfGrid.from_tuple(case))
    r = subprocess.run([DRIVE, str(tmp_path / "g.sdf"), str(tmp_path / "o.bin")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    (V, F, st), (V2, F2, st2) = read_drive_output(str(tmp_path / "o.bin"))
    ref = run_oracle(case)
    h = np.asarray(case[2], np.float64)
    for VV, FF, ss in ((V, F, st), (V2, F2, st2)):
        assert ss["vertex_count"] == ss["active_cells"] == len(ref["V"])
        assert ss["face_count"] == len(ref["F"])
        assert ss["total_cells"] == int(np.prod(np.asarray(case[1]) - 1))
        assert ss["bad_qef_count"] == 0 and ss["clamp_count"] == 0
        assert np.array_equal(FF, ref["F"])
        if len(VV):
            assert (np.abs(VV.astype(np.float64) - ref["V"]) / h).max() <= VERTEX_TOL
    assert np.array_equal(V, V2) and np.array_equal(F, F2)
    assert st["face_emission_ms"] >= 0 and st["face_fill_ms"] >= 0 and st["active_cell_marking_ms"] == st["marking_ms"]
