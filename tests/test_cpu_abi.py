"""CPU checks of the C ABI (include/dcb.h) and the host-side mirror of the reference API: the
library loads and exports every declared function, the ctypes structures have the C layout,
and the host logic validates its inputs. No compute call is made without a GPU."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "dcb.h")


def _declared():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(dcb_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_exported_list():
    from contouring_b200 import _lib
    assert _declared() == sorted(_lib.EXPORTED)


def test_library_exports_every_declared_symbol():
    from contouring_b200 import _lib
    L = _lib.lib()
    for name in _declared():
        assert hasattr(L, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert set(_declared()) <= exported


def test_library_resolves_every_engine_symbol():
    """A shared library links with undefined symbols; one of the engine's own (namespace dcb)
    left undefined means a source file missing from the build, found only when it is called."""
    from contouring_b200 import _lib
    out = subprocess.run(["nm", "-D", "--undefined-only", _lib.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    missing = [line.split()[-1] for line in out.splitlines() if "_ZN3dcb" in line or " dcb_" in line]
    assert not missing, missing


def test_abi_utilities():
    from contouring_b200 import _lib
    L = _lib.lib()
    assert L.dcb_abi_version() >= 4
    for code in range(0, -8, -1):
        assert L.dcb_status_string(code)
    assert L.dcb_status_string(-99) == b"unknown status"
    assert L.dcb_last_error(None) == b"null handle"


def test_default_opts_match_python_defaults():
    from contouring_b200 import ContouringOptions, _lib
    o = _lib.default_opts()
    p = ContouringOptions().to_c()
    for name, _ in _lib.DcbOpts._fields_:
        assert getattr(o, name) == getattr(p, name), name
    assert o.svd_threshold == 0.01 and o.outer_iters == 100 and o.inner_iters == 100


def test_struct_layouts_match_the_header():
    """Compile a probe against include/dcb.h with gcc and compare sizes and offsets with the
    ctypes mirrors."""
    from contouring_b200 import _lib
    structs = {"dcb_grid": _lib.DcbGrid, "dcb_opts": _lib.DcbOpts, "dcb_stats": _lib.DcbStats,
               "dcb_mesh_dev": _lib.DcbMeshDev, "dcb_mesh_host": _lib.DcbMeshHost,
               "dcb_sdf_stats": _lib.DcbSdfStats, "dcb_batch_mesh": _lib.DcbBatchMesh,
               "dcb_post_stats": _lib.DcbPostStats}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "dcb.h"', "int main(void) {"]
    for cname, py in structs.items():
        lines.append('printf("%s %%zu\\n", sizeof(%s));' % (cname, cname))
        for f, _ in py._fields_:
            lines.append('printf("%s.%s %%zu\\n", offsetof(%s, %s));' % (cname, f, cname, f))
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(c, "w").write("\n".join(lines))
        subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        got = dict(line.split() for line in subprocess.run([exe], capture_output=True, text=True,
                                                           check=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got["%s.%s" % (cname, f)]) == getattr(py, f).offset, (cname, f)


def test_null_arguments_are_rejected_without_a_device():
    from contouring_b200 import _lib
    L = _lib.lib()
    cnt = ctypes.c_int64(7)
    assert L.dcb_mark_active_cells_noalloc(None, None, 0, ctypes.byref(cnt), None) == _lib.DCB_ERR_INVALID_ARGUMENT
    assert L.dcb_create(None, 0) == _lib.DCB_ERR_INVALID_ARGUMENT
    assert L.dcb_destroy(None) in (_lib.DCB_OK, _lib.DCB_ERR_INVALID_ARGUMENT)
    # the mesh post-pass and the OBJ entry points
    assert L.dcb_postprocess_device(None, None, 0, None, 0, 1, 1, None, None, None) == _lib.DCB_ERR_INVALID_ARGUMENT
    assert L.dcb_postprocess_host(None, None, 0, None, 0, 1, 1, None, None, None) == _lib.DCB_ERR_INVALID_ARGUMENT
    assert L.dcb_copy_post_mesh(None, None, None, 1, None) == _lib.DCB_ERR_INVALID_ARGUMENT
    g = _lib.DcbGrid()
    V = np.zeros((2, 3), np.float32)
    assert L.dcb_obj_grid(None, 0, 8, ctypes.byref(g)) == _lib.DCB_ERR_INVALID_ARGUMENT
    assert L.dcb_obj_grid(V.ctypes.data, 2, 1, ctypes.byref(g)) == _lib.DCB_ERR_INVALID_ARGUMENT
    assert L.dcb_obj_grid(V.ctypes.data, 2, 8, None) == _lib.DCB_ERR_INVALID_ARGUMENT
    nv, nt = ctypes.c_int64(), ctypes.c_int64()
    assert L.dcb_read_obj(None, None, 0, None, 0, ctypes.byref(nv), ctypes.byref(nt)) == _lib.DCB_ERR_INVALID_ARGUMENT
    assert L.dcb_batch_graph_launch(None, None) == _lib.DCB_ERR_INVALID_ARGUMENT


def test_no_device_fails_loudly():
    """Without a CUDA device the backend raises: there is no CPU fallback."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from contouring_b200 import B200DualContouringBackend, DcbError
    with pytest.raises(DcbError):
        B200DualContouringBackend(0)


def test_dense_grid_mirrors_the_reference_type():
    """DenseSdfGrid keeps the reference's fields (dc_backend.h:13-21); DenseSdfGridDevice
    borrows a device pointer (dc_cuda.h:24-29)."""
    from contouring_b200 import DenseSdfGrid, DenseSdfGridDevice
    from contouring_b200 import synth
    t = synth.sphere(8)
    g = DenseSdfGrid.from_tuple(t)
    assert (g.nx, g.ny, g.nz) == (8, 8, 8)
    assert np.asarray(g.values).size == 512
    assert abs(g.vx - 1.0 / 7) < 1e-7 and g.ox == -0.5
    d = DenseSdfGridDevice(4, 4, 4, 1, 1, 1, 0, 0, 0, d_values=12345)
    assert d.pointer() == 12345


def test_contouring_options_mirror_the_reference():
    """ContouringOptions fields and defaults follow contouring.h:27-41."""
    from contouring_b200 import ContouringMethod, ContouringOptions
    o = ContouringOptions()
    assert o.method == ContouringMethod.DualContouring
    assert (o.outer_iters, o.inner_iters) == (100, 100)
    assert o.svd_threshold == 0.01
