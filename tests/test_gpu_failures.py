"""Host-side failure injection and non-finite inputs (nothing here faults, traps or hangs a GPU).

1. Forced allocation failure: dcb_debug_fail_allocations makes the k-th device or page-locked
   allocation of the library fail as cudaMalloc does when the device is full. For every k up to
   the first call that needs no more allocations, each entry point must return
   DCB_ERR_OUT_OF_MEMORY (never crash or report success with a wrong result), and the same handle
   must then produce the result of an untouched handle.
2. NaN grid values: the reference CPU backend treats NaN as neither sign, keeps the edge as a
   Hermite crossing (fa*fb > 0 is false, Cell.cpp:185) and propagates the NaN into the vertex;
   the engine must give the same cells, quads and NaN vertices (compared with the oracle and,
   where it was built, the reference's own compiled backend).
3. Infinite values: where an infinite value sits at the end a quad edge's representative cell
   interpolates from, the reference's Hermite lookup fails and it exits (contouring.cpp:590-594);
   the engine returns DCB_ERR_INVALID_ARGUMENT there instead, and elsewhere matches the oracle.
"""
import numpy as np
import pytest

from dc_compare import VERTEX_TOL

pytestmark = pytest.mark.gpu


def _be():
    from contouring_b200 import B200DualContouringBackend
    return B200DualContouringBackend(0)


def _hook(n):
    from contouring_b200 import _lib
    assert _lib.lib().dcb_debug_fail_allocations(int(n)) == 0


def _calls():
    """Entry point name -> (backend factory, fn(backend) returning a comparable result)."""
    import torch
    from contouring_b200 import (B200DualContouringBackend, B200SparseDualContouringBackend, DenseSdfGrid,
                                 mesh_to_sdf_tensor, postprocess_mesh_tensor, synth)
    grid = synth.csg(48, seed=1)
    dvals = grid[0].cuda()
    dims, sp, org = grid[1], grid[2], grid[3]
    g2 = synth.csg(32, seed=2)
    g2d = (g2[0].cuda(), g2[1], g2[2], g2[3])
    V, F = synth.icosphere_scene(4, 2, seed=1)
    mdims, msp, morg = synth.mesh_grid(V, 32)
    Vd, Fd = torch.from_numpy(V).cuda(), torch.from_numpy(F).cuda()
    dense_be = lambda: B200DualContouringBackend(0)
    sparse_be = lambda: B200SparseDualContouringBackend(device=0)

    def dense(be):
        V_, F_, _ = be.extract_tensor(dvals, dims, sp, org)
        return V_.cpu().numpy(), F_.cpu().numpy()

    def host(be):
        m, _ = be.extract(DenseSdfGrid.from_tuple(grid))
        return m.vertices.copy(), m.faces.copy()

    def batch(be):
        meshes, _ = be.extract_batch([(dvals, dims, sp, org), g2d])
        return [t.cpu().numpy() for m in meshes for t in m]

    def mesh_sdf(be):
        out, _ = mesh_to_sdf_tensor(be, Vd, Fd, mdims, morg, msp)
        return out.cpu().numpy()

    def post(be):
        V_, F_, _ = be.extract_tensor(dvals, dims, sp, org)
        Vo, Fo, _ = postprocess_mesh_tensor(be, V_, F_, True, True)
        return Vo.cpu().numpy(), Fo.cpu().numpy()

    def backward(be):
        V_, _, _ = be.extract_tensor(dvals, dims, sp, org)
        g = be.backward_tensor(dvals, dims, sp, org, torch.ones_like(V_))
        return g.cpu().numpy()

    return {"extract_device": (dense_be, dense), "extract_host": (dense_be, host), "extract_batch": (dense_be, batch),
            "sparse": (sparse_be, dense), "mesh_to_sdf": (dense_be, mesh_sdf), "postprocess": (dense_be, post),
            "backward": (dense_be, backward)}


def _same(a, b, rtol=0.0):
    if isinstance(a, (tuple, list)):
        return len(a) == len(b) and all(_same(x, y, rtol) for x, y in zip(a, b))
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    if rtol:
        return bool(np.allclose(a, b, rtol=rtol, atol=rtol * float(np.abs(b).max(initial=0.0)), equal_nan=True))
    return np.array_equal(a, b, equal_nan=a.dtype.kind == "f")


# d(loss)/d(grid) is accumulated with float atomics: equal up to the order of the additions
RTOL = {"backward": 1e-5}


@pytest.mark.parametrize("name", ["extract_device", "extract_host", "extract_batch", "sparse", "mesh_to_sdf",
                                  "postprocess", "backward"])
def test_allocation_failure_is_reported_and_recoverable(name):
    from contouring_b200 import _lib
    make, fn = _calls()[name]
    ref_be = make()
    try:
        expect = fn(ref_be)
    finally:
        ref_be.close()
    failures = 0
    for k in range(200):
        be = make()
        try:
            _hook(k)
            try:
                got = fn(be)
                ok = True
            except _lib.DcbError as e:
                assert e.status == _lib.DCB_ERR_OUT_OF_MEMORY, "%s, allocation %d: %s" % (name, k, e)
                ok = False
            finally:
                _hook(-1)
            if ok:
                assert _same(got, expect, RTOL.get(name, 0.0)), "%s succeeded after %d allocations with a different result" % (name, k)
                break
            failures += 1
            # the handle is still usable and gives the untouched handle's result
            assert _same(fn(be), expect, RTOL.get(name, 0.0)), "%s: handle unusable after a failure at allocation %d" % (name, k)
        finally:
            _hook(-1)
            be.close()
    else:
        pytest.fail("%s needed more than 200 allocations" % name)
    assert failures >= 1, "%s allocated nothing on a fresh handle" % name
    print("%s: %d allocation points, each reported DCB_ERR_OUT_OF_MEMORY and recovered" % (name, failures))


def _poisoned(kind, seed=5):
    from contouring_b200 import synth
    vals, dims, sp, org = synth.csg(40, seed=0)
    v = vals.numpy().copy()
    rng = np.random.default_rng(seed)
    if kind == "nan":
        v[rng.choice(v.size, 60, replace=False)] = np.nan
    elif kind == "inf_far":
        # infinities of the same sign only at points more than 8 cells from the surface: no
        # Hermite sample, averaging stencil or winding gradient reaches them
        far = rng.choice(np.nonzero(np.abs(v) > 8 * sp[0])[0], 40, replace=False)
        v[far] = np.where(v[far] > 0, np.inf, -np.inf)
    return v, dims, sp, org


def test_nan_values_match_oracle_and_reference():
    import oracle as O
    from contouring_b200 import DenseSdfGrid
    v, dims, sp, org = _poisoned("nan")
    be = _be()
    try:
        mesh, st = be.extract(DenseSdfGrid(*dims, *sp, *org, values=v))
        cells = be.active_cells()
    finally:
        be.close()
    ref = O.dc_extract(v, dims, sp, org)
    V = mesh.vertices.reshape(-1, 3).astype(np.float64)
    F = mesh.faces.reshape(-1, 4)
    assert np.array_equal(cells, ref["cells"])
    nan_rows = np.isnan(V).any(1)
    ref_nan = np.isnan(ref["V"]).any(1)
    assert nan_rows.any() and np.array_equal(nan_rows, ref_nan), "NaN vertices: engine %s, oracle %s" % (
        np.nonzero(nan_rows & ~ref_nan)[0][:8].tolist(), np.nonzero(ref_nan & ~nan_rows)[0][:8].tolist())
    err = np.abs(V[~nan_rows] - ref["V"][~nan_rows]) / np.asarray(sp)
    assert err.max() <= VERTEX_TOL
    bad = np.nonzero((F != ref["F"]).any(1))[0] if F.shape == ref["F"].shape else np.arange(1)
    assert len(bad) == 0, "%d quads differ (escalated %d), first: engine %s oracle %s, engine vertices %s, oracle %s" % (
        len(bad), st.escalated_fp64_cells, F[bad[:3]].tolist(), ref["F"][bad[:3]].tolist(),
        V[F[bad[0]]].tolist(), ref["V"][ref["F"][bad[0]]].tolist())
    r = O.ref_cpu_extract(v, dims, sp, org)
    if r is not None:
        rV, rF, _ = r
        assert np.array_equal(F, rF) and np.array_equal(np.isnan(rV).any(1), nan_rows)


def test_infinite_value_on_a_quad_edge_is_an_error():
    from contouring_b200 import DcbError, DenseSdfGrid, _lib, synth
    vals, dims, sp, org = synth.cli_sphere(24)
    v = vals.numpy().copy()
    # a point right at the surface, on a sign-changing x edge: its value goes to +inf (same sign)
    nx, ny = dims[0], dims[1]
    k = j = 12
    row = v[(k * ny + j) * nx:(k * ny + j + 1) * nx]
    i = int(np.nonzero((row[:-1] < 0) & (row[1:] > 0))[0][0]) + 1     # first positive point of the crossing
    v[(k * ny + j) * nx + i] = np.inf
    be = _be()
    try:
        with pytest.raises(DcbError) as e:
            be.extract(DenseSdfGrid(*dims, *sp, *org, values=v))
        assert e.value.status == _lib.DCB_ERR_INVALID_ARGUMENT
        # the handle stays usable
        mesh, _ = be.extract(DenseSdfGrid.from_tuple(synth.cli_sphere(24)))
        assert len(mesh.faces) > 0
    finally:
        be.close()
    import os
    import oracle as O
    if os.path.exists(os.path.join(os.path.dirname(O.__file__), "_ref", "ref_cpu_dc")):
        with pytest.raises(RuntimeError):      # the reference's own backend exits on this grid
            O.ref_cpu_extract(v, dims, sp, org)


def test_infinite_values_away_from_the_surface_match_oracle():
    import oracle as O
    from contouring_b200 import DenseSdfGrid
    v, dims, sp, org = _poisoned("inf_far")
    assert np.isinf(v).sum() > 0
    be = _be()
    try:
        mesh, _ = be.extract(DenseSdfGrid(*dims, *sp, *org, values=v))
        cells = be.active_cells()
    finally:
        be.close()
    ref = O.dc_extract(v, dims, sp, org)
    assert np.array_equal(cells, ref["cells"]) and np.array_equal(mesh.faces.reshape(-1, 4), ref["F"])
    V = mesh.vertices.reshape(-1, 3).astype(np.float64)
    assert (np.abs(V - ref["V"]) / np.asarray(sp)).max() <= VERTEX_TOL
    r = O.ref_cpu_extract(v, dims, sp, org)
    if r is not None:
        assert np.array_equal(mesh.faces.reshape(-1, 4), r[1])
