"""Parity at the benchmark size (1024^3 sharp-feature CSG), where the full oracle is too
slow: the engine's whole-grid result is compared, window by window, with the oracle run on
cubic windows of the same grid (with the whole grid's own float point positions). Cells and
faces at least MARGIN cells inside a window depend only on data inside it, so for those the
engine must match the oracle exactly (active set, vertex numbering, quads and winding) and
within 1e-4 cell widths (vertices)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RES = 1024
WIN = 72
MARGIN = 3
N_WINDOWS = 10


@pytest.fixture(scope="module")
def extraction():
    import torch
    from contouring_b200 import B200DualContouringBackend, synth
    vals, dims, sp, org = synth.csg(RES, seed=0, device="cuda")
    be = B200DualContouringBackend(0)
    V, F, stats = be.extract_tensor(vals, dims, sp, org)
    cells = be.active_cells()
    V2, F2, _ = be.extract_tensor(vals, dims, sp, org)
    det = bool(torch.equal(V, V2) and torch.equal(F, F2))
    out = dict(V=V.cpu().numpy(), F=F.cpu().numpy(), cells=cells, stats=stats, det=det,
               vals=vals.cpu().numpy().reshape(dims[2], dims[1], dims[0]), dims=dims, sp=sp, org=org)
    be.close()
    del vals, V, F, V2, F2
    torch.cuda.empty_cache()
    return out


def _axes(dims, sp, org):
    return [(np.float32(org[a]) + np.arange(dims[a], dtype=np.float32) * np.float32(sp[a])).astype(np.float64)
            for a in range(3)]


def test_deterministic_1024(extraction):
    assert extraction["det"]


def test_counts_consistent_1024(extraction):
    e = extraction
    F = e["F"]
    assert e["stats"].vertex_count == len(e["V"]) == len(e["cells"])
    assert F.min() >= 0 and F.max() < len(e["V"])
    assert np.all(np.diff(e["cells"]) > 0)          # strictly increasing linear order
    # every face's four cells are distinct
    assert np.all((F[:, 0] != F[:, 1]) & (F[:, 1] != F[:, 2]) & (F[:, 2] != F[:, 3]))


def test_windows_match_oracle_1024(extraction):
    import oracle as O
    e = extraction
    nx, ny, nz = e["dims"]
    cx, cy = nx - 1, ny - 1
    ax = _axes(e["dims"], e["sp"], e["org"])
    cells = e["cells"]
    V, F = e["V"].astype(np.float64), e["F"]
    # index of engine faces by (c2, c0): unique per face
    fkey = F[:, 2].astype(np.int64) * (1 << 31) + F[:, 0]
    order = np.argsort(fkey)
    fkey_sorted = fkey[order]
    rng = np.random.default_rng(7)
    centers = cells[rng.choice(len(cells), N_WINDOWS, replace=False)]
    worst = 0.0
    nfaces = 0
    for c in centers:
        ci, cj, ck = c % cx, (c // cx) % cy, c // (cx * cy)
        i0 = int(np.clip(ci - WIN // 2, 0, nx - WIN))
        j0 = int(np.clip(cj - WIN // 2, 0, ny - WIN))
        k0 = int(np.clip(ck - WIN // 2, 0, nz - WIN))
        sub = np.ascontiguousarray(e["vals"][k0:k0 + WIN, j0:j0 + WIN, i0:i0 + WIN])
        r = O.dc_extract_positions(sub, (WIN, WIN, WIN), ax[0][i0:i0 + WIN], ax[1][j0:j0 + WIN],
                                   ax[2][k0:k0 + WIN], threads=0)
        wc = WIN - 1
        la, lb, lc = r["cells"] % wc, (r["cells"] // wc) % wc, r["cells"] // (wc * wc)
        glob = (i0 + la) + cx * ((j0 + lb) + cy * (k0 + lc))
        interior = ((la >= MARGIN) & (la < wc - MARGIN) & (lb >= MARGIN) & (lb < wc - MARGIN) &
                    (lc >= MARGIN) & (lc < wc - MARGIN))
        # active set on the interior block
        gi, gj, gk = cells % cx, (cells // cx) % cy, cells // (cx * cy)
        in_block = ((gi >= i0 + MARGIN) & (gi < i0 + wc - MARGIN) & (gj >= j0 + MARGIN) & (gj < j0 + wc - MARGIN) &
                    (gk >= k0 + MARGIN) & (gk < k0 + wc - MARGIN))
        assert np.array_equal(np.sort(glob[interior]), cells[in_block]), "active set differs in window %s" % ((i0, j0, k0),)
        gidx = np.searchsorted(cells, glob)
        err = np.abs(V[gidx[interior]] - r["V"][interior]) / np.array(e["sp"])
        if err.size:
            worst = max(worst, float(err.max()))
        # faces whose four cells are interior
        ok = interior[r["F"]].all(axis=1)
        Fw = gidx[r["F"][ok]]
        nfaces += len(Fw)
        key = Fw[:, 2].astype(np.int64) * (1 << 31) + Fw[:, 0]
        pos = np.searchsorted(fkey_sorted, key)
        assert np.all(pos < len(fkey_sorted)) and np.all(fkey_sorted[np.minimum(pos, len(fkey_sorted) - 1)] == key), \
            "a window face is missing from the engine output"
        assert np.array_equal(F[order[pos]], Fw), "a window face differs (winding) in window %s" % ((i0, j0, k0),)
    print("windows=%d faces=%d max_vertex_err=%.3g cells, escalated=%d winding_fp64=%d" % (
        N_WINDOWS, nfaces, worst, e["stats"].escalated_fp64_cells, e["stats"].winding_fp64_faces))
    assert worst <= 1e-4
