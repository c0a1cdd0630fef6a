"""The adjoint of the vertices (dcb_backward) on the differentiable workload: a 128^3 float32
grid of a sphere (r = 0.3) perturbed by 64 Gaussian RBFs; loss = mean squared distance from
the extracted vertices to the nearest of 50,000 points on a second seeded perturbed sphere.

d(loss)/d(grid) from the GPU adjoint is checked against
  * the FP64 reference adjoint (dual-number Jacobians of every vertex, summed J^T g), and
  * FP64 central finite differences of the FP64 vertices on a double copy of the grid, at
    1000 random corners of active cells (|value| > 2e-4, so no sign changes; the
    nearest-point assignment held fixed): h = 1e-4 Richardson-extrapolated and h = 1e-6,
    relative error <= 1e-3;
and the forward + backward time against the forward alone (<= 2.5x)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

H = 1e-4
FD_REL_TOL = 1e-3
REF_REL_TOL = 1e-5


@pytest.fixture(scope="module")
def setup():
    import torch
    import oracle as O
    from scipy.spatial import cKDTree
    from contouring_b200 import B200DualContouringBackend, synth
    from dc_compare import grid_axes
    vals, dims, sp, org = synth.rbf_sphere(128)
    vals_np = vals.numpy()
    be = B200DualContouringBackend(0)
    d = vals.cuda()
    V, F, st = be.extract_tensor(d, dims, sp, org)
    cells = be.active_cells()
    ax = grid_axes(dims, sp, org)
    V64, kept = O.cell_vertices(vals_np, dims, ax, cells, return_kept=True)
    T = synth.rbf_sphere_points(50000, seed=1)
    _, nn = cKDTree(T).query(V64)
    tgt = T[nn]
    # dL/dV of L = mean |v - t|^2, at the FP64 vertices (rounded to the float the ABI takes)
    gV = (2.0 * (V64 - tgt) / len(V64)).astype(np.float32)
    dgrid = be.backward_tensor(d, dims, sp, org, torch.from_numpy(gV).cuda()).cpu().numpy().astype(np.float64)
    yield dict(be=be, vals=vals_np, d=d, dims=dims, sp=sp, org=org, ax=ax, cells=cells, V=V, F=F,
               V64=V64, kept=kept, tgt=tgt, gV=gV, dgrid=dgrid)
    be.close()


def test_matches_reference_adjoint(setup):
    import oracle as O
    S = setup
    ref = O.vertex_vjp(S["vals"], S["dims"], S["ax"], S["cells"], S["gV"].astype(np.float64))
    got = S["dgrid"]
    rel = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    worst = np.abs(got - ref).max() / np.abs(ref).max()
    print("vertices %d, nonzero grid gradients %d, rel err %.3g, max err / max %.3g" % (
        len(S["cells"]), int((ref != 0).sum()), rel, worst))
    assert rel <= REF_REL_TOL and worst <= REF_REL_TOL


def _fd_corners(S, n=1000, seed=0):
    vals, cells = S["vals"], S["cells"]
    nx, ny, nz = S["dims"]
    cx, cy = nx - 1, ny - 1
    rng = np.random.default_rng(seed)
    out, seen = [], set()
    while len(out) < n:
        c = cells[rng.integers(len(cells))]
        i, j, k = c % cx, (c // cx) % cy, c // (cx * cy)
        q = int(rng.integers(8))
        p = int((i + (q & 1)) + nx * ((j + ((q >> 1) & 1)) + ny * (k + (q >> 2))))
        if p in seen or abs(float(vals[p])) <= 2 * H:
            continue
        seen.add(p)
        out.append(p)
    return np.array(out, np.int64)


def test_matches_central_differences(setup):
    """FP64 central differences of the FP64 vertices at 1000 corners, at h = 1e-4 (plain, and
    Richardson-extrapolated with h/2, error O(h^4)) and at h = 1e-6. A corner where some
    nearby cell's solve keeps a different number of eigenvalues at +-h (an eigenvalue within
    h's reach of the truncation threshold) sits on a discontinuity of the vertex map; the
    adjoint holds that rank fixed, so h = 1e-4 differences are compared on the other corners
    (at most 2% are left out), h = 1e-6 ones on all."""
    import oracle as O
    S = setup
    nx, ny, nz = S["dims"]
    cx, cy = nx - 1, ny - 1
    cells, tgt, kept0 = S["cells"], S["tgt"], S["kept"]
    nv = len(cells)
    vd = S["vals"].astype(np.float64)
    corners = _fd_corners(S)
    fd = np.empty((len(corners), 3))
    flip = np.zeros(len(corners), bool)
    for r, p in enumerate(corners):
        pi, pj, pk = p % nx, (p // nx) % ny, p // (nx * ny)
        ii, jj, kk = np.meshgrid(np.arange(pi - 2, pi + 2), np.arange(pj - 2, pj + 2), np.arange(pk - 2, pk + 2),
                                 indexing="ij")
        ok = (ii >= 0) & (ii < cx) & (jj >= 0) & (jj < cy) & (kk >= 0) & (kk < nz - 1)
        lin = (ii + cx * (jj + cy * kk))[ok]
        pos = np.searchsorted(cells, lin)
        hit = (pos < nv) & (cells[np.minimum(pos, nv - 1)] == lin)
        aff, rank = lin[hit], pos[hit]
        t = tgt[rank]
        base = vd[p]
        for q, h in enumerate((H, H / 2, 1e-6)):
            vd[p] = base + h
            vp, kp = O.cell_vertices(vd, S["dims"], S["ax"], aff, return_kept=True)
            vd[p] = base - h
            vm, km = O.cell_vertices(vd, S["dims"], S["ax"], aff, return_kept=True)
            vd[p] = base
            if q == 0:
                flip[r] = np.any(kp != kept0[rank]) or np.any(km != kept0[rank])
            fd[r, q] = (((vp - t) ** 2).sum() - ((vm - t) ** 2).sum()) / (2 * h * nv)
    got = S["dgrid"][corners]

    def errs(g, f):
        per = np.abs(g - f) / np.maximum(np.abs(f), 1e-3 * np.abs(f).max())
        return np.linalg.norm(g - f) / np.linalg.norm(f), np.percentile(per, 99), per.max()

    sm = ~flip
    plain = errs(got[sm], fd[sm, 0])
    rich = errs(got[sm], (4 * fd[sm, 1] - fd[sm, 0]) / 3)
    fine = errs(got, fd[:, 2])
    print("corners %d, rank changes within h=1e-4: %d" % (len(corners), flip.sum()))
    for name, e in (("h=1e-4", plain), ("h=1e-4 Richardson", rich), ("h=1e-6", fine)):
        print("  %-18s aggregate rel err %.3g, per-corner p99 %.3g, max %.3g" % ((name,) + e))
    assert flip.sum() <= 0.02 * len(corners)
    assert rich[0] <= FD_REL_TOL and rich[1] <= FD_REL_TOL
    assert fine[0] <= FD_REL_TOL and fine[2] <= FD_REL_TOL


def test_autograd_function(setup):
    import torch
    from contouring_b200 import dual_contour
    S = setup
    be = S["be"]
    values = S["d"].clone().requires_grad_(True)
    V, F = dual_contour(values, S["dims"], S["sp"], S["org"], backend=be)
    assert not F.requires_grad and V.requires_grad
    assert torch.equal(V.detach(), S["V"]) and torch.equal(F, S["F"])
    tgt = torch.from_numpy(S["tgt"]).float().cuda()
    loss = ((V - tgt) ** 2).sum(1).mean()
    # an unrelated extraction on the same backend between forward and backward
    from contouring_b200 import synth
    small, sdims, ssp, sorg = synth.sphere(40)
    be.extract_tensor(small.cuda(), sdims, ssp, sorg)
    loss.backward()
    gV = (2.0 * (V.detach() - tgt) / V.shape[0]).contiguous()
    be.extract_tensor(S["d"], S["dims"], S["sp"], S["org"])
    want = be.backward_tensor(S["d"], S["dims"], S["sp"], S["org"], gV)
    diff = (values.grad.reshape(-1) - want).abs().max().item()
    assert diff <= 1e-6 * want.abs().max().item()


def test_accumulate_and_zero_gradient(setup):
    import torch
    S = setup
    be = S["be"]
    be.extract_tensor(S["d"], S["dims"], S["sp"], S["org"])
    gV = torch.from_numpy(S["gV"]).cuda()
    a = be.backward_tensor(S["d"], S["dims"], S["sp"], S["org"], gV)
    b = be.backward_tensor(S["d"], S["dims"], S["sp"], S["org"], gV, out=a.clone(), accumulate=True)
    assert torch.allclose(b, 2 * a, rtol=1e-5, atol=1e-12)
    z = be.backward_tensor(S["d"], S["dims"], S["sp"], S["org"], torch.zeros_like(gV))
    assert int(torch.count_nonzero(z)) == 0
    # gradients only inside the 4x4x4 stencils of active cells: nothing far from the surface
    far = np.abs(S["vals"]) > 4 * S["sp"][0] * np.sqrt(3)
    assert np.all(a.cpu().numpy()[far] == 0.0)


def test_rejects_mismatched_calls(setup):
    import torch
    from contouring_b200 import DcbError, synth
    S = setup
    be = S["be"]
    be.extract_tensor(S["d"], S["dims"], S["sp"], S["org"])
    with pytest.raises(DcbError):                         # wrong vertex-gradient size
        be.backward_tensor(S["d"], S["dims"], S["sp"], S["org"], torch.zeros(5, 3, device="cuda"))
    small, sdims, ssp, sorg = synth.sphere(40)
    with pytest.raises(DcbError):                         # not the grid of the last extraction
        be.backward_tensor(small.cuda(), sdims, ssp, sorg, torch.from_numpy(S["gV"]).cuda())
    be.extract_batch([(small.cuda(), sdims, ssp, sorg)] * 2)
    with pytest.raises(DcbError):                         # after a batch
        be.backward_tensor(S["d"], S["dims"], S["sp"], S["org"], torch.from_numpy(S["gV"]).cuda())


def test_forward_backward_time(setup):
    """Forward + backward (extraction, then the adjoint into a dense gradient grid) against
    the forward alone, both timed with CUDA events over 20 calls after warm-up."""
    import torch
    from contouring_b200.backend import DenseSdfGridDevice
    S = setup
    be = S["be"]
    g = DenseSdfGridDevice(*S["dims"], *S["sp"], *S["org"], d_values=S["d"])
    gV = torch.from_numpy(S["gV"]).cuda()
    out = torch.empty(S["d"].numel(), dtype=torch.float32, device="cuda")

    def fwd():
        be.extract_tensor_ptr(g)

    def fwd_bwd():
        be.extract_tensor_ptr(g)
        be.backward_tensor(S["d"], S["dims"], S["sp"], S["org"], gV, out=out)

    def timed(fn, n=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / n

    tf = timed(fwd)
    tfb = timed(fwd_bwd)
    print("forward %.3f ms, forward+backward %.3f ms, ratio %.2f" % (tf, tfb, tfb / tf))
    assert tfb <= 2.5 * tf
