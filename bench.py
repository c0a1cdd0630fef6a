#!/usr/bin/env python3
"""Benchmark: dense dual-contouring extraction of the 1024^3 sharp-feature CSG grid.

One step = one full extraction (mark + compaction, Hermite + averaging + QEF, quad
emission in the CPU backend's order) of a 1024^3 float32 grid that is resident in HBM.
Metric: Mcells/s = (nx-1)(ny-1)(nz-1) / step time, summed over ranks (each rank extracts
its own grid: weak scaling, no collective on the data path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--res 1024] [--impl reference]

Under torchrun each rank runs on its LOCAL_RANK GPU; rank 0 prints one JSON line.
``--impl reference`` times the CPU oracle (the FP64 restatement of the reference's
CpuDualContouringBackend, which is single-threaded C++ in the reference and cannot be
built here: it needs Eigen and libigl) with every host thread on a bounded sample of the
same grid (8 z-slabs spread evenly over it), and reports the same metric.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "phanty-sdf-cuda_b200"))

# Launches of the engine's own kernels per extraction: mark, 3 segment-scan passes, vertex
# offsets, rank expansion, cell-width tables, QEF (with the edge normals), Jacobi list, FP64
# vertices, 3 column-scan passes, face scatter, FP64 vertices for windings, FP64 windings,
# face order.
KERNELS_PER_STEP = 17
# DRAM traffic of k_mark_zmarch per grid point, from a single-kernel ncu capture of the 512^3
# CSG workload (dram__bytes_read.sum + dram__bytes_write.sum divided by the grid points of
# that capture; the kernel streams the grid once, so traffic scales with the number of
# points). None = not measured.
MARK_TRAFFIC_BYTES_PER_POINT = (564.13824e6 + 18.598144e6) / 512 ** 3
# DRAM traffic of a whole extraction (every kernel of one step), as grid-proportional bytes per
# point plus band-proportional bytes per active cell, from single-kernel-list ncu captures
# (dram__bytes_read.sum + dram__bytes_write.sum summed over the step's launches). None = not
# measured.
# From one extraction of the 512^3 CSG workload (1,534,557 active cells): the mark and the scans
# of segments and columns 5.89068e+08 B (grid-proportional), every other kernel 3.56506e+08 B
# (band-proportional).
PIPELINE_TRAFFIC_BYTES_PER_POINT = 5.89068e+08 / 512 ** 3
PIPELINE_TRAFFIC_BYTES_PER_ACTIVE = 3.56506e+08 / 1534557


def max_over_ranks(local, dist, device):
    """The slowest rank's time: every rank takes part in the MAX all-reduce (the job's time is
    the max over ranks); without a process group, the local value."""
    if dist is None or not dist.is_initialized():
        return float(local)
    import torch
    t = torch.tensor([float(local)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world, cells_per_rank, ms_per_step):
    """Whole-job Mcells/s: every rank extracts its own grid of the same size (replicas, weak
    scaling), so the job processes world * cells per step in the slowest rank's time."""
    return world * cells_per_rank / (ms_per_step / 1e3) / 1e6


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and throttle-reason sampling during the timed region: NVML polled every 2 ms
    from a thread (the timed calls release the GIL while they wait on the device), so a region
    of tens of milliseconds still gets samples; nvidia-smi every 100 ms when NVML is missing."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock event reason bits
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None
        self.nvml = None
        self.thread = None
        self.stop = False
        self.sm, self.mx, self.bits = [], None, 0

    def _nvml_handle(self):
        """This process's CUDA device as an NVML handle, found by its UUID (or its PCI
        address); only strings reach NVML's string arguments."""
        import pynvml
        import torch
        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.gpu)
        uuid = str(getattr(props, "uuid", "") or "")
        if uuid:
            return pynvml, pynvml.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
        bus = "%08x:%02x:%02x.0" % (int(props.pci_domain_id), int(props.pci_bus_id), int(props.pci_device_id))
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def _poll(self, pynvml, h):
        get_reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop:
            try:
                self.sm.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                self.bits |= int(get_reasons(h))
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        try:
            pynvml, h = self._nvml_handle()
            self.mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.nvml = pynvml
            self.thread = threading.Thread(target=self._poll, args=(pynvml, h), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.nvml = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.thread:
            self.stop = True
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.nvml is not None:
            reasons = sorted(n for n, bit in self.REASONS.items() if self.bits & bit)
            return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.mx,
                    "reasons": reasons, "samples": len(self.sm), "source": "nvml"}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            os.unlink(self.path)
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def make_grid(res, device):
    from contouring_b200 import synth
    return synth.csg(res, seed=0, device=device)


SAMPLE_SLABS = 8


def slab_ranges(nz, planes_total):
    """Point-plane ranges of SAMPLE_SLABS z-slabs spread evenly over the grid, about
    planes_total planes in all (each slab at least 2 planes)."""
    per = max(2, planes_total // SAMPLE_SLABS)
    out = []
    for s in range(SAMPLE_SLABS):
        c = int((s + 0.5) * nz / SAMPLE_SLABS)
        k0 = max(0, min(nz - per, c - per // 2))
        out.append((k0, k0 + per))
    return out


def grid_axes(dims, spacing, origin):
    """Float grid-point coordinates o + float(i) * v per axis, widened to FP64."""
    import numpy as np
    return [(np.float32(origin[a]) + np.arange(dims[a], dtype=np.float32) * np.float32(spacing[a])).astype(np.float64)
            for a in range(3)]


def cpu_sample(slabs, dims, spacing, origin, threads, keep=False):
    """Time the CPU oracle on z-slabs of the grid: ``slabs`` = [((k0, k1), float32 values of
    planes k0..k1-1)]. Returns (Mcells/s, seconds, cells[, per-slab results when keep])."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    nx, ny, _ = dims
    ax = grid_axes(dims, spacing, origin)
    dt, cells, kept = 0.0, 0, []
    for (k0, k1), v in slabs:
        t0 = time.perf_counter()
        r = O.dc_extract_positions(v, (nx, ny, k1 - k0), ax[0], ax[1], ax[2][k0:k1], threads=threads)
        dt += time.perf_counter() - t0
        cells += (nx - 1) * (ny - 1) * (k1 - k0 - 1)
        if keep:
            kept.append(r)
    if keep:
        return cells / dt / 1e6, dt, cells, kept
    return cells / dt / 1e6, dt, cells


# Cells closer than this to a slab's z faces depend on planes outside the slab.
SLAB_MARGIN = 3


def slab_vertex_error(slabs, kept, dims, spacing, V, cells):
    """Max and RMS difference, in cell widths, between the engine's vertices and the FP64
    oracle's on the slabs of the CPU sample: every active cell at least SLAB_MARGIN planes
    inside its slab (the slabs span the whole grid in x and y, so no other cell depends on
    data outside). Also checks that those cells are the same active cells."""
    import numpy as np
    nx, ny, _ = dims
    cx, cy = nx - 1, ny - 1
    h = np.asarray(spacing, np.float64)
    errs = []
    for ((k0, k1), _), r in zip(slabs, kept):
        lk = r["cells"] // (cx * cy)
        inner = (lk >= SLAB_MARGIN) & (lk < (k1 - k0 - 1) - SLAB_MARGIN)
        glob = r["cells"][inner] + k0 * cx * cy
        gidx = np.searchsorted(cells, glob)
        if len(glob) and not np.array_equal(cells[np.minimum(gidx, len(cells) - 1)], glob):
            raise RuntimeError("engine and oracle active cells differ in slab %s" % ((k0, k1),))
        errs.append((np.abs(V[gidx].astype(np.float64) - r["V"][inner]) / h).ravel())
    e = np.concatenate(errs) if errs else np.zeros(0)
    return {"max_cell_widths": float(e.max()) if e.size else 0.0,
            "rms_cell_widths": float(np.sqrt(np.mean(e * e))) if e.size else 0.0,
            "vertices_compared": int(e.size // 3),
            "against": "FP64 oracle on the CPU-sample slabs (cells >= %d planes inside)" % SLAB_MARGIN}


REF_CPU_DC = os.path.join(ROOT, "oracle", "_ref", "ref_cpu_dc")
REF_CUBE = 40          # points per side of each sub-cube the reference CPU backend runs on


def cube_origins(res, n):
    """n sub-cube corners spread over the grid: the cubes straddle the scene's surface-rich
    middle third in z and are spaced evenly in x and y."""
    import numpy as np
    rng = np.random.default_rng(11)
    lo, hi = res // 6, res - res // 6 - REF_CUBE
    return [tuple(int(x) for x in rng.integers(lo, hi, 3)) for _ in range(n)]


def ref_cpu_cubes(values_of_cube, origins, spacing, origin, workdir):
    """Write the sub-cube grids for the reference's own CPU backend (oracle/_ref/ref_cpu_dc):
    values_of_cube(i0, j0, k0) -> float32 REF_CUBE^3 values (x fastest). Returns the file paths
    and the cell count."""
    import numpy as np
    paths = []
    for q, (i0, j0, k0) in enumerate(origins):
        v = values_of_cube(i0, j0, k0)
        o = [float(np.float32(np.float32(origin[a]) + np.float32((i0, j0, k0)[a]) * np.float32(spacing[a])))
             for a in range(3)]
        path = os.path.join(workdir, "cube%d.sdf" % q)
        with open(path, "wb") as f:
            f.write(np.array([REF_CUBE] * 3, np.int32).tobytes())
            f.write(np.array(list(spacing) + o, np.float32).tobytes())
            f.write(np.ascontiguousarray(v, np.float32).tobytes())
        paths.append(path)
    return paths, len(origins) * (REF_CUBE - 1) ** 3


def ref_cpu_run(paths, workdir):
    """One step of the reference CPU arm: the reference's own (single-threaded) CPU backend on
    every sub-cube at once, one process per cube. Returns wall seconds."""
    import subprocess
    t0 = time.perf_counter()
    procs = [subprocess.Popen([REF_CPU_DC, p, os.path.join(workdir, "out%d.bin" % q)],
                              stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL) for q, p in enumerate(paths)]
    rcs = [p.wait() for p in procs]
    dt = time.perf_counter() - t0
    if any(rcs):
        raise RuntimeError("ref_cpu_dc failed: %s" % rcs)
    return dt


def _ref_sample_text(n, res, cells):
    return ("%d sub-cubes of %d^3 points inside the %d^3 CSG grid (%d cells), the reference's own CPU "
            "backend (compiled from its sources) on each, one process per cube" % (n, REF_CUBE, res, cells))


def _sample_text(dims, ranges, cells, res):
    return "%d z-slabs of %dx%dx%d points spread over the %d^3 CSG grid (%d cells, %.1f%% of the grid)" % (
        len(ranges), dims[0], dims[1], ranges[0][1] - ranges[0][0], res, cells,
        100.0 * cells / ((dims[0] - 1) * (dims[1] - 1) * (dims[2] - 1)))


def run_reference(args, rank, world):
    """CPU reference arm: the reference's own CPU backend (CpuDualContouringBackend::extract,
    compiled from its sources into oracle/_ref/ref_cpu_dc) on a bounded sample of the same grid,
    one process per host core; where that program was not built, the oracle port with all host
    threads on evenly spread z-slabs."""
    import numpy as np
    from contouring_b200 import synth
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    dims = (args.res,) * 3
    if os.path.exists(REF_CPU_DC):
        import tempfile
        ncube = max(1, min(threads, 16))
        origins = cube_origins(args.res, ncube)
        spacing = origin = None

        def cube(i0, j0, k0):
            nonlocal spacing, origin
            v, _, spacing, origin = synth.csg(args.res, seed=0, device="cpu", planes=(k0, k0 + REF_CUBE))
            return v.numpy().reshape(REF_CUBE, args.res, args.res)[:, j0:j0 + REF_CUBE, i0:i0 + REF_CUBE].copy()

        with tempfile.TemporaryDirectory() as td:
            cubes = [cube(*o) for o in origins]
            paths, cells = ref_cpu_cubes(lambda i0, j0, k0: cubes[origins.index((i0, j0, k0))], origins,
                                         spacing, origin, td)
            for _ in range(args.warmup):
                ref_cpu_run(paths, td)
            secs = [ref_cpu_run(paths, td) for _ in range(args.steps)]
        dt = float(np.median(secs))
        value = cells / dt / 1e6
        sample = _ref_sample_text(ncube, args.res, cells)
        line = {
            "metric": "dc_extract_mcells_per_s", "value": round(value, 4), "unit": "Mcells/s",
            "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1000 * dt, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "csg%d_dense_dc" % args.res, "grid": list(dims), "sample": sample},
            "cpu_baseline": {"value": round(value, 4), "unit": "Mcells/s", "cores": ncube,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": round(value, 4), "unit": "Mcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return 0
    ranges = slab_ranges(args.res, args.ref_zslab)
    slabs = []
    for r in ranges:
        v, _, spacing, origin = synth.csg(args.res, seed=0, device="cpu", planes=r)
        slabs.append((r, v.numpy()))
    for _ in range(args.warmup):
        cpu_sample(slabs, dims, spacing, origin, threads)
    rates, secs = [], []
    for _ in range(args.steps):
        rate, dt, cells = cpu_sample(slabs, dims, spacing, origin, threads)
        rates.append(rate)
        secs.append(dt)
    value = float(np.median(rates))
    sample = _sample_text(dims, ranges, cells, args.res)
    line = {
        "metric": "dc_extract_mcells_per_s", "value": round(value, 3), "unit": "Mcells/s",
        "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(1000 * float(np.median(secs)), 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "csg%d_dense_dc" % args.res, "grid": list(dims), "sample": sample},
        "cpu_baseline": {"value": round(value, 3), "unit": "Mcells/s", "cores": threads,
                         "kind": "port", "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "Mcells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batch_workload(args):
    """256 CSG shapes at uneven resolutions {32..192}^3 in one batched extraction per step,
    against the same shapes extracted one after another with plain single-grid calls."""
    import numpy as np
    import torch
    from contouring_b200 import B200DualContouringBackend, synth
    torch.cuda.set_device(0)
    grids = synth.csg_batch(256, seed=0, device="cuda")
    torch.cuda.synchronize()
    be = B200DualContouringBackend(0)
    ncell = sum((d[0] - 1) * (d[1] - 1) * (d[2] - 1) for _, d, _, _ in grids)
    waves, narrow, tune_ms = be.autotune_mark(grids)         # tile shapes for this batch
    qef_minb, qef_bps, face_bps, cells_ms = be.autotune_cells(grids)   # vertex / face kernel shapes
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(args.warmup):
        be.extract_batch_ptr(grids)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        _, st = be.extract_batch_ptr(grids)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_batch = e0.elapsed_time(e1) / args.steps
    from contouring_b200 import DenseSdfGridDevice

    def sequential():
        for v, d, sp, o in grids:
            be.extract_tensor_ptr(DenseSdfGridDevice(*d, *sp, *o, d_values=v))
    ms_seq = None
    if not args.no_sequential:
        for _ in range(max(1, args.warmup // 2)):
            sequential()
        torch.cuda.synchronize()
        e0.record(stream)
        reps = max(1, args.steps // 4)
        for _ in range(reps):
            sequential()
        e1.record(stream)
        torch.cuda.synchronize()
        ms_seq = e0.elapsed_time(e1) / reps
    # the same batch captured in a CUDA graph and replayed (no host synchronisation inside)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        be.batch_graph_create(grids, headroom=0.25)
        for _ in range(args.warmup):
            be.batch_graph_launch()
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        g0.record(side)
        for _ in range(args.steps):
            be.batch_graph_launch()
        g1.record(side)
        _, gst = be.batch_graph_finish()
    torch.cuda.synchronize()
    ms_graph = g0.elapsed_time(g1) / args.steps
    same_graph = gst.vertex_count == st.vertex_count and gst.face_count == st.face_count
    be.batch_graph_destroy()
    line = {
        "metric": "dc_extract_mcells_per_s", "value": round(ncell / (ms_batch / 1e3) / 1e6, 2), "unit": "Mcells/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_batch, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "csg_batch256", "grids": len(grids), "cells": ncell,
                   "resolutions": [32, 48, 64, 96, 128, 192], "vertices": st.vertex_count, "quads": st.face_count},
        "stage_ms": {"mark": round(st.marking_ms, 4), "scan": round(st.compaction_ms, 4),
                     "qef": round(st.qef_ms, 4), "faces": round(st.face_emission_ms, 4)},
        "escalated_fp64_cells": st.escalated_fp64_cells, "winding_fp64_faces": st.winding_fp64_faces,
        "mark_tiles": {"waves": waves, "narrow_tile_max_cells": narrow, "autotune_mark_ms": round(tune_ms, 4)},
        "cell_kernels": {"qef_min_blocks_per_sm": qef_minb, "qef_blocks_per_sm": qef_bps,
                         "face_blocks_per_sm": face_bps, "autotune_stage_ms": round(cells_ms, 4)},
        "sequential_plain_ms": round(ms_seq, 3) if ms_seq else None,
        "batched_speedup": round(ms_seq / ms_batch, 2) if ms_seq else None,
        "graph": {"ms_per_step": round(ms_graph, 4), "mcells_per_s": round(ncell / (ms_graph / 1e3) / 1e6, 2),
                  "same_counts_as_eager": bool(same_graph),
                  "speedup_vs_sequential": round(ms_seq / ms_graph, 2) if ms_seq else None},
    }
    print(json.dumps(line), flush=True)
    be.close()
    return 0


def _timed(fn, steps, warmup):
    """CUDA-event milliseconds per call of fn on the current stream, after warm-up."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _side_line(metric, value, unit, ms, args, config, **extra):
    line = {"metric": metric, "value": round(value, 3), "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if "ours" in metric or "fwd_bwd" in metric else "f32",
            "data": "synthetic", "config": config}
    line.update(extra)
    print(json.dumps(line), flush=True)


def run_adjoint_workload(args):
    """The differentiable workload: a 128^3 sphere (r = 0.3) perturbed by 64 Gaussian RBFs; a
    step is the extraction, the gradient of the mean squared distance from the vertices to their
    nearest of 50,000 points on a second perturbed sphere (nearest points found once, then held
    fixed), and the adjoint into a dense d(loss)/d(grid)."""
    import torch
    from contouring_b200 import B200DualContouringBackend, DenseSdfGridDevice, synth
    torch.cuda.set_device(0)
    vals, dims, sp, org = synth.rbf_sphere(128, device="cuda")
    T = torch.from_numpy(synth.rbf_sphere_points(50000, seed=1)).cuda().float()
    be = B200DualContouringBackend(0)
    g = DenseSdfGridDevice(*dims, *sp, *org, d_values=vals)
    V, F, st = be.extract_tensor(vals, dims, sp, org)
    nn = torch.cat([torch.cdist(V[a:a + 8192], T).argmin(1) for a in range(0, len(V), 8192)])
    tgt = T[nn]
    out = torch.empty(vals.numel(), dtype=torch.float32, device="cuda")
    ncell = (dims[0] - 1) * (dims[1] - 1) * (dims[2] - 1)

    def fwd():
        be.extract_tensor_ptr(g)

    def fwd_bwd():
        Vt, _, _ = be.extract_tensor(vals, dims, sp, org)
        dV = (2.0 / len(Vt)) * (Vt - tgt)
        be.backward_tensor(vals, dims, sp, org, dV, out=out)

    ms_f = _timed(fwd, args.steps, args.warmup)
    ms_fb = _timed(fwd_bwd, args.steps, args.warmup)
    _side_line("dc_fwd_bwd_mcells_per_s", ncell / (ms_fb / 1e3) / 1e6, "Mcells/s", ms_fb, args,
               {"workload": "rbf_sphere128_adjoint", "grid": list(dims), "vertices": st.vertex_count,
                "targets": 50000},
               forward_ms=round(ms_f, 4), fwd_bwd_over_fwd=round(ms_fb / ms_f, 3), gpu_launches=KERNELS_PER_STEP + 5)
    be.close()
    return 0


def run_ours_workload(args):
    """The refinement (ContouringMethod::Ours, 100 outer x 100 inner iterations) of the 128^3
    sphere (r = 0.35); a step is the extraction and its full refinement."""
    import torch
    from contouring_b200 import (B200DualContouringBackend, ContouringMethod, ContouringOptions,
                                 DenseSdfGridDevice, synth)
    torch.cuda.set_device(0)
    vals, dims, sp, org = synth.sphere(128, radius=0.35, device="cuda")
    be = B200DualContouringBackend(0)
    o = ContouringOptions()
    o.method = ContouringMethod.Ours
    be.options = o
    g = DenseSdfGridDevice(*dims, *sp, *org, d_values=vals)
    st = be.extract_tensor_ptr(g)[2]
    ms = _timed(lambda: be.extract_tensor_ptr(g), args.steps, args.warmup)
    ncell = (dims[0] - 1) * (dims[1] - 1) * (dims[2] - 1)
    _side_line("dc_ours_mcells_per_s", ncell / (ms / 1e3) / 1e6, "Mcells/s", ms, args,
               {"workload": "sphere128_ours", "grid": list(dims), "outer_iters": o.outer_iters,
                "inner_iters": o.inner_iters, "vertices": st.vertex_count})
    be.close()
    return 0


def run_mesh_workload(args):
    """mesh_to_sdf: 32 icospheres (163,840 triangles) into a 512^3 grid on the mesh's padded box;
    a step is one conversion of device-resident vertices and faces."""
    import torch
    from contouring_b200 import B200DualContouringBackend, mesh_to_sdf_tensor, synth
    torch.cuda.set_device(0)
    V, F = synth.icosphere_scene()
    dims, sp, org = synth.mesh_grid(V, 512)
    Vd, Fd = torch.from_numpy(V).cuda(), torch.from_numpy(F).cuda()
    be = B200DualContouringBackend(0)
    out = torch.empty(dims[0] * dims[1] * dims[2], dtype=torch.float32, device="cuda")
    ms = _timed(lambda: mesh_to_sdf_tensor(be, Vd, Fd, dims, org, sp, out=out), args.steps, args.warmup)
    _, st = mesh_to_sdf_tensor(be, Vd, Fd, dims, org, sp, out=out)      # stage times of a warm call
    npts = dims[0] * dims[1] * dims[2]
    extra = {}
    ref_path = os.path.join(ROOT, "oracle", "_ref", "libref_dc_cuda.so")
    if os.path.exists(ref_path):
        # same-GPU speed bar: the reference's own CUDA conversion (its own timer: mesh upload,
        # grid allocation, conversion); it caps the exterior flood at 40 passes, so a few far
        # values can differ: compared by sign only
        import ctypes
        import numpy as np
        ref = ctypes.CDLL(ref_path)
        ref.refsdf_compute.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int] + \
            [ctypes.c_int] * 3 + [ctypes.c_float] * 6 + [ctypes.POINTER(ctypes.c_float), ctypes.c_void_p]
        ref.refsdf_compute.restype = ctypes.c_int
        Vc = np.ascontiguousarray(V, np.float32)
        Fc = np.ascontiguousarray(F, np.int32)
        rms = ctypes.c_float()
        ts = []
        for q in range(args.warmup + args.steps):
            if ref.refsdf_compute(Vc.ctypes.data, len(Vc), Fc.ctypes.data, len(Fc), *dims, *org, *sp,
                                  ctypes.byref(rms), None) != 0:
                raise RuntimeError("reference conversion refused the grid")
            if q >= args.warmup:
                ts.append(rms.value)
        host = np.empty(npts, np.float32)
        ref.refsdf_compute(Vc.ctypes.data, len(Vc), Fc.ctypes.data, len(Fc), *dims, *org, *sp, ctypes.byref(rms),
                           host.ctypes.data)
        ours = out.cpu().numpy()
        ms_ref = statistics.median(ts)
        extra["reference_cuda"] = {"ms_per_step": round(ms_ref, 3), "sign_agreement": float(np.mean(np.sign(ours) == np.sign(host))),
                                   "speedup": round(ms_ref / ms, 2)}
    _side_line("mesh_to_sdf_mpoints_per_s", npts / (ms / 1e3) / 1e6, "Mpoints/s", ms, args,
               {"workload": "icospheres32_mesh_to_sdf512", "grid": list(dims), "triangles": len(F)},
               stage_ms={"bins": round(st.bins_ms, 4), "band": round(st.band_ms, 4), "sign": round(st.sign_ms, 4),
                         "relax": round(st.relax_ms, 4)}, **extra)
    # voxelize-first (dc_cli --voxelize-first, voxel_res = grid resolution by default)
    vres = dims[0]
    msv = _timed(lambda: mesh_to_sdf_tensor(be, Vd, Fd, dims, org, sp, out=out, voxelize_first=True, voxel_res=vres),
                 args.steps, args.warmup)
    _, stv = mesh_to_sdf_tensor(be, Vd, Fd, dims, org, sp, out=out, voxelize_first=True, voxel_res=vres)
    extra = {}
    if os.path.exists(ref_path):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import numpy as np
        import oracle as O        # only its ref_mesh_to_sdf: the reference's own CUDA code, the comparator
        ts = []
        r = None
        for q in range(min(args.warmup, 2) + min(args.steps, 3)):
            r = O.ref_mesh_to_sdf(V, F, dims, org, sp, voxelize_first=True, voxel_res=vres, exact=False)
            if r is None:
                break
            if q >= min(args.warmup, 2):
                ts.append(r[1])
        if r is not None:
            ours = out.cpu().numpy()
            ms_ref = statistics.median(ts)
            extra["reference_cuda"] = {"ms_per_step": round(ms_ref, 3),
                                       "sign_agreement": float(np.mean(np.sign(ours) == np.sign(r[0]))),
                                       "speedup": round(ms_ref / msv, 2)}
    _side_line("mesh_to_sdf_voxelized_mpoints_per_s", npts / (msv / 1e3) / 1e6, "Mpoints/s", msv, args,
               {"workload": "icospheres32_mesh_to_sdf512_voxelize_first", "grid": list(dims), "triangles": len(F),
                "voxel_res": vres},
               stage_ms={"bins": round(stv.bins_ms, 4), "band": round(stv.band_ms, 4),
                         "voxel_solid_and_sign": round(stv.sign_ms, 4)}, voxel_flood_passes=stv.flood_passes, **extra)
    be.close()
    return 0


def run_refcuda_workload(args):
    """Same-GPU speed bar: the reference's own CUDA dense backend
    (CudaDualContouringBackend::extract_device, built from its source into oracle/_ref/)
    against this engine on the same device-resident 512^3 CSG grid, both from the device grid
    to a host mesh, wall clock with the device synchronised (the reference times itself with a
    host clock the same way). 512^3 because the reference indexes grid edges with 32-bit ints
    and cannot run at 1024^3. Its vertices differ (no normal averaging, clamping): speed only."""
    import ctypes
    import torch
    from contouring_b200 import B200DualContouringBackend, DenseSdfGridDevice
    path = os.path.join(ROOT, "oracle", "_ref", "libref_dc_cuda.so")
    if not os.path.exists(path):
        print(json.dumps({"impl": "reference_cuda", "unavailable": "oracle/_ref/libref_dc_cuda.so was not built"}))
        return 0
    torch.cuda.set_device(0)
    res = 512
    vals, dims, sp, org = make_grid(res, torch.device("cuda", 0))
    torch.cuda.synchronize()
    ref = ctypes.CDLL(path)
    ref.refdc_extract_device.argtypes = [ctypes.c_int] * 3 + [ctypes.c_float] * 6 + [ctypes.c_void_p] + \
        [ctypes.POINTER(ctypes.c_double)] * 2 + [ctypes.POINTER(ctypes.c_int64)] * 2
    ref.refdc_extract_device.restype = ctypes.c_int
    rms, rstage, rnv, rnf = ctypes.c_double(), ctypes.c_double(), ctypes.c_int64(), ctypes.c_int64()
    ref_stage = []

    def ref_call():
        rc = ref.refdc_extract_device(*dims, *sp, *org, vals.data_ptr(), ctypes.byref(rms), ctypes.byref(rstage),
                                      ctypes.byref(rnv), ctypes.byref(rnf))
        if rc != 0:
            raise RuntimeError("reference CUDA backend refused the grid (%d)" % rc)
        torch.cuda.synchronize()
        ref_stage.append(rstage.value)

    be = B200DualContouringBackend(0)
    g = DenseSdfGridDevice(*dims, *sp, *org, d_values=vals)

    def ours_call():
        mesh, _ = be.extract_device(g)
        return mesh

    def wall(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append((time.perf_counter() - t0) * 1e3)
        return statistics.median(ts)

    ms_ref = wall(ref_call, args.steps, args.warmup)
    ref_kernels = statistics.median(ref_stage[args.warmup:])
    ms_ours = wall(ours_call, args.steps, args.warmup)
    ms_ours_dev = _timed(lambda: be.extract_tensor_ptr(g), args.steps, args.warmup)
    mesh = ours_call()
    ncell = (dims[0] - 1) * (dims[1] - 1) * (dims[2] - 1)
    _side_line("dc_extract_to_host_mcells_per_s", ncell / (ms_ours / 1e3) / 1e6, "Mcells/s", ms_ours, args,
               {"workload": "csg512_device_grid_to_host_mesh", "grid": list(dims)},
               reference_cuda={"ms_per_step": round(ms_ref, 3), "mcells_per_s": round(ncell / (ms_ref / 1e3) / 1e6, 1),
                               "stage_kernels_ms": round(ref_kernels, 3), "vertices": rnv.value, "quads": rnf.value},
               device_only_ms=round(ms_ours_dev, 4),
               vertices=len(mesh.vertices) // 3, quads=len(mesh.faces) // 4,
               speedup_vs_reference_cuda=round(ms_ref / ms_ours, 2),
               device_speedup_vs_reference_cuda_stages=round(ref_kernels / ms_ours_dev, 2))
    be.close()
    return 0


class _StdoutToStderr:
    """Sends file descriptor 1 to stderr for the duration (the reference's sparse backend
    prints a memory estimate on every call; the bench's stdout carries JSON lines only)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        os.dup2(2, 1)

    def __exit__(self, *a):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def run_sparse_workload(args):
    """The sparse backends (the reference's CudaSparseDualContouringBackend and its
    multi-vertex variant, dc_cli's default GPU backends) on the device-resident CSG grid
    (1024^3 unless --res): this engine's device time (CUDA events) and device grid -> host
    mesh wall clock, against the reference's own sparse CUDA code as shipped (built from its
    source into oracle/_ref/) on the same GPU, same grid, same brick size (8): wall clock from
    the device grid to the host mesh, and its own stage timers. One line per variant."""
    import numpy as np
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O          # only its ref_sparse: the reference's own CUDA code, the comparator
    from contouring_b200 import B200SparseDualContouringBackend, DenseSdfGridDevice
    torch.cuda.set_device(0)
    res = args.res
    vals, dims, sp, org = make_grid(res, torch.device("cuda", 0))
    torch.cuda.synchronize()
    ncell = (dims[0] - 1) * (dims[1] - 1) * (dims[2] - 1)
    g = DenseSdfGridDevice(*dims, *sp, *org, d_values=vals)

    def wall(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            ts.append((time.perf_counter() - t0) * 1e3)
        return statistics.median(ts)

    for mvdc in (False, True):
        be = B200SparseDualContouringBackend(multi_vertex_cells=mvdc)
        ms_dev = _timed(lambda: be.extract_tensor_ptr(g), args.steps, args.warmup)
        ms_host = wall(lambda: be.extract_device(g), args.steps, args.warmup)
        mesh, st = be.extract_device(g)
        ref = {}
        ref_res = []

        def ref_call():
            with _StdoutToStderr():
                r = O.ref_sparse(vals.data_ptr(), dims, sp, org, mvdc=mvdc, exact=False)
            if r is None:
                raise RuntimeError("reference sparse backend unavailable")
            ref_res.append(r)
        try:
            ms_ref = wall(ref_call, max(1, min(args.steps, 5)), min(args.warmup, 2))
            r = ref_res[-1]
            ours_f = mesh.faces.reshape(-1, 4)
            same_shape = len(r["V"]) * 3 == len(mesh.vertices) and r["F"].shape == ours_f.shape
            differing = int(np.any(r["F"] != ours_f, axis=1).sum()) if same_shape else None
            ref = {"ms_per_step": round(ms_ref, 3), "mcells_per_s": round(ncell / (ms_ref / 1e3) / 1e6, 1),
                   "own_total_ms": round(r["times"][0], 3),
                   "own_stage_kernels_ms": round(sum(r["times"][1:]), 3),
                   "vertices": int(len(r["V"])), "quads": int(len(r["F"])),
                   "quads_differing_from_ours": differing}
            extra = {"speedup_vs_reference_cuda": round(ms_ref / ms_host, 2),
                     "device_speedup_vs_reference_cuda_stages": round(sum(r["times"][1:]) / ms_dev, 2)}
        except (RuntimeError, OSError) as e:
            ref = {"unavailable": str(e)}
            extra = {}
        name = "sparse_mvdc" if mvdc else "sparse"
        _side_line("dc_%s_mcells_per_s" % name, ncell / (ms_dev / 1e3) / 1e6, "Mcells/s", ms_dev, args,
                   {"workload": "csg%d_%s_brick8" % (res, name), "grid": list(dims)},
                   device_grid_to_host_mesh_ms=round(ms_host, 3), vertices=st.vertex_count, quads=st.face_count,
                   active_cells=st.active_cells, active_bricks=st.active_bricks, two_vertex_cells=st.two_vertex_cells,
                   stage_ms={"mark": round(st.marking_ms, 4), "scan": round(st.compaction_ms, 4),
                             "vertices": round(st.qef_ms, 4), "faces": round(st.face_emission_ms, 4)},
                   reference_cuda=ref, **extra)
        be.close()
    return 0


def run_post_workload(args):
    """The mesh post-pass (postprocess_mesh, src/cpp/dc_backend.cpp:217-558, dc_cli's
    --close-holes / --remove-floaters) on meshes this engine extracts at --res (1024^3 unless
    given): the CSG scene (floaters, grid-cut holes) and a sphere larger than the grid (six
    large holes, each filled ring by ring). Device time per call (CUDA events; the call reads
    counts back to size its outputs), host mesh -> host mesh wall clock, and the reference's own
    postprocess_mesh (built from its source into oracle/_ref/; the oracle's restatement when
    absent) on the same host mesh, once, with the GPU output compared to it bit for bit."""
    import numpy as np
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O          # the reference's own CPU post-pass: the comparator
    from contouring_b200 import B200DualContouringBackend, DualContouringMesh, postprocess_mesh, postprocess_mesh_tensor
    from contouring_b200 import synth
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    res = args.res
    scenes = [("csg%d" % res, lambda: make_grid(res, dev))]

    def cut_sphere():
        dims, sp, org = synth._grid_params(res, -0.5, 0.5)
        vals = synth._eval_slabs(dims, sp, org, lambda q: (q - torch.tensor([0.05, 0.0, 0.0], device=q.device)).norm(dim=-1) - 0.6, dev)
        return vals, dims, sp, org
    scenes.append(("cut_sphere%d" % res, cut_sphere))
    be = B200DualContouringBackend(device=0)
    for name, make in scenes:
        vals, dims, sp, org = make()
        V, F, _ = be.extract_tensor(vals, dims, sp, org)
        del vals
        torch.cuda.synchronize()
        ms_dev = _timed(lambda: postprocess_mesh_tensor(be, V, F, True, True), args.steps, args.warmup)
        Vo, Fo, st = postprocess_mesh_tensor(be, V, F, True, True)
        Vh = V.cpu().numpy()
        Fh = F.cpu().numpy()
        mesh = DualContouringMesh(Vh.reshape(-1), Fh.reshape(-1))
        walls = []
        out = None
        for i in range(max(1, min(args.e2e_steps, 3)) + 1):
            out = None      # the previous result's page-locked arrays go back to the host cache
            t0 = time.perf_counter()
            out = postprocess_mesh(mesh, True, True, backend=be)
            if i:
                walls.append((time.perf_counter() - t0) * 1e3)
        ms_e2e = statistics.median(walls)
        t0 = time.perf_counter()
        r = O.ref_postprocess_mesh(Vh, Fh, True, True)
        kind = "reference"
        if r is None:
            r = O.postprocess_mesh(Vh, Fh, True, True)[:2]
            kind = "port"
        ms_ref = (time.perf_counter() - t0) * 1e3
        identical = (r[0].shape == tuple(Vo.shape) and r[1].shape == tuple(Fo.shape)
                     and bool(np.array_equal(r[0].view(np.uint32), Vo.cpu().numpy().view(np.uint32)))
                     and bool(np.array_equal(r[1], Fo.cpu().numpy())))
        nf = int(F.shape[0])
        h2d = int(Vh.nbytes + Fh.nbytes)
        d2h = int(np.asarray(out.vertices).nbytes + np.asarray(out.faces).nbytes)
        _side_line("post_mquads_per_s", nf / (ms_dev / 1e3) / 1e6, "Mquads/s", ms_dev, args,
                   {"workload": "postprocess_%s_close_holes_remove_floaters" % name, "grid": list(dims),
                    "input_vertices": int(V.shape[0]), "input_quads": nf},
                   stats=st.as_dict(),
                   e2e={"value": round(nf / (ms_e2e / 1e3) / 1e6, 3), "unit": "Mquads/s", "ms_per_step": round(ms_e2e, 3),
                        "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
                   cpu_baseline={"value": round(nf / (ms_ref / 1e3) / 1e6, 3), "unit": "Mquads/s", "cores": 1,
                                 "kind": kind, "sample": "the whole mesh, once", "ms": round(ms_ref, 1)},
                   identical_to_reference=identical,
                   speedup_e2e_vs_reference=round(ms_ref / ms_e2e, 2))
        del V, F, Vo, Fo
    be.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--res", type=int, default=1024)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--ref-zslab", type=int, default=96, help="point planes per CPU sample (over 8 slabs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sequential", action="store_true", help="batch256: skip the one-by-one comparison")
    ap.add_argument("--workload", default="csg1024", choices=["csg1024", "batch256", "adjoint128", "ours128", "mesh512", "refcuda512", "sparse1024",
                             "post1024"],
                    help="side workloads (not the headline): batch256 = 256 uneven CSG grids batched vs one "
                         "by one; adjoint128 = forward + adjoint; ours128 = the full refinement; mesh512 = "
                         "mesh_to_sdf; refcuda512 = the reference's CUDA backend vs this engine at 512^3; "
                         "sparse1024 = the sparse and multi-vertex backends vs the reference's at --res; "
                         "post1024 = the mesh post-pass on meshes extracted at --res vs the reference's")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.workload == "batch256":
        return run_batch_workload(args)
    if args.workload == "adjoint128":
        return run_adjoint_workload(args)
    if args.workload == "ours128":
        return run_ours_workload(args)
    if args.workload == "mesh512":
        return run_mesh_workload(args)
    if args.workload == "refcuda512":
        return run_refcuda_workload(args)
    if args.workload == "sparse1024":
        return run_sparse_workload(args)
    if args.workload == "post1024":
        return run_post_workload(args)

    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from contouring_b200 import B200DualContouringBackend, DenseSdfGrid, DenseSdfGridDevice

    dev = torch.device("cuda", local)
    vals, dims, spacing, origin = make_grid(args.res, dev)
    torch.cuda.synchronize()
    be = B200DualContouringBackend(local)
    stream = torch.cuda.current_stream()
    gdev = DenseSdfGridDevice(*dims, *spacing, *origin, d_values=vals)
    ncell = (dims[0] - 1) * (dims[1] - 1) * (dims[2] - 1)
    # vertex / face kernel shapes for this grid, kept by the handle (untimed, before warm-up)
    qef_minb, qef_bps, face_bps, _ = be.autotune_cells([(vals, dims, spacing, origin)])

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        _, _, st = be.extract_tensor_ptr(gdev)
    torch.cuda.synchronize()
    barrier()
    mark_ms, stats = [], None
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier()
        e0.record(stream)
        for _ in range(args.steps):
            _, _, stats = be.extract_tensor_ptr(gdev)
            mark_ms.append(stats.marking_ms)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms_total = max_over_ranks(e0.elapsed_time(e1), dist, dev)
    ms_step = ms_total / args.steps
    value = job_value(world, ncell, ms_step)

    # End to end through the public API: pinned host grid in, host mesh out, every step.
    host = torch.empty(vals.numel(), dtype=torch.float32, pin_memory=True)
    host.copy_(vals.cpu())
    hgrid = DenseSdfGrid(*dims, *spacing, *origin, values=host.numpy())
    for _ in range(args.warmup):             # steady state of the pinned output buffers too
        mesh, _ = be.extract(hgrid)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        mesh, est = be.extract(hgrid)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / max(1, args.e2e_steps), dist, dev)
    e2e_value = job_value(world, ncell, e2e_s * 1e3) if args.e2e_steps > 0 else None
    h2d = 4 * vals.numel()
    d2h = int(mesh.vertices.nbytes + mesh.faces.nbytes)

    peak, peak_kind = _peaks()
    npts = dims[0] * dims[1] * dims[2]
    mark_avg_ms = float(np.mean(mark_ms))
    mark_bytes = 4.0 * npts                       # algorithmic: every grid value read once
    achieved = mark_bytes / (mark_avg_ms / 1e3) / 1e9
    nv, nf = stats.vertex_count, stats.face_count
    # whole extraction: grid read once, vertices and quads written once
    pipe_bytes = 4.0 * npts + 12.0 * nv + 16.0 * nf
    pipe_gbs = pipe_bytes / (ms_step / 1e3) / 1e9
    traffic = (MARK_TRAFFIC_BYTES_PER_POINT * npts) if MARK_TRAFFIC_BYTES_PER_POINT else None
    pipe_traffic = None
    if PIPELINE_TRAFFIC_BYTES_PER_POINT and PIPELINE_TRAFFIC_BYTES_PER_ACTIVE:
        pipe_traffic = PIPELINE_TRAFFIC_BYTES_PER_POINT * npts + PIPELINE_TRAFFIC_BYTES_PER_ACTIVE * nv
    # stage times of the last timed extraction (CUDA events inside the library)
    band_bytes = 12.0 * nv                         # vertices written (stencils come from L2 / HBM re-reads)
    face_bytes = 16.0 * nf
    kernels = [
        {"stage": "mark (k_mark_zmarch)", "ms": round(stats.marking_ms, 4), "algorithmic_bytes": mark_bytes,
         "achieved_gbs": round(mark_bytes / (stats.marking_ms / 1e3) / 1e9, 1) if stats.marking_ms else None,
         "frac": round(mark_bytes / (stats.marking_ms / 1e3) / 1e9 / peak, 4) if stats.marking_ms else None},
        {"stage": "segment scan", "ms": round(stats.compaction_ms, 4)},
        {"stage": "vertices (k_expand_ranks, k_cell_qef, k_cell_jacobi, k_vertex_fp64)", "ms": round(stats.qef_ms, 4),
         "algorithmic_bytes": band_bytes},
        {"stage": "faces (column scan, k_face_scatter, FP64 windings, k_face_order)",
         "ms": round(stats.face_emission_ms, 4), "algorithmic_bytes": face_bytes,
         "sub_ms": {"count": round(stats.face_count_ms, 4), "prefix_sum": round(stats.face_prefix_sum_ms, 4),
                    "fill": round(stats.face_fill_ms, 4)}},
    ]

    cpu = None
    vertex_error = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        ranges = slab_ranges(dims[2], args.ref_zslab)
        plane = dims[0] * dims[1]
        slabs = [(r, vals[r[0] * plane:r[1] * plane].cpu().numpy()) for r in ranges]
        rate, dt, cells, kept = cpu_sample(slabs, dims, spacing, origin, threads, keep=True)
        # one host thread, as the reference CPU backend runs, on the first slab
        rate1, dt1, cells1 = cpu_sample(slabs[:1], dims, spacing, origin, 1)
        cpu = {"value": round(rate, 3), "unit": "Mcells/s", "cores": threads, "kind": "port",
               "sample": _sample_text(dims, ranges, cells, args.res) + ", %.1f s" % dt,
               "single_thread": {"value": round(rate1, 3), "unit": "Mcells/s", "cores": 1,
                                 "sample": "the first of those slabs (%d cells), %.1f s" % (cells1, dt1)}}
        if os.path.exists(REF_CPU_DC):
            # the reference's own CPU backend (compiled from its sources), one process per cube
            import tempfile
            ncube = max(1, min(threads, 16))
            origins = cube_origins(args.res, ncube)
            vz = vals.view(dims[2], dims[1], dims[0])

            def cube(i0, j0, k0):
                return vz[k0:k0 + REF_CUBE, j0:j0 + REF_CUBE, i0:i0 + REF_CUBE].cpu().numpy()

            with tempfile.TemporaryDirectory() as td:
                paths, rcells = ref_cpu_cubes(cube, origins, spacing, origin, td)
                ref_cpu_run(paths, td)
                rdt = ref_cpu_run(paths, td)
            port = dict(cpu)
            cpu = {"value": round(rcells / rdt / 1e6, 4), "unit": "Mcells/s", "cores": ncube, "kind": "reference",
                   "sample": _ref_sample_text(ncube, args.res, rcells) + ", %.1f s" % rdt, "port": port}
        # vertex error of this run against the FP64 oracle on the same slabs
        Vt, _, _ = be.extract_tensor(vals, dims, spacing, origin)
        vertex_error = slab_vertex_error(slabs, kept, dims, spacing, Vt.cpu().numpy().reshape(-1, 3),
                                         be.active_cells())
        del Vt

    if rank == 0:
        line = {
            "metric": "dc_extract_mcells_per_s", "value": round(value, 2), "unit": "Mcells/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "csg%d_dense_dc" % args.res, "grid": list(dims),
                       "cells": ncell, "vertices": nv, "quads": nf,
                       "l2": "input (%.2f GB) larger than L2; no flush needed" % (4 * npts / 1e9),
                       "parallelism": "replicas: one independent grid per rank",
                       "cell_kernels": {"qef_min_blocks_per_sm": qef_minb, "qef_blocks_per_sm": qef_bps,
                                        "face_blocks_per_sm": face_bps}},
            # the whole extraction (every kernel of a step) against the measured copy bandwidth
            "roofline": {"bound": "hbm", "kernel": "whole extraction (%d launches)" % KERNELS_PER_STEP,
                         "achieved": round(pipe_gbs, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(pipe_gbs / peak, 4), "traffic": pipe_traffic, "peak_source": peak_kind,
                         "algorithmic_bytes": pipe_bytes, "avg_launch_ms": round(ms_step, 4)},
            # the grid scan alone (the one kernel that streams the 4 GB grid)
            "mark_roofline": {"bound": "hbm", "kernel": "k_mark_zmarch", "achieved": round(achieved, 1),
                              "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                              "traffic": traffic, "peak_source": peak_kind,
                              "algorithmic_bytes": mark_bytes, "avg_launch_ms": round(mark_avg_ms, 4)},
            "kernels": kernels,
            "stage_ms": {"mark": round(stats.marking_ms, 4), "scan": round(stats.compaction_ms, 4),
                         "qef": round(stats.qef_ms, 4),
                         "faces": round(stats.face_emission_ms, 4)},
            "vertex_error": vertex_error,
            "escalated_fp64_cells": stats.escalated_fp64_cells, "winding_fp64_faces": stats.winding_fp64_faces,
            "e2e": {"value": round(e2e_value, 2) if e2e_value else None, "unit": "Mcells/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": round(e2e_s * 1e3, 2),
                    "last_step_upload_ms": round(est.upload_ms, 2) if args.e2e_steps > 0 else None,
                    "last_step_download_ms": round(est.download_ms, 2) if args.e2e_steps > 0 else None},
            "gpu_launches": KERNELS_PER_STEP * args.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    be.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
