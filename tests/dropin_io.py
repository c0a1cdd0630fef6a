"""Reader of the output file of oracle/ref_b200_drive (the reference-side C++ driver of
include/dc_b200.h): two meshes (extract, then extract_device) with their DualContouringStats."""
import numpy as np

STAT_COUNTS = ("total_cells", "active_cells", "vertex_count", "face_count", "qef_fallback_count", "clamp_count",
               "bad_qef_count")
STAT_TIMES = ("upload_ms", "marking_ms", "compaction_ms", "active_cell_marking_ms", "active_cell_compaction_ms",
              "qef_ms", "face_emission_ms", "face_count_ms", "face_prefix_sum_ms", "face_fill_ms", "download_ms",
              "total_ms")


def read_drive_output(path):
    buf = open(path, "rb").read()
    pos = 0
    out = []
    for _ in range(2):
        nv, nf, vpf = np.frombuffer(buf, np.int64, 3, pos)
        pos += 24
        V = np.frombuffer(buf, np.float32, 3 * nv, pos).reshape(-1, 3)
        pos += 12 * int(nv)
        F = np.frombuffer(buf, np.int32, int(vpf * nf), pos).reshape(-1, int(vpf)) if vpf else np.zeros((0, 4), np.int32)
        pos += 4 * int(vpf * nf)
        counts = np.frombuffer(buf, np.int32, len(STAT_COUNTS), pos)
        pos += 4 * len(STAT_COUNTS)
        times = np.frombuffer(buf, np.float32, len(STAT_TIMES), pos)
        pos += 4 * len(STAT_TIMES)
        stats = dict(zip(STAT_COUNTS, counts.tolist()))
        stats.update(zip(STAT_TIMES, times.tolist()))
        out.append((V, F, stats))
    assert pos == len(buf)
    return out
