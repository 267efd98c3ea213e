"""Command-line drop-in for the FVM part of `fases3D` (3D-solver/core/main3D.cu:26-1449):

    python -m fases_b200.fz3d <scene.obj> <config.txt> <src.txt> <rec.txt> [--fp64] [--estimate]
                              [--keep-other-sources] [--no-autotune]

Reads the same project files through libfz.so (fz_load_project), runs the Nt time steps of the
configuration on the GPU, prints the integer progress lines the GUI parses ("NN%" every 5 %,
functions3D.cuh:1431-1439, parsed by the regex (\\d+)\\s*% in common/gui.py:6713), and writes
output/IR<r>_<s>.bin, output/VEL<r>_<s>.bin and output/header.txt in the reference formats
(config/p_ref.bin and output/pre_header.txt are written by the loader), plus the animation slices
pressure{X,Y,Z}.bin and I*_*.bin. The geometry is built from the OBJ on the GPU and cached in
output/S.bin, output/oid.bin, output/scene_cache.txt exactly as the reference caches it.

--estimate (main3D.cu:505-525) runs no time step: it prints the effective air volume (air cells x h^3)
and the "[MEM] key=value" pre-flight line the GUI parses (common/gui.py:11017-11033) for this
library's memory needs.
"""
import os
import sys
import time

from .solver import Solver


def _project_output_dir(config_path):
    cfg = os.path.abspath(config_path)
    cdir = os.path.dirname(cfg)
    if os.path.basename(cfg) == "config.txt" and os.path.basename(cdir) == "config":
        return os.path.join(os.path.dirname(cdir), "output")
    return os.path.join(os.getcwd(), "output")


def _src_index(config_path):
    vals = []
    for line in open(config_path):
        line = line.split("#", 1)[0].strip()
        if not line:
            continue
        try:
            vals.append(float(line.split()[0]))
        except ValueError:
            continue
    return int(vals[17]) if len(vals) > 17 else 0


_SLICE_FILES = ("pressureX.bin", "pressureY.bin", "pressureZ.bin", "Iy_X.bin", "Iz_X.bin", "Ix_Y.bin", "Iz_Y.bin",
                "Ix_Z.bin", "Iy_Z.bin", "header.txt", "pre_header.txt")


def purge_outputs(out_dir, src_idx, keep_other_sources=False):
    """Removes the stale outputs of earlier runs before a run, as fases3D does (main3D.cu:170-216):
    the animation slices, header.txt and pre_header.txt, and every IR/VEL/HIR/HRT/ARR*.bin (their
    names vary with receivers, sources and bands, and a changed dt leaves bins of another length);
    with keep_other_sources (--keep-other-sources, the auralization runs 2..N) only the bins of
    this source are removed. S.bin / oid.bin stay: they are the scene cache."""
    if not os.path.isdir(out_dir):
        return []
    removed = []
    for fn in _SLICE_FILES:
        p = os.path.join(out_dir, fn)
        if os.path.exists(p):
            os.remove(p)
            removed.append(fn)

    def file_src(name):  # PREFIX<rec>_<src>[_band].bin -> <src>
        u = name.find("_")
        if u < 0:
            return -1
        rest = name[u + 1:]
        e = min([i for i in (rest.find("_"), rest.find(".")) if i >= 0] or [len(rest)])
        try:
            return int(rest[:e])
        except ValueError:
            return -1

    for fn in sorted(os.listdir(out_dir)):
        if not fn.endswith(".bin") or len(fn) <= 4:
            continue
        if not any(fn.startswith(pfx) for pfx in ("HIR", "HRT", "IR", "ARR", "VEL")):
            continue
        if keep_other_sources and file_src(fn) != src_idx:
            continue
        os.remove(os.path.join(out_dir, fn))
        removed.append(fn)
    return removed


def _config_values(config_path):
    vals = []
    for line in open(config_path):
        line = line.split("#", 1)[0].strip()
        if not line:
            continue
        try:
            vals.append(float(line.split()[0]))
        except ValueError:
            continue
    return vals


def estimate(scene, config, precision="fp32", device=0):
    """The --estimate pre-flight line: voxel count of the padded grid and this library's memory
    model -- host ~11 B per voxel (S, oid, class bytes and copies), device 49 B (FP32 fields) or
    97 B (FP64) -- against free memory (thresholds 0.7 host, 0.9 device as in the reference)."""
    import ctypes as C

    from ._abi import check, lib
    h = _config_values(config)[0]
    dims = (C.c_int32 * 3)()
    check(lib().fz_scene_dims(os.fsencode(scene), float(h), dims, None))
    nvox = dims[0] * dims[1] * dims[2]
    avail = 0
    try:
        for line in open("/proc/meminfo"):
            if line.startswith("MemAvailable:"):
                avail = int(line.split()[1]) * 1024
    except OSError:
        pass
    free, total = C.c_int64(), C.c_int64()
    gpu_ok = lib().fz_device_memory(int(device), C.byref(free), C.byref(total)) == 0
    need_host = 11.0 * nvox
    need_dev = (97.0 if precision == "fp64" else 49.0) * nvox
    over = 0.0
    if avail > 0 and need_host > 0.7 * avail:
        over = max(over, need_host / (0.7 * avail))
    if gpu_ok and need_dev > 0.9 * free.value:
        over = max(over, need_dev / (0.9 * free.value))
    min_h = h * over ** (1.0 / 3.0) if over > 0.0 else h
    if gpu_ok:  # effective air volume: air cells x h^3 (main3D.cu:445-446), from the GPU-built scene
        from .scenes import from_obj
        sc = from_obj(scene, h, device=device)
        print("[OK] estimate: V = %.3f m^3" % (float((sc.S > 0).sum()) * h ** 3), flush=True)
    print("[MEM] voxels=%d need_host_gb=%.3f need_dev_gb=%.3f free_host_gb=%.3f free_dev_gb=%.3f over=%.4f min_h=%.4g"
          % (nvox, need_host / 1e9, need_dev / 1e9, avail / 1e9, (free.value if gpu_ok else 0) / 1e9, over, min_h),
          flush=True)
    return 0


def main(argv=None):
    argv = list(sys.argv[1:] if argv is None else argv)
    if len(argv) < 4:
        print("Usage: fz3d <scene> <config> <src> <rec> [--fp64] [--estimate] [--keep-other-sources] [--no-autotune]")
        return 1
    precision = "fp64" if "--fp64" in argv else "fp32"
    scene, config, src, rec = argv[:4]
    if "--estimate" in argv:
        return estimate(scene, config, precision)
    if "--ga-only" in argv or "--dump-rays" in argv:
        print("[!] --ga-only / --dump-rays run the geometric-acoustics part (image sources, ray tracing), "
              "which this solver does not implement", flush=True)
        return 2
    purge_outputs(_project_output_dir(config), _src_index(config), "--keep-other-sources" in argv)
    s, nt = Solver.from_project(scene, config, src, rec, precision=precision)
    if nt >= 200 and "--no-autotune" not in argv:
        depth, _ = s.autotune()  # a few stage launches; pays for itself on runs of this length
        print(f"[OK] stage tile depth {depth} planes (autotuned)", flush=True)
    print(f"[OK] Will now start {nt} iterations", flush=True)
    t0 = time.perf_counter()
    s.run_progress(nt, lambda done, total: print("%d%%" % int(100.0 * done / total + 0.5), flush=True), 5)
    print("[OK] Simulation time: %f min" % ((time.perf_counter() - t0) / 60.0), flush=True)
    out = _project_output_dir(config)
    s.write_outputs(out, _src_index(config), os.path.abspath(scene))
    print("[OK] Printed header.txt for plot.py", flush=True)
    s.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
