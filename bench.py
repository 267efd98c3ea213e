"""Benchmark of the plain 3D FP32 stepper (SSP-RK3 step of WENO-Z / Godunov / cPML / ADE band).

Workload (one GPU): a 500 x 400 x 200-cell shoebox (10 x 8 x 4 m at h = 0.02 m; 506 x 406 x 206
padded cells), 5 seeded rigid box obstacles, 6 seeded passive ADE wall materials with 2 real
poles + 2 complex pairs, a 20-cell cPML on one open face, a Gaussian pressure pulse (sigma = 2
cells), c = 343 m/s, rho = 1.2 kg/m^3, CFL 0.5, 16 receivers. A step is one full SSP-RK3 time step
of every cell. Inputs are synthetic and seeded. The field sets (3 x 4 x 183 MB) exceed L2, so no
flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl fz|reference] [--room NX NY NZ]

The line states the result's accuracy: the e2e job's receiver traces against the all-FP64 path
on the same room, source and receivers (`accuracy`, rel-L2 per receiver; --no-accuracy skips that
run). The timed steps start with both step graphs instantiated (autotune, then graph set-up, then
the warm-up steps); clocks are sampled through NVML every 5 ms during them.

--impl reference times the CPU restatement of the reference update loop (the reference has no
CPU solver of its own; its CUDA solver has no library interface) on bounded z-slab samples of
the same room. Multi-GPU: independent replicas, one per rank (one solve runs on one GPU; a
second GPU solves its own room), max time over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gcell-updates/s (SSP-RK3 cell updates of the room per second, whole job)"
UNIT = "Gcell/s"
BYTES_PER_CELL_STEP = 131  # FP32: 4 fields x 4 B read/write over 3 stages (128 B) + 1 B class x 3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="fz", choices=["fz", "reference"])
    ap.add_argument("--room", type=int, nargs=3, default=[500, 400, 200])
    ap.add_argument("--e2e-steps", type=int, default=12000, help="length of the end-to-end job")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the all-FP64 run of the e2e job that gives the IR error of the FP32 result")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--config", default="plain3d", choices=["plain3d", "plain2d", "precision", "batched", "adjoint",
                                                            "legacy2d"],
                    help="plain3d: the headline room (default); plain2d: the 2D FP64 room; "
                         "precision: FP32 bulk vs all-FP64 on a 256^3 room; batched: 64 sources in one "
                         "192^3 room and 32 rooms in one graph; adjoint: misfit gradient on a 256^3 room; "
                         "legacy2d: the reference's 2D legacy scheme on an 803x815-node grid")
    return ap.parse_args()


def dist_setup(n):
    from fases_b200.replicas import Replicas
    rep = Replicas()
    return rep.rank, rep.world, rep.local, rep


def barrier(rep):
    rep.barrier()


def max_over_ranks(rep, x):
    return rep.max(x)


def _nvml_handle(device):
    """NVML handle of CUDA device `device` (matched by PCI bus id, so CUDA_VISIBLE_DEVICES and
    NVML's own ordering cannot disagree)."""
    import pynvml
    pynvml.nvmlInit()
    try:
        from cuda.bindings import runtime as rt
        err, bus = rt.cudaDeviceGetPCIBusId(32, device)
        if int(err) == 0:
            bus = bus.decode() if isinstance(bus, bytes) else str(bus)
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus.strip("\x00"))
    except Exception:
        pass
    return pynvml.nvmlDeviceGetHandleByIndex(device)


class Clocks:
    """SM clock, power and clock-event reasons sampled during the timed region: NVML from a
    thread every 5 ms (the timed region can be ~50 ms), nvidia-smi at 200 ms when NVML is
    unavailable."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4), ("hw_power_brake_slowdown", 0x80))

    def __init__(self, gpu, interval_s=0.005):
        self.gpu = gpu
        self.interval = interval_s
        self.rows = []  # (sm_mhz, sm_max_mhz, power_w, reasons bitmask)
        self.proc = None
        self.th = None
        self.stop = threading.Event()
        self.source = None

    def _nvml_loop(self, hd):
        import pynvml
        mx = pynvml.nvmlDeviceGetMaxClockInfo(hd, pynvml.NVML_CLOCK_SM)
        while not self.stop.is_set():
            try:
                sm = pynvml.nvmlDeviceGetClockInfo(hd, pynvml.NVML_CLOCK_SM)
                pw = pynvml.nvmlDeviceGetPowerUsage(hd) / 1000.0
                rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(hd)
                self.rows.append((float(sm), float(mx), pw, int(rs)))
            except Exception:
                pass
            self.stop.wait(self.interval)

    def _smi_read(self):
        for line in self.proc.stdout:
            r = [x.strip() for x in line.split(",")]
            try:
                mask = 0
                for (nm, bit), v in zip(self.REASONS[:4], r[4:8]):
                    if v.lower() == "active":
                        mask |= bit
                self.rows.append((float(r[0]), float(r[1]), float(r[2]), mask))
            except (ValueError, IndexError):
                pass

    def __enter__(self):
        try:
            hd = _nvml_handle(self.gpu)
            self.th = threading.Thread(target=self._nvml_loop, args=(hd,), daemon=True)
            self.th.start()
            self.source = "nvml, 5 ms"
            return self
        except Exception:
            pass
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._smi_read, daemon=True)
            self.th.start()
            self.source = "nvidia-smi, 200 ms"
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.th:
            self.th.join(timeout=5)

    def summary(self, quarters=False):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [r[0] for r in self.rows]
        reasons = sorted({nm for r in self.rows for nm, bit in self.REASONS if r[3] & bit})
        out = {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(r[1] for r in self.rows),
               "sm_mhz_min": min(sm), "power_w_max": max(r[2] for r in self.rows), "reasons": reasons,
               "samples": len(self.rows), "sampler": self.source}
        if quarters and len(self.rows) >= 8:
            # medians over each quarter of a long run: a drift of clock or power shows here
            q = np.array_split(np.array([(r[0], r[2]) for r in self.rows]), 4)
            out["sm_mhz_by_quarter"] = [float(np.median(x[:, 0])) for x in q]
            out["power_w_by_quarter"] = [round(float(np.median(x[:, 1])), 1) for x in q]
        return out


def workload(room):
    from fases_b200 import materials as mats
    from fases_b200 import scenes
    b = scenes.benchmark_room(room_cells=tuple(room))
    b["packed"] = mats.pack(b["materials"])
    return b


def make_solver(b, precision, capacity, device=0):
    from fases_b200 import Solver, params
    prm = params(h=b["h"], c=b["c"], rho=b["rho"], dt=b["dt"], pml=b["pml"], pml_cells=20, precision=precision,
                 device=device)
    s = Solver(prm)
    sc = b["scene"]
    s.load_geometry(sc.S, sc.oid)
    m = b["packed"]
    s.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
    s.set_receivers(b["receivers"], capacity)
    s.set_fields(p=b["p0"])
    return s


def cpu_baseline(room, steps=6, threads=None):
    """The FP64 CPU restatement on a z-slab sample of the room (same x-y extent, 24 cells high)."""
    from fases_b200 import materials as mats
    from fases_b200 import scenes
    from oracle.oracle import Oracle
    threads = threads or os.cpu_count()
    slab = (room[0], room[1], 24)
    b = scenes.benchmark_room(room_cells=slab, n_obstacles=0, n_receivers=2)
    sc = b["scene"]
    o = Oracle(sc.S, sc.oid, b["h"], b["c"], b["rho"], b["dt"], pml=b["pml"], materials=mats.pack(b["materials"]),
               rec_cells=b["receivers"], max_steps=steps + 1)
    o.set_fields(p=b["p0"])
    o.run(1, threads=threads)
    t = time.perf_counter()
    o.run(steps, threads=threads)
    dtm = time.perf_counter() - t
    cells = slab[0] * slab[1] * slab[2]
    return {"value": cells * steps / dtm / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} FP64 steps of a {slab[0]}x{slab[1]}x{slab[2]}-cell z-slab of the room, "
                      f"{threads} OpenMP threads, {dtm:.1f} s"}


def run_reference(args, rank):
    if rank != 0:
        return
    room = args.room
    from fases_b200 import materials as mats
    from fases_b200 import scenes
    from oracle.oracle import Oracle
    threads = os.cpu_count()
    slab = (room[0], room[1], 16)
    b = scenes.benchmark_room(room_cells=slab, n_obstacles=0, n_receivers=2)
    sc = b["scene"]
    o = Oracle(sc.S, sc.oid, b["h"], b["c"], b["rho"], b["dt"], pml=b["pml"], materials=mats.pack(b["materials"]),
               rec_cells=b["receivers"], max_steps=args.steps + args.warmup + 1)
    o.set_fields(p=b["p0"])
    o.run(args.warmup, threads=threads)
    t = time.perf_counter()
    o.run(args.steps, threads=threads)
    dtm = time.perf_counter() - t
    cells = slab[0] * slab[1] * slab[2]
    v = cells * args.steps / dtm / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dtm * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": f"plain 3D shoebox {room[0]}x{room[1]}x{room[2]}, sampled as a {slab[2]}-cell z-slab",
                   "room_cells": room, "sample_cells": list(slab)},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} FP64 steps of a {slab[0]}x{slab[1]}x{slab[2]}-cell z-slab per run"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def rel_l2(a, b):
    a = np.asarray(a, float)
    b = np.asarray(b, float)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run_plain2d(args):
    """Config 1: 256 x 256 planar room, FP64, 2000 steps (--steps overrides), 4 receivers; the IR
    error against the FP64 oracle on the whole run, and the oracle's own speed."""
    from fases_b200 import Solver, params
    from fases_b200 import materials as mats
    from fases_b200 import scenes
    from oracle.oracle import Oracle
    b = scenes.benchmark_2d()
    steps = args.steps if args.steps != 300 else 2000
    sc = b["scene"]
    m = mats.pack(b["materials"])
    prm = params(h=b["h"], c=b["c"], rho=b["rho"], dt=b["dt"], pml=b["pml"], pml_cells=b["pml_cells"],
                 precision="fp64", two_d=True)
    s = Solver(prm)
    s.load_geometry(sc.S, sc.oid)
    s.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
    s.set_receivers(b["receivers"], steps)
    s.set_fields(p=b["p0"])
    ms = s.run_timed(steps)
    ir = s.ir()
    s.close()
    cells = 256 * 256
    threads = os.cpu_count()
    o = Oracle(sc.S, sc.oid, b["h"], b["c"], b["rho"], b["dt"], pml=b["pml"], pml_cells=b["pml_cells"], materials=m,
               rec_cells=b["receivers"], max_steps=steps, two_d=True)
    o.set_fields(p=b["p0"])
    t = time.perf_counter()
    o.run(steps, threads=threads)
    t_cpu = time.perf_counter() - t
    ir_o, _ = o.ir()
    errs = [rel_l2(ir[r], ir_o[r]) for r in range(ir.shape[0])]
    print(json.dumps({
        "metric": "Gcell-updates/s, 2D FP64 (config 1)", "value": cells * steps / (ms / 1e3) / 1e9, "unit": UNIT,
        "n_gpus": 1, "steps": steps, "ms_per_step": ms / steps, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": "planar 256x256 room, h=0.02, 16-cell cPML on x-hi, rigid x-lo/y-hi, ADE y-lo "
                               "(2 real poles), Gaussian pulse sigma=3, 4 receivers", "room_cells": cells},
        "ir_rel_l2_vs_fp64_oracle": errs,
        "cpu_baseline": {"value": cells * steps / t_cpu / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"the full {steps}-step run, FP64, {t_cpu:.1f} s"}}), flush=True)


def run_legacy2d(args):
    """The 2D legacy scheme (include/fz_legacy2d.h) on a grid the size of the reference's shipped
    2D project (2D-solver/input/scene/hybridTST.obj: 4.006 x 4.067 m at h = 5 mm, 803 x 815 nodes)
    with two synthetic rectangular obstacles of two ADE materials (2 real poles, 1 complex pair),
    sPML on the y faces, the raised-cosine plane wave, FP32 as the reference; the CPU restatement
    (oracle, all host threads) timed on a bounded number of steps of the same grid."""
    from fases_b200.legacy2d import Legacy2D, plane_wave_fields, rect_scene
    from oracle.oracle import legacy2d_run
    Nx, Ny = 803, 815
    s = Legacy2D(Nx, Ny, precision=args.precision)
    P = s.params
    S, oid = rect_scene(Nx, Ny, P.h, [((1.4, 0.3), (1.5, 2.6), 1), ((2.4, 2.0), (3.2, 2.3), 2)])
    mats = {"Rinf": np.array([0.83, 0.7]),
            "A": np.array([[171.9, -343.5], [120.0, 0.0]]), "zeta": np.array([[317.2, 3796.2], [900.0, 0.0]]),
            "B": np.array([[-21.96], [15.0]]), "C": np.array([[-42.35], [-30.0]]),
            "alpha": np.array([[39.14], [600.0]]), "beta": np.array([[348.0], [1800.0]])}
    s.load_geometry(S, oid)
    s.set_materials(mats["Rinf"], mats["A"], mats["zeta"], mats["B"], mats["C"], mats["alpha"], mats["beta"])
    p0, u0, v0 = plane_wave_fields(Nx, Ny, P.h, 0.5, P.rho, P.c)
    s.set_fields(p0, u0, v0)
    steps = args.steps if args.steps != 300 else 2000
    warm = max(args.warmup, 64)  # builds the 32-step CUDA graph before the timed region
    s.set_receiver(Nx // 2, Ny // 2, warm + steps)
    s.run(warm)
    ms = s.run_timed(steps)
    ir = s.ir()
    nodes = (Nx - 6) * (Ny - 6)
    s.close()
    nb = 60
    t = time.perf_counter()
    legacy2d_run(S, oid, P.h, P.dt, P.rho, P.c, P.eps, P.tol, (P.pml_n, P.pml_s, P.pml_e, P.pml_w), mats, p0, u0, v0,
                 (Nx // 2, Ny // 2), nb, use_float=args.precision == "fp32")
    t_cpu = time.perf_counter() - t
    print(json.dumps({
        "metric": "Gnode-updates/s, 2D legacy scheme (WENO-JS, sPML, bicubic ADE boundary)",
        "value": nodes * steps / (ms / 1e3) / 1e9, "unit": "Gnode/s", "n_gpus": 1, "steps": steps,
        "warmup": warm, "ms_per_step": ms / steps, "higher_is_better": True,
        "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic (seeded)",
        "config": {"workload": "2D legacy scheme, 803x815 nodes (4.0 x 4.07 m at h=5 mm), 2 rectangular ADE "
                               "obstacles, sPML on y faces, raised-cosine plane wave, 1 receiver",
                   "interior_nodes": nodes, "timer": "CUDA events on the solve's stream",
                   "l2": "grid fits in L2 (3 buffers x 3 fields x 2.6 MB); no flush, as in a real run"},
        "finite": bool(np.isfinite(ir).all()),
        "cpu_baseline": {"value": nodes * nb / t_cpu / 1e9, "unit": "Gnode/s", "cores": os.cpu_count(),
                         "kind": "port",
                         "sample": f"{nb} steps of the same grid, the restatement on {os.cpu_count()} OpenMP threads, "
                                   f"{t_cpu:.1f} s"}}), flush=True)


def run_precision(args):
    """Config 3: 256^3 room with the config-2 material model; FP32 field state (FP64 ADE state,
    FP64 receiver samples) against all-FP64, per-receiver IR rel-L2 and energy drift."""
    from fases_b200 import materials as mats
    from fases_b200 import scenes
    steps = args.steps if args.steps != 300 else 30000
    b = scenes.benchmark_room(room_cells=(256, 256, 256), n_obstacles=5, n_receivers=8)
    b["packed"] = mats.pack(b["materials"])
    chunks = 10
    out = {}
    for prec in ("fp32", "fp64"):
        s = make_solver(b, prec, steps)
        E = [s.energy()]
        t_ms = 0.0
        for q in range(chunks):
            n = steps // chunks + (1 if q < steps % chunks else 0)
            t_ms += s.run_timed(n)
            E.append(s.energy())
        out[prec] = {"ir": s.ir(), "E": np.array(E), "ms": t_ms}
        s.close()
    ir32, ir64 = out["fp32"]["ir"], out["fp64"]["ir"]
    errs = [rel_l2(ir32[r], ir64[r]) for r in range(ir64.shape[0])]
    E32, E64 = out["fp32"]["E"], out["fp64"]["E"]
    drift = np.abs(E32 - E64) / np.maximum(E64, 1e-300)
    cells = 256 ** 3
    print(json.dumps({
        "metric": "precision study (config 3): FP32 bulk vs all-FP64", "steps": steps,
        "value": cells * steps / (out["fp32"]["ms"] / 1e3) / 1e9, "unit": UNIT,
        "fp64_gcell_s": cells * steps / (out["fp64"]["ms"] / 1e3) / 1e9,
        "ir_rel_l2_fp32_vs_fp64": errs, "ir_rel_l2_max": max(errs),
        "energy_fp64": E64.tolist(), "energy_rel_diff_fp32_vs_fp64": drift.tolist(),
        "energy_rel_change_fp64": float(E64[-1] / E64[0] - 1.0),
        "config": {"workload": "256^3 shoebox, 5 rigid obstacles, 6 ADE walls (2 real + 2 complex poles), "
                               "20-cell cPML on one face, Gaussian pulse, 8 receivers"}}), flush=True)


def _batched_solver(b, precision, capacity, cells, u_s, sval, batch=1, members=None):
    from fases_b200 import Solver, params
    s = Solver(params(h=b["h"], c=b["c"], rho=b["rho"], dt=b["dt"], pml=b["pml"], pml_cells=20,
                      precision=precision, batch=batch))
    sc = b["scene"]
    s.load_geometry(sc.S, sc.oid)
    m = b["packed"]
    s.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
    s.set_sources(cells, np.full(len(cells), sval), 0, u_s=u_s)
    if members is not None:
        s.set_source_members(members)
    s.set_receivers(b["receivers"], capacity)
    return s


def run_batched(args):
    """Config 4. (a) 64 seeded PCS source positions in one 192^3 room (6 ADE walls, 5 obstacles,
    cPML face): one batched solver (64 field sets stepped by the same launches) against one
    single-source solve of the same room, per-source throughput. (b) 32 rooms with edges drawn
    from [64, 160] cells per axis (seeded), advanced as one group (shared launches: per stage two
    stage launches of 16 rooms and one band launch for all, one CUDA graph per 10 steps) against the
    same rooms solved one after another."""
    from fases_b200 import Group, source_waveform
    from fases_b200 import materials as mats
    from fases_b200 import scenes
    steps_a = args.steps if args.steps != 300 else 200
    nsrc = 64
    b = scenes.benchmark_room(room_cells=(192, 192, 192), seed=4, n_obstacles=5, n_receivers=8)
    b["packed"] = mats.pack(b["materials"])
    rng = np.random.default_rng(44)
    cand = scenes.free_cells(b["scene"], scenes.seeded_cells(rng, (192, 192, 192), 4 * nsrc, margin_cells=24), 6.0)
    cells = np.asarray(cand[:nsrc], np.int32)
    us, _, pk = source_waveform(0, 0.25 * b["f_cutoff"], b["f_cutoff"], b["dt"], steps_a + 40, b["h"], b["rho"])
    room = 192 ** 3
    single = _batched_solver(b, "fp32", steps_a + 20, cells[:1], us, 1.0 / pk)
    single.run(20)
    depth_single, _ = single.autotune()  # both arms on their own tuned tile depth
    ms_single = single.run_timed(steps_a)
    ir_single = single.ir()
    single.close()
    bat = _batched_solver(b, "fp32", steps_a + 20, cells, us, 1.0 / pk, batch=nsrc, members=np.arange(nsrc))
    bat.run(20)
    depth_batch, _ = bat.autotune()
    ms_batch = bat.run_timed(steps_a)
    ir_batch = bat.ir()
    bat.close()
    per_src_single = room * steps_a / (ms_single / 1e3) / 1e9
    per_src_batch = nsrc * room * steps_a / (ms_batch / 1e3) / 1e9
    a_line = {
        "metric": "batched sources (config 4a): Gcell-updates/s per source, summed over sources",
        "value": per_src_batch, "unit": UNIT, "single_source_value": per_src_single,
        "per_source_speedup": per_src_batch / per_src_single, "steps": steps_a,
        "ms_per_step_batch": ms_batch / steps_a, "ms_per_step_single": ms_single / steps_a,
        "member0_bitwise_equal_single": bool(np.array_equal(ir_batch[0], ir_single)),
        "tile_depth": {"single": depth_single, "batch": depth_batch, "chosen_by": "fz_autotune"},
        "config": {"workload": "192^3 shoebox, 5 rigid obstacles, 6 ADE walls (2 real + 2 complex poles), "
                               "20-cell cPML on one face, 64 seeded PCS source positions, 8 receivers, FP32",
                   "sources": nsrc, "room_cells": room}}
    print(json.dumps(a_line), flush=True)

    steps_b = args.steps if args.steps != 300 else 5000
    nroom = 32
    rng = np.random.default_rng(45)
    rooms = [tuple(int(x) for x in rng.integers(64, 161, size=3)) for _ in range(nroom)]
    solvers, cells_b = [], 0
    for q, r in enumerate(rooms):
        bq = scenes.benchmark_room(room_cells=r, seed=100 + q, n_obstacles=2, n_receivers=4)
        bq["packed"] = mats.pack(bq["materials"])
        usq, _, pkq = source_waveform(0, 0.25 * bq["f_cutoff"], bq["f_cutoff"], bq["dt"], steps_b + 10, bq["h"],
                                      bq["rho"])
        src = np.asarray([bq["source_cell"]], np.int32)
        solvers.append((_batched_solver(bq, "fp32", steps_b, src, usq, 1.0 / pkq),
                        _batched_solver(bq, "fp32", steps_b, src, usq, 1.0 / pkq)))
        cells_b += r[0] * r[1] * r[2]
    ms_seq = 0.0
    for solo, _ in solvers:
        solo.autotune()  # each room alone on its own tuned tile depth
        solo.prepare()
        ms_seq += solo.run_timed(steps_b)
    grp = Group([g for _, g in solvers])
    depth_grp, _ = grp.autotune()  # tile depth and launch arrangement
    shared, branches = grp.shared_launches(), grp.branches()
    grp.run(10)  # the group's step graphs, outside the timed steps
    ms_grp = grp.run_timed(steps_b)
    # the arrangements the tuner did not keep, on a bounded number of steps (members keep running:
    # their traces beyond the first steps_b steps are not compared)
    arrangements = {}
    n_alt = min(steps_b, 1000)
    for mode in (-1, 1, 4):
        grp.set_branches(mode)
        grp.run(10)
        arrangements["member_branches" if mode < 0 else f"shared_{mode}_branches"] = \
            cells_b * n_alt / (grp.run_timed(n_alt) / 1e3) / 1e9
    same = all(np.array_equal(solo.ir(), g.ir()) for solo, g in solvers)
    grp.close()
    for solo, g in solvers:
        solo.close()
        g.close()
    b_line = {
        "metric": "grouped rooms (config 4b): Gcell-updates/s over all rooms",
        "value": cells_b * steps_b / (ms_grp / 1e3) / 1e9, "unit": UNIT,
        "sequential_value": cells_b * steps_b / (ms_seq / 1e3) / 1e9, "per_room_speedup": ms_seq / ms_grp,
        "steps": steps_b, "ms_group": ms_grp, "ms_sequential": ms_seq, "members_bitwise_equal_solo": same,
        "tile_depth_group": depth_grp, "shared_launches": shared, "branches": branches,
        "arrangements_gcell_s": arrangements,
        "config": {"workload": "32 shoeboxes, edges uniform in [64, 160] cells (seed 45), 2 rigid obstacles, "
                               "6 ADE walls, cPML face, PCS source, 4 receivers each, FP32",
                   "rooms": rooms, "room_cells_total": cells_b}}
    print(json.dumps(b_line), flush=True)


def run_adjoint(args):
    """Config 5: 256^3 room with the config-2 material model; misfit J = sum_r ||IR_r(theta) -
    IR_r(theta_true)||^2 over 8 receivers after 8000 FP32 steps (--steps overrides); gradient with
    respect to every ADE coefficient by the discrete adjoint with checkpoints every 100 steps.
    Reports the backward / forward device-time ratio."""
    from fases_b200 import materials as mats
    from fases_b200 import scenes
    steps = args.steps if args.steps != 300 else 8000
    seg = 100
    room = (256, 256, 256) if list(args.room) == [500, 400, 200] else tuple(int(x) for x in args.room)
    b = scenes.benchmark_room(room_cells=room, n_obstacles=5, n_receivers=8)
    b["packed"] = mats.pack(b["materials"])
    rng = np.random.default_rng(9)
    true = {k: np.array(v, dtype=np.float64, copy=True) for k, v in b["packed"].items()}
    for k in ("A", "B", "Cc"):
        true[k] = true[k] * (1.0 + 0.1 * rng.standard_normal(true[k].shape))
    bt = dict(b, packed=true)
    s = make_solver(bt, "fp32", steps)
    s.run(steps)
    target = s.ir()
    s.close()
    s = make_solver(b, "fp32", steps)
    g = s.misfit_gradient(target, nsteps=steps, segment_steps=seg)
    s.close()
    # the same pass with every gradient: sources, cPML profile, initial fields
    s = make_solver(b, "fp32", steps)
    g_all = s.misfit_gradient(target, nsteps=steps, segment_steps=seg, sources=True, pml=True, initial=True)
    s.close()
    s = make_solver(b, "fp32", steps)
    s.run(20)
    ms_plain = s.run_timed(steps) if steps <= 2000 else s.run_timed(2000) * steps / 2000.0
    s.close()
    cells = room[0] * room[1] * room[2]
    print(json.dumps({
        "metric": "adjoint (config 5): backward / forward device time", "value": g["backward_ms"] / g["forward_ms"],
        "unit": "ratio", "higher_is_better": False, "steps": steps, "segment_steps": seg,
        "forward_ms": g["forward_ms"], "backward_ms": g["backward_ms"], "plain_forward_ms": ms_plain,
        "forward_gcell_s": cells * steps / (g["forward_ms"] / 1e3) / 1e9, "J": g["J"],
        "grad_norm": float(np.linalg.norm(g["raw"])), "n_parameters": int(g["raw"].size),
        "all_gradients": {"value": g_all["backward_ms"] / g_all["forward_ms"], "forward_ms": g_all["forward_ms"],
                          "backward_ms": g_all["backward_ms"],
                          "what": "ADE coefficients + source strength and waveform + cPML R0/kappa_max/alpha_max "
                                  "+ initial fields",
                          "dJ_dpml": g_all["pml"], "dJ_dsval": [float(x) for x in g_all["sval"]]},
        "config": {"workload": f"{room[0]}x{room[1]}x{room[2]} shoebox, 5 rigid obstacles, 6 ADE walls (2 real + 2 complex poles), "
                               "20-cell cPML on one face, Gaussian pulse, 8 receivers, FP32; target from "
                               "A, B, C perturbed by 10 % (seed 9)"}}), flush=True)


def main():
    args = parse()
    rank, world, local, pg = dist_setup(args.gpus)
    # the reference arm and the side configurations run on rank 0 only; the other ranks leave
    side = {"plain2d": run_plain2d, "precision": run_precision, "batched": run_batched, "adjoint": run_adjoint,
            "legacy2d": run_legacy2d}
    if args.impl == "reference" or args.config in side:
        if rank == 0:
            if args.impl == "reference":
                run_reference(args, rank)
            else:
                side[args.config](args)
        pg.close()
        return
    room = args.room
    b = workload(room)
    room_cells = int(room[0]) * int(room[1]) * int(room[2])
    nsteps_total = args.warmup + args.steps
    s = make_solver(b, args.precision, nsteps_total + 31, device=local)
    info = s.info()
    depth, _ = s.autotune()  # z chunks of the stage kernels, timed on this room
    depth_heuristic = s.kz_chunk()[1]
    zsched = s.z_schedule()
    s.prepare()  # both step graphs instantiated and uploaded before the warm-up and the timed steps
    s.run(args.warmup)
    barrier(pg)
    # the timed steps: CUDA graphs of 10 steps, as fz_run issues them
    with Clocks(local) as clk:
        ms = s.run_timed(args.steps)
    ms = max_over_ranks(pg, ms)
    launches = args.steps * (3 + (3 if info["n_band"] > 0 else 0) + 1)
    value = world * room_cells * args.steps / (ms / 1e3) / 1e9
    # per-kernel device times from a shorter pass with events around every launch (no graphs)
    s.profile(True)
    s.run(min(args.steps, 30))
    prof = s.profile_read()
    s.profile(False)
    stage_ms = sum(prof[k][0] for k in ("stage0", "stage1", "stage2"))
    stage_launches = sum(prof[k][1] for k in ("stage0", "stage1", "stage2"))
    # roofline of the dominant kernel (the fused stage kernel): algorithmic bytes per launch over
    # its average launch time
    bytes_per_launch = room_cells * BYTES_PER_CELL_STEP / 3.0
    achieved = bytes_per_launch / (stage_ms / stage_launches / 1e3) / 1e9
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "stage_kernel_traffic.json")) as f:
            tr = json.load(f)
            traffic = tr.get("dram_bytes_per_launch_full_room")
    except Exception:
        pass
    ir_bench = s.ir()
    finite = bool(np.all(np.isfinite(ir_bench)))
    s.close()

    # end to end through the public API: host buffers in, full job, receiver traces out
    barrier(pg)
    from fases_b200 import Solver, params
    sc = b["scene"]
    m = b["packed"]
    ne = args.e2e_steps
    t0 = time.perf_counter()
    phases, t_mark = {}, [t0]

    def mark(name):  # host wall time of each part of the job (the calls below return when done)
        t = time.perf_counter()
        phases[name] = round(t - t_mark[0], 4)
        t_mark[0] = t

    prm = params(h=b["h"], c=b["c"], rho=b["rho"], dt=b["dt"], pml=b["pml"], pml_cells=20, precision=args.precision,
                 device=local)
    e = Solver(prm)
    mark("create")
    e.load_geometry(sc.S, sc.oid)
    mark("geometry_and_band")
    e.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
    e.set_receivers(b["receivers"], ne)
    e.set_fields(p=b["p0"])
    mark("materials_receivers_fields")
    e.autotune()
    mark("autotune")
    with Clocks(local, interval_s=0.05) as clk_e2e:
        e.run(ne)
        ir = e.ir()
    mark("steps")
    vel = e.vel()
    mark("readback")
    t_e2e = time.perf_counter() - t0
    e.close()
    t_e2e = max_over_ranks(pg, t_e2e)

    # accuracy of the e2e job: its receiver traces against the all-FP64 path on the same room,
    # source and receivers (the FP64 path matches the CPU oracle to 1e-10 on small rooms)
    accuracy = None
    if not args.no_accuracy and args.precision == "fp32":
        prm64 = params(h=b["h"], c=b["c"], rho=b["rho"], dt=b["dt"], pml=b["pml"], pml_cells=20, precision="fp64",
                       device=local)
        r64 = Solver(prm64)
        r64.load_geometry(sc.S, sc.oid)
        r64.set_materials(m["Rinf"], m["A"], m["zeta"], m["B"], m["Cc"], m["alpha"], m["beta"])
        r64.set_receivers(b["receivers"], ne)
        r64.set_fields(p=b["p0"])
        r64.autotune()
        t64 = time.perf_counter()
        r64.run(ne)
        ir64 = r64.ir()
        t64 = time.perf_counter() - t64
        r64.close()
        errs = [rel_l2(ir[r], ir64[r]) for r in range(ir64.shape[0])]
        accuracy = {"ir_rel_l2_vs_fp64": errs, "ir_rel_l2_max": max(errs), "steps": ne, "target": 1e-5,
                    "reference": "all-FP64 GPU path (FZ_FP64) on the same room, source and receivers",
                    "fp64_seconds": t64}
    h2d = sc.S.nbytes + sc.oid.nbytes + b["p0"].nbytes + sum(np.asarray(v).nbytes for v in m.values())
    d2h = ir.nbytes + vel.nbytes
    e2e = {"value": world * room_cells * ne / t_e2e / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d / ne,
           "d2h_bytes_per_step": d2h / ne, "steps": ne, "seconds": t_e2e, "phases_s": phases,
           "clocks": clk_e2e.summary(quarters=True),
           "timer": "host wall clock around create, geometry/material/field upload, autotune, run, IR/VEL readback"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(room)
        except Exception as ex:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {ex}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else "f64", "data": "synthetic (seeded)",
            "config": {"workload": f"plain 3D shoebox {room[0]}x{room[1]}x{room[2]} cells (h=0.02 m), 5 rigid "
                                   f"obstacles, 6 ADE walls (2 real + 2 complex poles), 20-cell cPML on one face, "
                                   f"Gaussian pulse, 16 receivers, FP32 state / FP64 ADE",
                       "room_cells": room_cells, "padded_cells": int(np.prod(info["dims"])),
                       "band_cells": info["n_band"], "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (3 field sets of 4 x 183 MB)",
                       "value_per_padded_cell": value * np.prod(info["dims"]) / room_cells,
                       "tile": {"columns": [32, 16], "depth": depth, "heuristic_depth": depth_heuristic,
                                "z_chunks": zsched, "chosen_by": "fz_autotune"}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "k_stage (fused WENO-Z/Godunov/RK/cPML/source), 131/3 B per room cell per launch",
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback"},
            "kernel_ms": {k: v[0] / max(v[1], 1) for k, v in prof.items()},
            "clocks": clk.summary(),
            "e2e": e2e,
            "gpu_launches": launches,
            "cpu_baseline": cpu,
            "finite": finite,
            "accuracy": accuracy,
        }
        print(json.dumps(line), flush=True)
    pg.close()


if __name__ == "__main__":
    main()
