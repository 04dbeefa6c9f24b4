"""Benchmark of the B200 element-loop hot path (one JSON line on rank 0).

Workload (the transonic bump channel): a 200 x 60 x 50 Kuhn-split box
(3.6 M tets, 625,311 nodes), bump amplitude 0.08, M_inf = 0.85, evaluated at
the five seeded potentials phi = U x + 0.01 U (smooth random modes), cycled
one per step.  A step is one fused residual + Newton Jacobian evaluation
(velocities, limiter, density, walk, upwinded density, sensitivities,
residual R and the Jacobian on the P1 pattern, plus Term 3) -- the work of
``NewtonWorkspace.eval_residual`` + ``assemble_coupled`` without a wake.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

value: device-timed Melem/s with inputs resident in HBM (the mesh data is
~1.3 GB, larger than L2, so no flush is needed between steps).
e2e:   the same through the public API with host buffers: each step copies
phi host->device and R + the Jacobian data device->host.
--impl reference: the CPU oracle (C/OpenMP restatement of the reference's
Numba kernels) on all host cores, same workload, rank 0 only.
"""

from __future__ import annotations

import argparse
import contextlib
import gc
import json
import os
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

MESH = (200, 60, 50)
AMPLITUDE = 0.08
M_INF = 0.85
N_STATES = 5


# The port against the reference's own Numba chain on one host (the
# reference cannot travel to the GPU box): 200x60x50, 8 cores, median of 3
# chains after JIT -- the port is the faster CPU baseline.
PORT_VS_NUMBA = {"host_cores": 8, "workload": "200x60x50 residual+Jacobian chain at seeded states",
                 "reference_numba_melem_s": 6.39, "port_melem_s": 10.42, "port_over_reference": 1.63}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2000)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--mesh", default="x".join(map(str, MESH)))
    p.add_argument("--e2e-steps", type=int, default=100)
    p.add_argument("--cpu-states", type=int, default=40)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--pocket-steps", type=int, default=300)
    p.add_argument("--order", default="given", choices=["given", "morton", "hilbert"],
                   help="node/element numbering of the device mesh")
    p.add_argument("--tune", default="auto",
                   help="launch shapes: 'auto' (autotuner), 'default', or "
                        "'persistent,threads_per_sm,row_lanes[,row_plan8]'")
    p.add_argument("--adjoint", default="100x30x25:0.05:0.80",
                   help="mesh:bump:Mach of the adjoint shape-gradient case ('' to skip)")
    p.add_argument("--batched", default="12:20x6x5:100x30x25:0.5:0.75",
                   help="cases:smallest:largest:mach_lo:mach_hi of the batched comparison ('' to skip); "
                        "the full batched configuration is 48:20x6x5:200x60x50:0.5:0.85")
    p.add_argument("--weighted", default="200x60x50:0.8",
                   help="mesh:mach of the weighted upwind timing ('' to skip)")
    p.add_argument("--wake", default="200x60x50",
                   help="channel mesh of the wake-elimination timing ('' to skip)")
    p.add_argument("--wall", default="100x30x25",
                   help="channel mesh of the wall-force timing ('' to skip)")
    p.add_argument("--lifting", default="100x30x25:0.7:2:40x12x10",
                   help="mesh:Mach:alpha:oracle_mesh of the wake-coupled (lifting) Newton solve ('' to skip)")
    p.add_argument("--naca", default="1", help="NACA0012 2.5D timings ('' to skip)")
    p.add_argument("--newton", default="200x60x50:0.08:0.70",
                   help="mesh:bump:Mach of the time-to-1e-10 Newton solves ('' to skip)")
    p.add_argument("--c4", default="320x96x80:0.05:0.75:0.70:0.025",
                   help="mesh:bump:Mach[:m_start[:dm]] of a one-run FP64 / mixed Newton comparison on the "
                        "large mesh (14.7 M tets, bump 0.05: M0.75 is below its choking Mach 0.7685) "
                        "('' to skip)")
    p.add_argument("--parity", type=int, default=2,
                   help="1: compare the timed states with the oracle after timing; 2: also the pocket states; "
                        "0: skip")
    p.add_argument("--linear", type=int, default=1,
                   help="1: SpMV / V-cycle / GMRES timings on the bench mesh's Jacobian")
    return p.parse_args()


def workload(shape):
    from up3d_b200.mesh.kuhn import bump_channel, seeded_state
    mesh = bump_channel(*shape, amplitude=AMPLITUDE, seed=0)
    phis = [seeded_state(mesh, s) for s in range(N_STATES)]
    return mesh, phis


def config_dict(shape, mesh):
    nx, ny, nz = shape
    d = {"workload": f"transonic bump channel {nx}x{ny}x{nz} Kuhn-split "
                     f"({mesh.n_tets} tets), M_inf {M_INF}, fused residual + Newton Jacobian "
                     f"at {N_STATES} seeded phi states",
         "mesh": f"{nx}x{ny}x{nz}", "n_tets": mesh.n_tets, "n_nodes": mesh.n_nodes,
         "m_inf": M_INF, "bump_amplitude": AMPLITUDE, "states": N_STATES,
         "l2": "inputs larger than L2 (mesh data ~1.3 GB >> 126 MB); no flush",
         "parallelism": "replicas"}
    return d


# ---------------------------------------------------------------- CPU side

def cpu_chain_timing(mesh, phis, n_states, threads):
    """The oracle's residual + Jacobian chain (its restatement of the
    reference kernels), timed on the host cores."""
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as O
    op, upw = oracle_ops(mesh)
    O.chain(op, upw, phis[0], M_INF)          # warm (page-in, thread pool)
    t0 = time.perf_counter()
    for k in range(n_states):
        O.chain(op, upw, phis[k % len(phis)], M_INF)
    dt = time.perf_counter() - t0
    return mesh.n_tets * n_states / dt / 1e6, dt, O.num_threads()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    shape = tuple(int(v) for v in args.mesh.split("x"))
    threads = os.cpu_count() or 1
    mesh, phis = workload(shape)
    os.environ["OMP_NUM_THREADS"] = str(threads)
    from oracle import oracle as O
    op = O.PicardOperator(mesh.nodes, mesh.elements)
    upw = O.UpwindOperator(mesh.nodes, mesh.elements)
    for w in range(min(max(args.warmup, 1), 3)):
        O.chain(op, upw, phis[w % N_STATES], M_INF)
    steps = max(1, min(args.steps, 20))
    t0 = time.perf_counter()
    for k in range(steps):
        O.chain(op, upw, phis[k % N_STATES], M_INF)
    dt = time.perf_counter() - t0
    value = mesh.n_tets * steps / dt / 1e6
    sample = (f"{steps} full-mesh residual+Jacobian chains (oracle restatement of the reference "
              f"Numba kernels, colour-ordered OpenMP) on {O.num_threads()} threads")
    line = {"impl": "reference", "metric": "residual+Jacobian Melem/s", "value": round(value, 4),
            "unit": "Melem/s", "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * dt / steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(shape, mesh),
            "cpu_baseline": {"value": round(value, 4), "unit": "Melem/s",
                             "cores": O.num_threads(), "kind": "port", "sample": sample,
                             "port_vs_reference_numba": PORT_VS_NUMBA},
            "e2e": {"value": round(value, 4), "unit": "Melem/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- clocks

class ClockSampler:
    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str | None):
        self.bus_id = bus_id
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                   "-lms", "100"]
            if self.bus_id:
                cmd += ["-i", self.bus_id]
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(cmd, stdout=self.out, stderr=subprocess.DEVNULL)
            time.sleep(0.25)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.out.close()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[4:8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v == "Active"})
        sm = [r[0] for r in rows]
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(r[1] for r in rows),
                "samples": len(rows), "reasons": reasons}


# ---------------------------------------------------------------- GPU side

def bytes_model(info, n_active=0):
    """Compulsory bytes per launch of the fused residual + Jacobian, Layout A
    (the reference's stored geometry: B, V, int32 maps): every API input read
    once and every output written once, intermediates free.  The element
    sweep's share is its inputs (conn, B, V, face neighbours, centroids,
    node coordinates, phi) and the upstream output; the row gather's share is
    the scatter map (elem_to_csr as int32) and the outputs R and J.  Term 3
    adds 16 COO triplets (8 + 4 + 4 bytes) per active element.

    `design` counts what this library's layout moves instead: the sweep
    recomputes B and V from the node coordinates (no 104 bytes per element)
    but reads the walk's face displacements and round-trips the local
    matrices between the two kernels."""
    E, N, Z = info["n_tets"], info["n_nodes"], info["nnz"]
    elem = E * (16 + 96 + 8 + 16 + 24 + 4) + N * (24 + 8)
    row = E * 64 + N * 8 + Z * 8
    t3 = n_active * 16 * 16
    design_elem = (E * (16 + 16 + 96 + 4 + 14 * 8 + 1) + N * (24 + 8))
    design_row = (E * (16 + 24 + 14 * 8) + Z * (4 + 4 + 8) + N * (4 * 3 + 8))
    out = {"elem_sweep": elem, "row_gather": row, "term3": t3, "fused": elem + row + t3,
           "design": {"elem_sweep": design_elem, "row_gather": design_row}}
    ti = info.get("tiles")
    if ti:
        # the tiled form: per element its local connectivity (8), internal
        # face neighbours (16), id map (4), upstream out (4), Term-3 flag
        # (1), node entries (2 x 4) and edge contributors (2 x 6); per
        # tile-node its global id (4), offset (4), destination (8) and the
        # staged position + potential (32 + 8, L2 hits where tiles share
        # nodes); per tile-edge its offset (4) and destination (8); every
        # partial written and read (8 + 8) with its combine index (4); the
        # outputs R and J
        out["design"]["tile_eval"] = (E * (8 + 16 + 4 + 4 + 1 + 8 + 12) + ti["n_tile_nodes"] * (4 + 4 + 8 + 40)
                                      + ti["n_tile_edges"] * (4 + 8) + ti["n_partials"] * (8 + 8 + 4)
                                      + N * 8 + Z * 8)
    return out


def read_peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def read_traffic(kernel: str, n_tets: int):
    """DRAM bytes per launch at n_tets from a committed ncu summary (its
    measured bytes per element times the element count), if one exists."""
    import re
    for f in sorted((REPO / "profiles").glob(f"{kernel}*.md")):
        for line in f.read_text().splitlines():
            if line.startswith("dram_bytes_per_launch_full_size:"):
                m = re.search(r"\(([0-9.]+) B/elem", line)
                return None if m is None else round(float(m.group(1)) * n_tets)
    return None


@contextlib.contextmanager
def settled_gc():
    """Wall-clock solve timings: the cyclic garbage of earlier runs (device
    buffers of dropped workspaces among it) is collected before the clock
    starts and the cyclic collector stays off until it stops, so that no
    collection, and no implicit device synchronisation of the buffers it
    frees, lands inside a timed solve."""
    gc.collect()
    gc.disable()
    try:
        yield
    finally:
        gc.enable()


def empty_pool():
    """Each solver leg starts from an empty device block cache: the blocks
    that earlier legs left cached are released here, outside any clock,
    instead of being evicted (deferred cudaFree calls) inside a timed solve."""
    from up3d_b200 import _lib as L
    gc.collect()
    L.pool_release()


def newton_timing(spec, reps=4):
    """Time-to-1e-10 of the device Newton solve (Picard seed, exact
    Jacobian, GMRES + AMG, line search, frozen finish) from the freestream
    potential, plain FP64 and mixed precision (FP32 Jacobian SpMV and FP32
    AMG inside FP64-refined GMRES), each after an untimed solve of the same
    case; wall clock with the device synchronised."""
    import torch
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.solve.newton import ChannelWorkspace, solve_newton_transonic
    parts = spec.split(":")
    shape_s, amp_s, mach_s = parts[:3]
    shape = tuple(int(v) for v in shape_s.split("x"))
    amp, mach = float(amp_s), float(mach_s)
    m_start = float(parts[3]) if len(parts) > 3 else mach
    dm_step = float(parts[4]) if len(parts) > 4 else 0.05
    mesh = bump_channel(*shape, amplitude=amp, seed=0)
    from up3d_b200.mesh.kuhn import choking_mach
    out = {"case": f"bump channel {shape_s} Kuhn-split ({mesh.n_tets} tets), bump {amp}, "
                   f"M_inf {mach}" + (f" (Mach ramp from {m_start} by {dm_step})" if m_start < mach else "")
                   + ", from freestream to |R_free|inf < 1e-10",
           "n_tets": mesh.n_tets,
           "choking_mach_quasi_1d": round(choking_mach(amp), 4),
           "timed_runs": (f"median of {reps - 1} after an untimed one (each with a fresh workspace)" if reps > 1
                          else "first (workspace and tile plan built before the clock)")}
    phis = {}
    for prec in ("fp64", "mixed"):
        empty_pool()
        runs = []
        for rep_ in range(reps):
            ws = None
            with settled_gc():
                ws = ChannelWorkspace(mesh.nodes, mesh.elements, mesh.dirichlet_nodes)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                r = solve_newton_transonic(ws, mach, m_start=m_start, dm=dm_step, precision=prec)
                torch.cuda.synchronize()
                dt = time.perf_counter() - t0
            if reps == 1 or rep_ > 0:
                runs.append((dt, r))
        runs.sort(key=lambda x: x[0])
        dt, res = runs[len(runs) // 2]
        phis[prec] = res["phi"]
        out[prec] = {"time_s": round(dt, 4), "runs_s": [round(x[0], 4) for x in runs],
                     "converged": bool(res["converged"]),
                     "final_residual": float(res["residual_history"][-1]),
                     "n_newton": int(sum(lv[1] for lv in res["level_history"])),
                     "n_gmres": int(sum(lv[3] for lv in res["level_history"])),
                     "n_refinements": int(res.get("n_refinements", 0)),
                     "n_supersonic": int(res["n_supersonic"]),
                     "phases_s": {k: round(v, 4) for k, v in res["timings"].items()}}
        out[prec]["levels"] = [[round(float(lv[0]), 4), int(lv[1]), float(lv[2])] for lv in res["level_history"]]
    out["mixed_vs_fp64_max_dphi"] = float((phis["mixed"] - phis["fp64"]).abs().max())
    out["speedup_mixed"] = round(out["fp64"]["time_s"] / out["mixed"]["time_s"], 3)
    return out


def adjoint_timing(spec):
    """Shape (16 Gaussian bump modes) and Mach gradient of the lift-like
    wall integral through the device adjoint: forward continuation solve
    from M 0.70, then one transpose solve and two vector-Jacobian products;
    the second of two runs is timed."""
    import torch
    from up3d_b200.adjoint import BumpShape, adjoint_gradient
    shape_s, amp_s, mach_s = spec.split(":")
    nx, ny, nz = (int(v) for v in shape_s.split("x"))
    shape = BumpShape(nx, ny, nz, amplitude=float(amp_s), seed=0)
    mach = float(mach_s)
    g = None
    empty_pool()
    for _ in range(2):
        with settled_gc():
            g = adjoint_gradient(shape, mach, m_start=min(0.70, mach))
    torch.cuda.synchronize()
    return {"case": f"bump channel {shape_s} ({len(shape.elements)} tets), bump {amp_s}, M_inf {mach}, "
                    f"{shape.n_params} shape modes + Mach",
            "objective": g["F"], "dF_dM": g["dF_dM"],
            "dF_dp_norm": float(np.linalg.norm(g["dF_dp"])),
            "forward_s": round(g["timings"]["forward_s"], 4),
            "adjoint_s": round(g["timings"]["adjoint_s"], 4),
            "transpose_gmres_iterations": int(g["gmres_iterations"]),
            "check": "tests/test_gpu_adjoint.py: finite differences to 1e-6 relative"}


def weighted_timing(spec):
    """The weighted upwind densities (UpwindOperator(weighted=True), modes
    "kernel" and "blend", kernels/upwind.py:176-454) on a channel mesh at
    the three supersonic-pocket states: device time per sweep (CUDA events,
    inputs resident), the neighbourhood build, and the oracle's time on the
    box's host cores for the same sweep (a bounded sample: one state)."""
    import torch
    from oracle import oracle as O
    from up3d_b200.kernels.upwind import UpwindOperator
    from up3d_b200.mesh.kuhn import bump_channel, pocket_state
    mesh_s, mach_s = spec.split(":")
    shape = tuple(int(v) for v in mesh_s.split("x"))
    M = float(mach_s)
    m = bump_channel(*shape, amplitude=AMPLITUDE, seed=0)
    op = O.PicardOperator(m.nodes, m.elements)
    states = []
    for fam in ("accelerating", "shockpoint", "mixed"):
        grad, q2 = op.velocities(pocket_state(m, fam))
        q2l = O.limit_q2_field(q2, M, 3.0)
        rho = O.density_field(q2l, M)
        states.append((grad.copy(), q2l, rho))
    dev = [tuple(torch.from_numpy(a).cuda() for a in st) for st in states]
    out = {"mesh": mesh_s, "n_tets": int(m.n_tets), "m_inf": M}
    for mode in ("kernel", "blend"):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        upw = UpwindOperator(m.nodes, m.elements, weighted=True, mode=mode)
        torch.cuda.synchronize()
        setup_s = time.perf_counter() - t0
        for k in range(3):
            upw.rho_tilde(*dev[k], M, 1.5, 0.95)
        reps = 30
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record()
        for k in range(reps):
            upw.rho_tilde(*dev[k % 3], M, 1.5, 0.95)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / reps
        ref = O.UpwindOperator(m.nodes, m.elements, weighted=True, mode=mode)
        t0 = time.perf_counter()
        r = ref.rho_tilde(*states[0], M, 1.5, 0.95).copy()
        cpu_s = time.perf_counter() - t0
        d = upw.rho_tilde(*dev[0], M, 1.5, 0.95).cpu().numpy()
        out[mode] = {"ms_per_sweep": round(ms, 4), "melem_s": round(m.n_tets / ms / 1e3, 1),
                     "setup_s": round(setup_s, 4),
                     "n_supersonic": int(upw.n_supersonic),
                     "cpu_oracle_s": round(cpu_s, 4), "cpu_cores": O.num_threads(),
                     "max_rel_err_vs_oracle": float(np.abs(d - r).max() / np.abs(r).max())}
        if mode == "kernel":
            out[mode]["neighbors_per_element"] = round(float(len(upw._nb_idx)) / m.n_tets, 2)
    return out


def wake_timing(spec):
    """The wake master-slave elimination (constraints/wake.py:59-97) on a
    plane sheet cut into the channel (the sheet at mid-height over the
    downstream half, one station per spanwise line): A_red = T^T A T and
    the Gamma columns H for a matrix on the cut mesh's P1 pattern.  Device
    time per reduction (CUDA events, A resident), the host symbolic phase
    once per pattern, and the oracle's scipy reduction on the host."""
    import torch
    from oracle import oracle as O
    from up3d_b200 import _lib as L
    from up3d_b200.constraints.wake import WakeConstraint
    from up3d_b200.mesh.device import DeviceCSR, DeviceMesh
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.mesh.wake_cut import cut_channel_sheet
    shape = tuple(int(v) for v in spec.split("x"))
    cut = cut_channel_sheet(bump_channel(*shape, amplitude=AMPLITUDE, seed=0))
    dm = DeviceMesh(cut.nodes, cut.elements)
    g = torch.Generator(device="cuda").manual_seed(3)
    A = DeviceCSR(dm.indptr, dm.indices, torch.rand(dm.nnz, dtype=torch.float64, device="cuda", generator=g),
                  (dm.n_nodes, dm.n_nodes))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    con = WakeConstraint(A, cut.wc)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    plan = con._plan
    red = torch.empty(plan.nnz_red, dtype=torch.float64, device="cuda")
    h = torch.empty(max(plan.nnz_h, 1), dtype=torch.float64, device="cuda")

    def once():
        L.call("up3d_wake_reduce", plan.handle, A.data.data_ptr(), red.data_ptr(), h.data_ptr(), L.stream_ptr())
    for _ in range(3):
        once()
    reps = 50
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(reps):
        once()
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    A_h = A.to_scipy()
    t0 = time.perf_counter()
    ref = O.WakeConstraint(A_h, cut.wc)
    cpu_s = time.perf_counter() - t0
    err = float(np.abs(red.cpu().numpy() - ref.A_reduced.data).max() / np.abs(ref.A_reduced.data).max())
    bytes_moved = 8 * plan.nnz_a + 8 * plan.nnz_red + 16 * plan.nnz_red + 8 * plan.nnz_h
    return {"mesh": spec, "n_cut": int(dm.n_nodes), "n_red": int(plan.n_red),
            "n_slaves": int(len(cut.wc.slave_nodes)), "n_stations": int(cut.wc.n_stations),
            "nnz_a": int(plan.nnz_a), "nnz_red": int(plan.nnz_red), "nnz_h": int(plan.nnz_h),
            "ms_per_reduce": round(ms, 4), "gbs": round(bytes_moved / (ms * 1e-3) / 1e9, 1),
            "symbolic_s": round(setup_s, 3), "cpu_oracle_s": round(cpu_s, 3),
            "max_rel_err_vs_oracle": err}


def lifting_timing(spec):
    """Wake-coupled Newton (solve_newton_lifting, solve/newton.py:516-1141,
    probe Kutta estimator) on a bump channel cut by a plane sheet normal to
    y with the far-field vortex on the trailing-edge line: time from the
    freestream to |R_f|inf < 1e-10 and |F|inf < 1e-8 on the device
    (GMRES(60) on the coupled operator, AMG on the reduced Picard block,
    the frozen-selection finish from |R| < 1e-6 or a stall), the upward
    Mach continuation to M + 0.05 from M - 0.1 (solve_newton_transonic,
    :1144-1307), and, on a smaller mesh, the device solve beside the
    oracle's exact-step (sparse LU + Woodbury) solve on the host, both with
    the live selection, with the distance between their solutions."""
    import torch
    from oracle import oracle as O
    from up3d_b200.constraints.dirichlet import FarfieldBasis, freestream_phi
    from up3d_b200.mesh.kuhn import bump_channel
    from up3d_b200.mesh.wake_cut import channel_vortex_center, cut_channel_sheet
    from up3d_b200.solve.lifting import NewtonWorkspace, solve_newton_lifting, solve_newton_transonic
    parts = spec.split(":")
    shape = tuple(int(v) for v in parts[0].split("x"))
    m_inf, alpha = float(parts[1]), float(parts[2])

    def case(sh):
        cut = cut_channel_sheet(bump_channel(*sh, amplitude=AMPLITUDE, seed=0), normal="y")
        return cut, channel_vortex_center(cut)

    def device_solve(cut, vc, freeze_tol):
        t0 = time.perf_counter()
        ws = NewtonWorkspace(cut, cut.wc, alpha, vortex_center=vc)
        torch.cuda.synchronize()
        setup = time.perf_counter() - t0
        res = solve_newton_lifting(cut, cut.wc, m_inf, alpha_deg=alpha, vortex_center=vc, workspace=ws,
                                   n_picard_seed=0, freeze_tol=freeze_tol)
        return ws, res, setup

    cut, vc = case(shape)
    empty_pool()
    device_solve(cut, vc, 1e-6)                # warm-up (library, mesh caches)
    with settled_gc():
        ws, res, setup = device_solve(cut, vc, 1e-6)
    out = {"case": f"bump channel {parts[0]} Kuhn-split, y-normal wake sheet from x = {vc[0]:.2f}, "
                   f"M_inf {m_inf}, alpha {alpha} deg, from the freestream",
           "n_tets": int(len(cut.elements)), "n_red": int(ws.n_red), "n_stations": int(ws.n_st),
           "time_s": round(res["timings"]["wall"], 4), "setup_s": round(setup, 3),
           "converged": bool(res["converged"]), "n_newton": int(res["n_newton"]),
           "n_gmres": int(res["n_gmres_total"]), "n_freeze_refresh": int(res["n_freeze_refresh"]),
           "final_residual": res["residual_history"][-1], "final_F": res["F_history"][-1],
           "n_supersonic": int(res["n_nu_active"]), "n_term3_active": int(res["n_term3_active"]),
           "phases_s": {k: round(v, 4) for k, v in res["timings"].items()}}
    with settled_gc():
        t0 = time.perf_counter()
        cont = solve_newton_transonic(cut, cut.wc, m_inf + 0.05, alpha, m_start=m_inf - 0.1,
                                      newton_kw={"vortex_center": vc})
        cont_s = time.perf_counter() - t0
    out["continuation"] = {"mach": [round(m_inf - 0.1, 3), round(m_inf + 0.05, 3)],
                           "time_s": round(cont_s, 3), "converged": bool(cont["converged"]),
                           "levels": [[round(m, 4), n, r] for m, n, r in cont["level_history"]],
                           "n_supersonic": int(cont["n_nu_active"])}
    if len(parts) > 3 and parts[3]:
        sh = tuple(int(v) for v in parts[3].split("x"))
        cut, vc = case(sh)
        ws, res, _ = device_solve(cut, vc, None)
        basis = FarfieldBasis(cut, cut.wc, alpha, 1.0, vc)
        vals0, V = basis.at_mach(float(np.sqrt(1.0 - m_inf ** 2)))
        sysm = O.LiftingSystem(cut.nodes, cut.elements, cut.wc, basis.dir_red, vals0, V)
        phi0 = freestream_phi(cut.nodes[:sysm.n_red], alpha, 1.0)
        t0 = time.perf_counter()
        phi_o, gam_o, hist, ok = sysm.solve(phi0[sysm.free], np.zeros(sysm.n_st), m_inf)
        cpu_s = time.perf_counter() - t0
        out["oracle_comparison"] = {
            "mesh": parts[3], "n_tets": int(len(cut.elements)), "device_s": round(res["timings"]["wall"], 4),
            "device_converged": bool(res["converged"]), "device_n_newton": int(res["n_newton"]),
            "cpu_oracle_s": round(cpu_s, 3), "cpu_oracle_n_newton": len(hist) - 1,
            "cpu_oracle_converged": bool(ok), "cpu_cores": O.num_threads(),
            "max_abs_phi_diff": float(np.abs(res["phi"].cpu().numpy() - phi_o).max()),
            "max_abs_gamma_diff": float(np.abs(res["gamma"].cpu().numpy() - gam_o).max())}
    return out


def naca_timing():
    """The reference's own NACA0012 2.5D meshes (read from MSH 2.2 by
    up3d_b200.mesh.reader; arrays in tests/golden): (1) the Picard matrix
    assembly on the medium mesh (61,788 tets), the one hot-path timing the
    reference publishes (2.1 ms per call, colour-ordered Numba, 16 threads:
    cases/demo/p3_subsonic/results/assembly_debt.csv), timed on the device
    (CUDA events, median of 50) and by the oracle on the host; (2) the
    lifting Newton on the coarse mesh cut by the reference's cut_wake at
    the reference's own subsonic case (M0.5, alpha 1.25 deg; published
    conforming Newton 2.716 s wall including a 1.92 s Picard seed,
    cases/analysis/a1_solver_bottleneck/results/a1_runs.csv:3), from the
    freestream on the device, beside the oracle's exact-step solve; (3)
    the nested lifting Picard on the coarse mesh at the same case
    (published 6.247 s, 15 outer iterations, 35 linear solves:
    a1_runs.csv:2)."""
    import torch
    from oracle import oracle as O
    from up3d_b200.constraints.dirichlet import FarfieldBasis, freestream_phi
    from up3d_b200.kernels.jacobian import PicardOperator
    from up3d_b200.mesh.wake_cut import load_cut
    from up3d_b200.solve.lifting import NewtonWorkspace, solve_newton_lifting
    golden = REPO / "tests" / "golden"
    med = np.load(golden / "naca_medium_mesh.npz")
    nodes, elements = med["nodes"], med["elements"]
    op = PicardOperator(torch.as_tensor(nodes).cuda(), torch.as_tensor(elements).cuda())
    rho = torch.rand(len(elements), dtype=torch.float64, device="cuda") + 0.5
    for _ in range(5):
        op.assemble_matrix(rho)
    times = []
    for _ in range(50):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        op.assemble_matrix(rho)
        b.record()
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b))
    dev_ms = float(np.median(times))
    oop = O.PicardOperator(nodes, elements)
    rho_h = rho.cpu().numpy()
    oop.assemble_matrix(rho_h)
    t0 = time.perf_counter()
    for _ in range(10):
        A_h = oop.assemble_matrix(rho_h)
    cpu_ms = (time.perf_counter() - t0) / 10 * 1e3
    A_d = op.assemble_matrix(rho).to_scipy()
    err = float(np.abs(A_d.data - A_h.data).max() / np.abs(A_h.data).max())
    out = {"picard_assembly_medium": {
        "n_tets": int(len(elements)), "n_nodes": int(len(nodes)), "device_ms": round(dev_ms, 4),
        "device_melem_s": round(len(elements) / (dev_ms * 1e-3) / 1e6, 1),
        "reference_published_ms": 2.1, "cpu_oracle_ms": round(cpu_ms, 3), "cpu_cores": O.num_threads(),
        "max_rel_diff_vs_oracle": err}}
    g = np.load(golden / "naca_coarse.npz")
    mc, wc = load_cut(g)
    m_inf, alpha = 0.5, 1.25
    solve_newton_lifting(mc, wc, m_inf, alpha_deg=alpha, n_picard_seed=0)   # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ws = NewtonWorkspace(mc, wc, alpha)
    res = solve_newton_lifting(mc, wc, m_inf, alpha_deg=alpha, n_picard_seed=0, workspace=ws)
    torch.cuda.synchronize()
    dev_s = time.perf_counter() - t0
    basis = FarfieldBasis(mc, wc, alpha, 1.0)
    vals0, V = basis.at_mach(float(np.sqrt(1.0 - m_inf ** 2)))
    t0 = time.perf_counter()
    sysm = O.LiftingSystem(mc.nodes, mc.elements, wc, basis.dir_red, vals0, V)
    phi0 = freestream_phi(mc.nodes[:sysm.n_red], alpha, 1.0)
    phi_o, gam_o, hist, ok = sysm.solve(phi0[sysm.free], np.zeros(sysm.n_st), m_inf)
    cpu_s = time.perf_counter() - t0
    from up3d_b200.solve.lifting import solve_subsonic_lifting
    solve_subsonic_lifting(mc, wc, m_inf, alpha_deg=alpha, workspace=ws)        # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pic = solve_subsonic_lifting(mc, wc, m_inf, alpha_deg=alpha, workspace=NewtonWorkspace(mc, wc, alpha))
    torch.cuda.synchronize()
    out["picard_coarse_m05"] = {
        "device_s": round(time.perf_counter() - t0, 4), "converged": bool(pic["converged"]),
        "n_picard": int(pic["n_picard"]), "n_lin_solves": int(pic["n_solves_total"]),
        "n_cg": int(pic["n_cg_total"]), "gamma": float(pic["gamma"].mean()),
        "reference_published": {"wall_s": 6.247, "n_outer": 15, "n_lin_solves": 35, "n_lin_iters": 5381,
                                "source": "cases/analysis/a1_solver_bottleneck/results/a1_runs.csv:2"}}
    from up3d_b200.solve.lifting import solve_newton_transonic
    recipe = dict(m_start=0.70, dm=0.025, dm_min=0.003, freeze_tol=1e-6,
                  newton_kw=dict(freeze_refresh_max=8, precond="direct", n_newton_max=60, n_picard_seed=0))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tr = solve_newton_transonic(mc, wc, 0.8, alpha, **recipe)
    torch.cuda.synchronize()
    out["transonic_coarse_m08"] = {
        "device_s": round(time.perf_counter() - t0, 3), "converged": bool(tr["converged"]),
        "levels": [[round(m, 4), n] for m, n, _ in tr["level_history"]],
        "n_newton_total": int(sum(n for _, n, _ in tr["level_history"])), "gamma": float(tr["gamma"][0]),
        "n_supersonic": int(tr["n_nu_active"]),
        "recipe": "Mach ramp 0.70 -> 0.80 by 0.025, freeze 1e-6, exact (dense LU) steps, from the freestream",
        "reference_published": {"wall_s": 4.712, "n_levels": 5, "n_newton": 57, "gamma": 0.233826,
                                "note": "with a Picard warm start (2.689 s of it) and sparse LU, 16 threads",
                                "source": "cases/analysis/a1_solver_bottleneck/results/a1_runs.csv:7"}}
    # the medium mesh end to end: cut, then the lifting Newton at M0.5
    from up3d_b200.mesh.reader import Mesh
    from up3d_b200.mesh.wake_cut import cut_wake
    mm = Mesh()
    mm.nodes, mm.elements = nodes, elements
    mm.boundary_faces = {k.split("/", 1)[1]: med[k] for k in med.files if k.startswith("faces/")}
    mm.element_tags = np.zeros(len(elements), dtype=np.int32)
    mm.tag_names = ["fluid"]
    t0 = time.perf_counter()
    mcm, wcm = cut_wake(mm)
    cut_s = time.perf_counter() - t0
    solve_newton_lifting(mcm, wcm, 0.5, alpha_deg=1.25, n_picard_seed=0)             # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rm = solve_newton_lifting(mcm, wcm, 0.5, alpha_deg=1.25, n_picard_seed=0,
                              workspace=NewtonWorkspace(mcm, wcm, 1.25))
    torch.cuda.synchronize()
    out["lifting_medium_m05"] = {
        "n_tets": int(len(elements)), "n_copies": int(len(wcm.slave_nodes)), "cut_wake_s": round(cut_s, 3),
        "device_s": round(time.perf_counter() - t0, 4), "converged": bool(rm["converged"]),
        "n_newton": int(rm["n_newton"]), "n_gmres": int(rm["n_gmres_total"]), "gamma": float(rm["gamma"][0])}
    out["lifting_coarse_m05"] = {
        "n_tets": int(len(mc.elements)), "n_stations": int(wc.n_stations), "m_inf": m_inf, "alpha_deg": alpha,
        "device_s": round(dev_s, 4), "device_converged": bool(res["converged"]),
        "device_n_newton": int(res["n_newton"]), "device_n_gmres": int(res["n_gmres_total"]),
        "gamma_mean": float(res["gamma"].mean()), "reference_published_wall_s": 2.716,
        "reference_published_note": "conforming Newton with a 5-step Picard seed (1.919 s), 16 threads",
        "cpu_oracle_s": round(cpu_s, 3), "cpu_oracle_n_newton": len(hist) - 1, "cpu_oracle_converged": bool(ok),
        "max_abs_phi_diff_vs_oracle": float(np.abs(res["phi"].cpu().numpy() - phi_o).max())}
    return out


def wall_timing(spec):
    """Wall Cp and pressure forces (post/surface.py:309-363) on the
    channel's lower wall at a pocket state, M0.8, two smoothing passes:
    time per evaluation on a wall handle (CUDA events; each evaluation ends
    with the 3-value read-back), one call through the public function, the
    one-time owner/adjacency set-up, and the oracle's numpy evaluation on
    the host."""
    import torch
    from oracle import oracle as O
    from up3d_b200.adjoint import lower_wall_faces
    from up3d_b200.mesh.kuhn import bump_channel, pocket_state
    from up3d_b200.post.surface import wall_force_coefficients
    shape = tuple(int(v) for v in spec.split("x"))
    m = bump_channel(*shape, amplitude=AMPLITUDE, seed=0)
    wf = lower_wall_faces(m.elements, m.shape)[:, 1:]
    phi = torch.from_numpy(pocket_state(m, "mixed")).cuda()
    t0 = time.perf_counter()
    r = wall_force_coefficients(m.nodes, m.elements, wf, phi, m_inf=0.8, smooth_passes=2)
    setup_s = time.perf_counter() - t0
    from up3d_b200.post.surface import _wall
    w = _wall(m.nodes, m.elements, wf)
    reps = 50
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(reps):
        w.run(phi, 1.0, 0.8, 1.4, 1.0, 2, want=("cp",))
    b.record()
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / reps
    t0 = time.perf_counter()
    wall_force_coefficients(m.nodes, m.elements, wf, phi, m_inf=0.8, smooth_passes=2)
    api_ms = (time.perf_counter() - t0) * 1e3
    # the same call with the mesh as device tensors: found by identity and
    # in-place version, no digest (the first call digests them once)
    nodes_d, elements_d = torch.from_numpy(m.nodes).cuda(), torch.from_numpy(m.elements).cuda()
    wall_force_coefficients(nodes_d, elements_d, wf, phi, m_inf=0.8, smooth_passes=2)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(10):
        wall_force_coefficients(nodes_d, elements_d, wf, phi, m_inf=0.8, smooth_passes=2)
    api_t_ms = (time.perf_counter() - t0) * 1e3 / 10
    t0 = time.perf_counter()
    ref = O.wall_force_coefficients(m.nodes, m.elements, wf, phi.cpu().numpy(), m_inf=0.8, smooth_passes=2)
    cpu_s = time.perf_counter() - t0
    return {"mesh": spec, "n_wall_triangles": int(len(wf)), "ms_per_evaluation": round(ms, 4),
            "ms_per_api_call": round(api_ms, 2), "ms_per_api_call_tensors": round(api_t_ms, 3),
            "api_note": "with writeable numpy arrays the call looks the mesh handle up by a digest of nodes "
                        "and elements; with tensors (or read-only arrays) seen before, by identity",
            "first_call_s": round(setup_s, 3), "cpu_oracle_s": round(cpu_s, 3),
            "cl": r["cl"], "max_abs_cf_diff_vs_oracle": float(np.abs(r["cf"] - ref["cf"]).max())}


def batched_timing(spec, seed=0):
    """Many cases in one launch: meshes of log-uniform size between the
    smallest and largest box, M_inf ~ U[mach_lo, mach_hi], bump amplitude ~
    U[0.02, 0.08], one seed.  Reports the residual+Jacobian throughput of
    one batched evaluation against the same cases evaluated one by one, and
    the time to converge every case (|R_free|inf < 1e-10) with the lockstep
    batched Newton against sequential plain solves."""
    import torch
    from up3d_b200.mesh.kuhn import bump_channel, seeded_state
    from up3d_b200.solve.batched import BatchedChannels, CaseSet, solve_newton_batched
    from up3d_b200.solve.fused import FlowParams
    from up3d_b200.solve.newton import ChannelWorkspace, solve_newton_transonic
    k_s, lo_s, hi_s, mlo_s, mhi_s = spec.split(":")
    K = int(k_s)
    lo = np.array([int(v) for v in lo_s.split("x")], dtype=float)
    hi = np.array([int(v) for v in hi_s.split("x")], dtype=float)
    rng = np.random.default_rng(seed)
    f = np.exp(rng.uniform(0.0, np.log(hi[0] / lo[0]), size=K))
    shapes = [tuple(int(round(v)) for v in lo * fi) for fi in f]
    machs_drawn = rng.uniform(float(mlo_s), float(mhi_s), size=K)
    amps = rng.uniform(0.02, 0.08, size=K)
    # a case above its bump's choking Mach has no steady solution: cap it
    # 0.02 below (mesh.kuhn.choking_mach)
    from up3d_b200.mesh.kuhn import choking_mach
    machs = np.minimum(machs_drawn, np.array([choking_mach(float(a)) - 0.02 for a in amps]))
    meshes = [bump_channel(*sh, amplitude=float(a), seed=c) for c, (sh, a) in enumerate(zip(shapes, amps))]
    # the ordering and launch shapes picked by the tuner (timed candidates)
    t_tune = time.perf_counter()
    batch = BatchedChannels.tuned(meshes, machs)
    t_tune = time.perf_counter() - t_tune
    shapes_tuned = batch.ws.ev.mesh.tuning()
    E = batch.n_tets
    # assembly throughput: seeded states
    states = [seeded_state(m, c) for c, m in enumerate(meshes)]
    phi = batch.union_phi(states)
    wss = [ChannelWorkspace(m.nodes, m.elements, m.dirichlet_nodes) for m in meshes]
    phis = [torch.from_numpy(p).cuda() for p in states]
    flows = [FlowParams(m_inf=float(M)) for M in machs]

    def t_events(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    ms_b = t_events(lambda: batch.evaluate(phi, machs, jacobian=True), 20)

    def seq():
        for c in range(K):
            wss[c].ev.evaluate(phis[c], flows[c], jacobian=True, keep_state=False)
    ms_s = t_events(seq, 10)
    out = {"cases": K, "shapes": ["x".join(map(str, sh)) for sh in shapes],
           "machs": [round(float(m), 4) for m in machs], "amplitudes": [round(float(a), 4) for a in amps],
           "machs_drawn": [round(float(m), 4) for m in machs_drawn],
           "mach_cap": "each case at most 0.02 below its bump's choking Mach (quasi-1-D sonic-throat estimate)",
           "total_tets": int(E),
           "tuning": {"ordering": batch.ordering, "tuner_s": round(t_tune, 3),
                      "candidates_ms": {k: round(v["ms"], 4) for k, v in batch.tuning_report["candidates"].items()},
                      "shapes": {k: (round(v, 2) if isinstance(v, float) else v) for k, v in shapes_tuned.items()}},
           "assembly": {"batched_ms": round(ms_b, 4), "sequential_ms": round(ms_s, 4),
                        "batched_melem_s": round(E / ms_b / 1e3, 1),
                        "sequential_melem_s": round(E / ms_s / 1e3, 1)}}
    # time to 1e-10: batched lockstep vs sequential plain solves (second run timed)
    def fresh():
        b = BatchedChannels(meshes, ordering=batch.ordering)
        b.ws.ev.mesh.set_tuning(shapes_tuned["elem_persistent"], shapes_tuned["elem_threads_per_sm"],
                                shapes_tuned["row_lanes"], shapes_tuned["row_plan8"], shapes_tuned["assembly"],
                                shapes_tuned["tile_elems"], shapes_tuned["tile_stretch"])
        if shapes_tuned["assembly"] == 1:
            b.ws.ev.mesh.tile_info()
        return b
    res_b = None
    empty_pool()
    for _ in range(2):
        with settled_gc():
            res_b = solve_newton_batched(fresh(), machs)
    with settled_gc():
        res_ng = solve_newton_batched(fresh(), machs, use_graphs=False)
    seq_s, seq_ok, seq_phi = [], [], []
    empty_pool()
    for c, m in enumerate(meshes):
        ws = None
        with settled_gc():
            ws = ChannelWorkspace(m.nodes, m.elements, m.dirichlet_nodes)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = solve_newton_transonic(ws, float(machs[c]), m_start=min(0.70, float(machs[c])))
            torch.cuda.synchronize()
            seq_s.append(time.perf_counter() - t0)
        seq_ok.append(bool(r["converged"]))
        seq_phi.append(r["phi"].cpu())
    out["newton"] = {"batched_s": round(res_b["time_s"], 4), "sequential_s": round(float(sum(seq_s)), 4),
                     "batched_without_graphs_s": round(res_ng["time_s"], 4),
                     "batched_phases_s": {k: round(v, 4) for k, v in res_b["timings"].items()},
                     "batched_without_graphs_phases_s": {k: round(v, 4) for k, v in res_ng["timings"].items()},
                     "batched_n_newton": [int(v) for v in res_b["n_newton"]],
                     "batched_n_gmres": int(res_b["n_gmres_total"]),
                     "speedup": round(float(sum(seq_s)) / res_b["time_s"], 3),
                     "batched_converged": [bool(v) for v in res_b["converged"]],
                     "sequential_converged": seq_ok,
                     "batched_case_s": [None if np.isnan(v) else round(float(v), 4)
                                        for v in res_b["converged_s"]],
                     "sequential_case_s": [round(v, 4) for v in seq_s]}
    # the mixed schedule: the small cases in one lockstep union, the large
    # ones alone (built before the clock, like the sequential workspaces)
    for below in (100_000, 300_000):
        cs = None
        empty_pool()
        cs = CaseSet(meshes, machs, batch_below=below)
        with settled_gc():
            res_cs = cs.solve()
        out["newton"][f"mixed_schedule_{below // 1000}k"] = {
            "batch_below_tets": below, "n_batched": res_cs["n_batched"], "n_plain": res_cs["n_plain"],
            "batched_tets": int(sum(meshes[c].n_tets for c in cs.small)),
            "time_s": round(res_cs["time_s"], 4),
            "batched_s": None if "batched_s" not in res_cs else round(res_cs["batched_s"], 4),
            "sequential_s_same_cases": {"batched": round(float(sum(seq_s[c] for c in cs.small)), 4),
                                        "plain": round(float(sum(seq_s[c] for c in cs.large)), 4)},
            "speedup_vs_sequential": round(float(sum(seq_s)) / res_cs["time_s"], 3),
            "converged": bool(res_cs["converged"].all()),
            "max_dphi_vs_sequential": float(max(float((res_cs["phi"][c].cpu() - seq_phi[c]).abs().max())
                                                for c in range(len(meshes))))}
        del cs
    return out


_ORACLE_OPS = {}


def oracle_ops(mesh):
    """The oracle's operators on the bench mesh (built once per process)."""
    from oracle import oracle as O
    key = id(mesh)
    if key not in _ORACLE_OPS:
        _ORACLE_OPS[key] = (O.PicardOperator(mesh.nodes, mesh.elements), O.UpwindOperator(mesh.nodes, mesh.elements))
    return _ORACLE_OPS[key]


def bench_parity(mesh, order, ev, flow, d_phis, phis, pocket: bool):
    """The timed states (and, when asked, the three supersonic-pocket
    families) evaluated once more outside the timed region and compared
    with the oracle's chain of the reference kernels: largest relative
    error of R, rho~ and the merged Newton Jacobian (over the union
    pattern), upstream mismatches, Term-3 counts."""
    from oracle import oracle as O
    from up3d_b200.mesh.kuhn import pocket_state
    op, upw = oracle_ops(mesh)
    states = [(f"seed{k}", phis[k], d_phis[k]) for k in range(len(phis))]
    if pocket:
        import torch
        for fam in ("accelerating", "shockpoint", "mixed"):
            ph = pocket_state(mesh, fam)
            states.append((fam, ph, torch.from_numpy(order.nodal(ph)).cuda()))
    t0 = time.perf_counter()
    worst = {"R": 0.0, "rho_tilde": 0.0, "J": 0.0}
    per = {}
    mism = 0
    for label, ph, pd in states:
        ev.evaluate(pd, flow, jacobian=True, keep_state=True)
        R = order.nodal_back(ev.R.cpu().numpy())
        rt = order.elemental_back(ev.rho_tilde.cpu().numpy())
        up = order.element_ids_back(order.elemental_back(ev.upstream.cpu().numpy()))
        n3 = int(ev.read_monitors()["n_term3_active"])
        J = ev.jacobian().to_scipy()
        if not order.identity:
            J = J[order.node_inv][:, order.node_inv]
        ref = O.chain(op, upw, ph, M_INF)
        eR = float(np.abs(R - ref["R"]).max() / np.abs(ref["R"]).max())
        ert = float(np.abs(rt - ref["rho_tilde"]).max() / np.abs(ref["rho_tilde"]).max())
        D = (J - ref["J"]).tocoo()
        eJ = float((np.abs(D.data).max() if D.nnz else 0.0) / np.abs(ref["J"].data).max())
        nm = int(np.count_nonzero(up != ref["upstream"]))
        mism += nm
        worst["R"] = max(worst["R"], eR)
        worst["rho_tilde"] = max(worst["rho_tilde"], ert)
        worst["J"] = max(worst["J"], eJ)
        per[label] = {"R": eR, "rho_tilde": ert, "J": eJ, "upstream_mismatch": nm,
                      "n_term3_active": n3, "oracle_n_term3_active": int(ref["n_term3_active"])}
    return {"max_rel_err": worst, "upstream_mismatch": mism, "tolerance": 1e-12,
            "ok": bool(max(worst.values()) < 1e-12 and mism == 0), "states": per,
            "reference": "oracle chain (C/OpenMP restatement of the reference kernels, pinned to "
                         "reference-generated fixtures)",
            "seconds": round(time.perf_counter() - t0, 1)}


def linear_timing(ev, dmesh, mesh, order, phi_d, flow):
    """The Krylov solve's kernels on the bench mesh's Newton Jacobian at the
    first timed state (Dirichlet inflow/outflow rows masked): FP64 and FP32
    SpMV against their compulsory bytes (12 Z + 4 (N+1) + 16 N and
    8 Z + 4 (N+1) + 8 N, plus the N-byte mask), the AMG V-cycle in FP64 and
    FP32, and one GMRES(60) restart cycle with the FP64 V-cycle as
    preconditioner (per Arnoldi step).  CUDA events, inputs resident."""
    import torch
    from up3d_b200 import _lib as L
    from up3d_b200.solve.linear import build_amg_preconditioner, solve_gmres, with_dirichlet
    ev.evaluate(phi_d, flow, jacobian=True, keep_state=False)
    J = ev.jacobian()
    N, Z = dmesh.n_nodes, int(J.data.numel())
    mask_h = np.zeros(N, dtype=np.uint8)
    mask_h[mesh.dirichlet_nodes] = 1
    mask = torch.from_numpy(order.nodal(mask_h)).cuda()
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.rand(N, dtype=torch.float64, device="cuda", generator=g)
    y = torch.empty_like(x)
    x32, y32, d32 = x.float(), torch.empty(N, dtype=torch.float32, device="cuda"), J.data.float()
    st = L.stream_ptr()

    def t_events(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    peak, _ = read_peaks()
    ms64 = t_events(lambda: L.call("up3d_spmv", N, J.indptr.data_ptr(), J.indices.data_ptr(), J.data.data_ptr(),
                                   x.data_ptr(), y.data_ptr(), mask.data_ptr(), st), 100)
    ms32 = t_events(lambda: L.call("up3d_spmv_f32", N, J.indptr.data_ptr(), J.indices.data_ptr(), d32.data_ptr(),
                                   x32.data_ptr(), y32.data_ptr(), mask.data_ptr(), st), 100)
    b64 = 12 * Z + 4 * (N + 1) + 16 * N + N
    b32 = 8 * Z + 4 * (N + 1) + 8 * N + N
    A = with_dirichlet(J, mask)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ml, M = build_amg_preconditioner(A, fp32="both")
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    z = torch.empty_like(x)
    z32 = torch.empty_like(x32)
    v64 = t_events(lambda: L.call("up3d_amg_vcycle", M.handle, x.data_ptr(), z.data_ptr(), st), 20)
    v32 = t_events(lambda: L.call("up3d_amg_vcycle_f32", M.handle, x32.data_ptr(), z32.data_ptr(), st), 20)
    b = x.clone()
    b[mask.bool()] = 0.0
    solve_gmres(A, b, M=M, rtol=1e-30, restart=60, maxiter=1, on_fail="return")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, n_inner, _ = solve_gmres(A, b, M=M, rtol=1e-30, restart=60, maxiter=1, on_fail="return")
    torch.cuda.synchronize()
    gm_s = time.perf_counter() - t0
    return {"matrix": f"Newton Jacobian of the bench mesh at the first timed state ({N} rows, {Z} entries)",
            "spmv_fp64": {"ms": round(ms64, 5), "bytes": b64, "gbs": round(b64 / (ms64 * 1e-3) / 1e9, 1),
                          "frac": round(b64 / (ms64 * 1e-3) / 1e9 / peak, 4)},
            "spmv_fp32": {"ms": round(ms32, 5), "bytes": b32, "gbs": round(b32 / (ms32 * 1e-3) / 1e9, 1),
                          "frac": round(b32 / (ms32 * 1e-3) / 1e9 / peak, 4)},
            "amg": {"setup_s": round(setup_s, 3), "levels": ml.level_rows,
                    "operator_complexity": round(ml.operator_complexity, 3),
                    "vcycle_fp64_ms": round(v64, 4), "vcycle_fp32_ms": round(v32, 4)},
            "gmres_fp64": {"restart": 60, "arnoldi_steps": int(n_inner),
                           "ms_per_arnoldi_step": round(1e3 * gm_s / max(n_inner, 1), 4),
                           "note": "one restart cycle, wall clock with the device synchronised"}}


def run_ours(args):
    import torch
    import torch.distributed as dist

    from up3d_b200.replicas import max_over_ranks
    from up3d_b200.replicas import world as world_env

    rank, world, local = world_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from up3d_b200 import _lib as L
    from up3d_b200.mesh.device import DeviceMesh
    from up3d_b200.solve.fused import FlowParams, ResidualJacobian

    shape = tuple(int(v) for v in args.mesh.split("x"))
    mesh, phis = workload(shape)
    from up3d_b200.mesh.order import renumber
    order = renumber(mesh.nodes, mesh.elements, args.order)
    dmesh = DeviceMesh(order.nodes, order.elements)
    phis_dev = [order.nodal(p) for p in phis]
    info = {"n_tets": dmesh.n_tets, "n_nodes": dmesh.n_nodes, "nnz": dmesh.nnz}
    ev = ResidualJacobian(dmesh)
    flow = FlowParams(m_inf=M_INF)
    d_phis = [torch.from_numpy(p).cuda() for p in phis_dev]
    stream = torch.cuda.current_stream()

    if args.tune == "auto":
        dmesh.autotune(d_phis[0], flow, reps=5)
    elif args.tune != "default":
        dmesh.set_tuning(*(int(v) for v in args.tune.split(",")))
    tuning = dmesh.tuning()
    tiled = tuning["assembly"] == 1
    if tiled:
        info["tiles"] = dmesh.tile_info()

    def step(k):
        ev.evaluate(d_phis[k % N_STATES], flow, jacobian=True, keep_state="upstream")

    for w in range(max(args.warmup, 3)):
        step(w)
    torch.cuda.synchronize()
    mon = ev.read_monitors()

    props = torch.cuda.get_device_properties(local)
    bus = None
    try:
        bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
    except Exception:
        bus = None

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- device-timed region
    with ClockSampler(bus) as clocks:
        L.profile(True)
        launches0 = L.launch_count()
        barrier()
        torch.cuda.synchronize()
        t_start = torch.cuda.Event(enable_timing=True)
        t_stop = torch.cuda.Event(enable_timing=True)
        t_start.record(stream)
        for k in range(args.steps):
            step(k)
        t_stop.record(stream)
        torch.cuda.synchronize()
        barrier()
        launches = L.launch_count() - launches0
        prof = L.profile_read()
        L.profile(False)
        ms = t_start.elapsed_time(t_stop)

        # ---- sustained: the same step for about two seconds (at least 200
        # steps), so that the clock record covers a long stretch of work
        n_sus = max(200, int(2000.0 / max(ms / max(args.steps, 1), 1e-3)))
        barrier()
        torch.cuda.synchronize()
        s_start = torch.cuda.Event(enable_timing=True)
        s_stop = torch.cuda.Event(enable_timing=True)
        s_start.record(stream)
        for k in range(n_sus):
            step(k)
        s_stop.record(stream)
        torch.cuda.synchronize()
        barrier()
        sus_ms = s_start.elapsed_time(s_stop)

        # ---- end-to-end through the public API with host buffers: every
        # step uploads its phi and downloads R and the Jacobian data; the
        # double-buffered pipeline overlaps one step's copies with the
        # neighbouring step's evaluation
        from up3d_b200.solve.fused import HostPipeline
        h_phis = [torch.from_numpy(p).pin_memory() for p in phis_dev]
        h_R = torch.empty(dmesh.n_nodes, dtype=torch.float64).pin_memory()
        h_J = torch.empty(dmesh.nnz, dtype=torch.float64).pin_memory()
        pipe = HostPipeline(ev)
        n_e2e = max(1, args.e2e_steps)
        for k in range(2):
            pipe.submit(h_phis[k % N_STATES], flow, h_R, h_J)
        pipe.finish()
        barrier()
        torch.cuda.synchronize()
        e_start = torch.cuda.Event(enable_timing=True)
        e_stop = torch.cuda.Event(enable_timing=True)
        e_start.record(stream)
        for k in range(n_e2e):
            pipe.submit(h_phis[k % N_STATES], flow, h_R, h_J)
        pipe.finish()
        e_stop.record(stream)
        torch.cuda.synchronize()
        barrier()
        e2e_ms = e_start.elapsed_time(e_stop)

    # ---- supersonic-pocket states (upwind branches and Term 3 active), the
    # same step timed the same way
    pocket = None
    if args.pocket_steps > 0:
        from up3d_b200.mesh.kuhn import pocket_state
        fams = ("accelerating", "shockpoint", "mixed")
        p_phis = [torch.from_numpy(order.nodal(pocket_state(mesh, f))).cuda() for f in fams]
        for k in range(3):
            ev.evaluate(p_phis[k], flow, jacobian=True, keep_state=False)
        p_mon = [None] * 3
        for k in range(3):
            ev.evaluate(p_phis[k], flow, jacobian=True, keep_state=False)
            p_mon[k] = ev.read_monitors()
        barrier()
        torch.cuda.synchronize()
        p_start = torch.cuda.Event(enable_timing=True)
        p_stop = torch.cuda.Event(enable_timing=True)
        p_start.record(stream)
        for k in range(args.pocket_steps):
            ev.evaluate(p_phis[k % 3], flow, jacobian=True, keep_state=False)
        p_stop.record(stream)
        torch.cuda.synchronize()
        barrier()
        p_ms = p_start.elapsed_time(p_stop)
        p_ms = max_over_ranks([p_ms], device="cuda")[0]
        # per-phase split of the pocket step (a separate, profiled pass)
        n_prof = min(args.pocket_steps, 30)
        L.profile(True)
        for k in range(n_prof):
            ev.evaluate(p_phis[k % 3], flow, jacobian=True, keep_state=False)
        torch.cuda.synchronize()
        p_prof = L.profile_read()
        L.profile(False)
        # one pocket state repeated (the frozen finish and late Newton steps
        # keep the active set and upstream map): Term 3 from the recorded
        # pattern, values only
        hits0 = dmesh.term3_cache_hits()
        for _ in range(3):
            ev.evaluate(p_phis[2], flow, jacobian=True, keep_state="upstream")
        n_rep = max(1, min(args.pocket_steps, 100))
        torch.cuda.synchronize()
        L.profile(True)
        r_start = torch.cuda.Event(enable_timing=True)
        r_stop = torch.cuda.Event(enable_timing=True)
        r_start.record(stream)
        for _ in range(n_rep):
            ev.evaluate(p_phis[2], flow, jacobian=True, keep_state="upstream")
        r_stop.record(stream)
        torch.cuda.synchronize()
        r_prof = L.profile_read()
        L.profile(False)
        r_ms = r_start.elapsed_time(r_stop)
        repeat = {"family": fams[2], "steps": n_rep, "ms_per_step": round(r_ms / n_rep, 5),
                  "term3_cache_hits": dmesh.term3_cache_hits() - hits0,
                  "phases_ms_per_step": {k: round(v["ms"] / n_rep, 5) for k, v in r_prof.items() if v["calls"]},
                  "note": "profiled pass (per-phase events); the same pocket state every step"}
        pocket = {"families": list(fams), "steps": args.pocket_steps, "repeated_state": repeat,
                  "value": round(dmesh.n_tets * args.pocket_steps * world / (p_ms * 1e-3) / 1e6, 3),
                  "unit": "Melem/s", "ms_per_step": round(p_ms / args.pocket_steps, 5),
                  "n_supersonic": [int(m["n_supersonic"]) for m in p_mon],
                  "n_term3_active": [int(m["n_term3_active"]) for m in p_mon],
                  "phases_ms_per_step": {k: round(v["ms"] / n_prof, 5) for k, v in p_prof.items() if v["calls"]},
                  "n_term3_extra": [int(m["n_term3_extra"]) for m in p_mon],
                  "nu_max": [float(m["nu_max"]) for m in p_mon]}

    # the solver-level timings run on one GPU only: a scaling run (N > 1)
    # measures the replicated step alone
    solo = world == 1
    newton = newton_timing(args.newton) if args.newton and solo else None
    c4 = newton_timing(args.c4, reps=1) if args.c4 and solo else None
    adjoint = adjoint_timing(args.adjoint) if args.adjoint and solo else None
    batched = batched_timing(args.batched) if args.batched and solo else None
    weighted = weighted_timing(args.weighted) if args.weighted and solo else None
    wake = wake_timing(args.wake) if args.wake and solo else None
    wall = wall_timing(args.wall) if args.wall and solo else None
    lifting = lifting_timing(args.lifting) if args.lifting and solo else None
    naca = naca_timing() if args.naca and solo else None

    parity = bench_parity(mesh, order, ev, flow, d_phis, phis, args.parity >= 2) if args.parity and solo else None
    linear = linear_timing(ev, dmesh, mesh, order, d_phis[0], flow) if args.linear and solo else None

    ms, e2e_ms, sus_ms = max_over_ranks([ms, e2e_ms, sus_ms], device="cuda")
    value = dmesh.n_tets * args.steps * world / (ms * 1e-3) / 1e6
    e2e_value = dmesh.n_tets * n_e2e * world / (e2e_ms * 1e-3) / 1e6

    # roofline of the dominant kernel, timed live over the timed region
    bm = bytes_model(info, n_active=int(mon["n_term3_active"]))
    peak, peak_kind = read_peaks()
    if tiled:
        # the tile kernel does both passes' work (every element, every
        # output of the tile); the combine adds the partials of outputs
        # shared by tiles: the pair is timed and credited together
        dom = "tile_eval+combine"
        calls = max(prof["elem_sweep"]["calls"], 1)
        per_launch_ms = (prof["elem_sweep"]["ms"] + prof["row_gather"]["ms"]) / calls
        dom_bytes = bm["elem_sweep"] + bm["row_gather"]
        design_bytes = bm["design"]["tile_eval"]
        traffic = read_traffic("tile_eval", dmesh.n_tets)
    else:
        dom = max(("elem_sweep", "row_gather"), key=lambda s: prof[s]["ms"])
        per_launch_ms = prof[dom]["ms"] / max(prof[dom]["calls"], 1)
        dom_bytes = bm[dom]
        design_bytes = bm["design"][dom]
        traffic = read_traffic(dom, dmesh.n_tets)
    achieved = dom_bytes / (per_launch_ms * 1e-3) / 1e9
    step_bytes = bm["fused"]
    phase_names = {"elem_sweep": "tile_eval", "row_gather": "combine"} if tiled else {}

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline and args.cpu_states > 0:
            threads = os.cpu_count() or 1
            v, dt, used = cpu_chain_timing(mesh, phis, args.cpu_states, threads)
            cpu = {"value": round(v, 4), "unit": "Melem/s", "cores": used, "kind": "port",
                   "sample": f"{args.cpu_states} full-mesh residual+Jacobian chains of the oracle "
                             f"(C/OpenMP restatement of the reference kernels), {dt:.1f} s",
                   "port_vs_reference_numba": PORT_VS_NUMBA}
        line = {
            "metric": "residual+Jacobian Melem/s", "value": round(value, 3), "unit": "Melem/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3),
            "ms_per_step": round(ms / args.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(shape, mesh),
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1),
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / peak, 4),
                         "traffic": traffic,
                         "algorithmic_bytes": dom_bytes,
                         "design_bytes": design_bytes,
                         "ms_per_launch": round(per_launch_ms, 5)},
            "step_roofline": {"algorithmic_bytes": step_bytes,
                              "achieved_gbs": round(step_bytes / (ms / args.steps * 1e-3) / 1e9, 1),
                              "frac": round(step_bytes / (ms / args.steps * 1e-3) / 1e9 / peak, 4),
                              "phases_ms_per_step": {phase_names.get(k, k): round(v["ms"] / max(args.steps, 1), 5)
                                                     for k, v in prof.items() if v["calls"]}},
            "sustained": {"steps": n_sus, "ms_per_step": round(sus_ms / n_sus, 5),
                          "value": round(dmesh.n_tets * n_sus * world / (sus_ms * 1e-3) / 1e6, 3),
                          "unit": "Melem/s",
                          "note": "the timed step repeated for ~2 s right after the timed region, "
                                  "inside the clock record"},
            "assembly": "tiled" if tiled else "two-pass",
            "tiles": info.get("tiles"),
            "parity": parity,
            "linear": linear,
            "cpu_baseline": cpu,
            "e2e": {"value": round(e2e_value, 3), "unit": "Melem/s",
                    "h2d_bytes_per_step": 8 * dmesh.n_nodes,
                    "d2h_bytes_per_step": 8 * dmesh.n_nodes + 8 * dmesh.nnz},
            "gpu_launches": int(launches),
            "tuning": {k: (round(v, 2) if isinstance(v, float) else v) for k, v in tuning.items()},
            "mesh_order": args.order,
            "clocks": clocks.summary(),
            "monitors": {k: (float(v) if isinstance(v, float) else int(v)) for k, v in mon.items()},
            "pocket_states": pocket,
            "newton": newton,
            "newton_large": c4,
            "adjoint": adjoint,
            "batched": batched,
            "weighted_upwind": weighted,
            "wake_elimination": wake,
            "wall_forces": wall,
            "lifting_newton": lifting,
            "naca0012": naca,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
