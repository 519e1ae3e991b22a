#!/usr/bin/env python
"""Benchmark: batched BEM solves/s at N=2048 panels on B200.

Workload (one "step" = one pass of the hot path over one batch): a
hemisphere of radius 1 m meshed with 32 x 64 panels (2048), 64 frequencies
omega = linspace(0.3, 3.0), heave and surge radiating/influenced, one
incident heading (beta = 0), Rankine + reflected Rankine + tabulated
Guevel-Delhommeau wave term, direct formulation; mixed precision (FP32 LU,
FP64 refinement to max|r|/max|b| <= 1e-10).  A solve is one (mesh,
frequency) problem with all its right-hand sides and outputs (A, B, F, FK).

  value  solves/s with the mesh already resident on the device
  e2e    the same through the C ABI from pinned host buffers: mesh upload,
         batch call, outputs back to the host, every step
  grads  adjoint grads/s: one grad = one (mesh, frequency) problem solved
         forward, its adjoint solve and the tangent contraction, giving the
         cotangents of every mesh field and of omega for a scalar objective
         J = sum(wA A) + sum(wB B) + Re sum(conj(wF) F) (seeded weights), and
         from them dJ/dR through the exact mesh tangent; mixed path, with
         the FP64 GPU path and the gradient agreement beside it

Also reported: the plain FP64 GPU path (cuSOLVER zgetrf) on a frequency
subsample, the relative error of the mixed outputs against it, per-phase
times measured with CUDA events on the library's stream, clocks sampled
during the timed region, and the CPU oracle baseline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import ctypes
import datetime
import importlib.util
import json
import os
import pathlib
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
METRIC = "BEM solves/s + adjoint grads/s, N=2048 panels: mixed vs FP64 GPU at 1e-6 err"
WORKLOAD = "hemisphere_2048p_64omega_heave_surge_diffraction_delhommeau_direct"


def load_package():
    name = "marinehydro_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg_dir = ROOT / "marinehydro.jl_b200"
    spec = importlib.util.spec_from_file_location(
        name, pkg_dir / "__init__.py", submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def workload(mh, res, n_omega):
    mesh = mh.mesh_hemisphere(1.0, (0.0, 0.0, 0.0), tuple(res))
    body = mh.FloatingBody.rigid(mesh, ["Heave", "Surge"])
    dofs = list(body.dofs.values())
    omegas = np.linspace(0.3, 3.0, n_omega)
    betas = [0.0]
    gfs = (mh.Rankine(), mh.RankineReflected(), mh.ExactGuevelDelhommeau())
    return mesh, dofs, omegas, betas, gfs


def config_dict(mesh, omegas, args):
    return {"workload": WORKLOAD, "panels": int(mesh.nfaces), "resolution": list(args.res),
            "n_omega": int(len(omegas)), "omega_range": [float(omegas[0]), float(omegas[-1])],
            "dofs": ["Heave", "Surge"], "headings": [0.0],
            "green_functions": "Rankine+RankineReflected+ExactGuevelDelhommeau(table)",
            "formulation": "direct",
            "precision": ("mixed: FP16 tcgen05 trailing update / FP32 LU, FP64 refinement"
                          if args.lu == "tcgen05" else "mixed: FP32 LU, FP64 refinement"),
            "lu_backend": args.lu,
            "tol": args.tol, "solve": "one (mesh, omega) problem, 3 right-hand sides",
            "l2": "working set ~11 GB per step, larger than the 126 MB L2 (no flush needed)"}


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------

class ClockSampler:
    """SM clock and clock-event reasons of the bench's GPU while the timed
    region runs.  Read-only NVML queries from a background thread every
    5 ms (the library calls release the GIL), so a timed region of tens of
    milliseconds still gets a few dozen samples; without NVML, nvidia-smi
    polls every 50 ms into a temporary file.  Nothing is changed on the GPU."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: str, device: int = 0):
        import threading

        self.sm, self.mx, self.reasons = [], None, set()
        self.proc = self.thread = None
        self.stop_flag = threading.Event()
        try:
            import pynvml as nv
            import torch

            nv.nvmlInit()
            prop = torch.cuda.get_device_properties(device)
            bus = f"{prop.pci_domain_id:08x}:{prop.pci_bus_id:02x}:{prop.pci_device_id:02x}.0"
            try:
                h = nv.nvmlDeviceGetHandleByPciBusId(bus.encode())
            except nv.NVMLError:
                h = nv.nvmlDeviceGetHandleByIndex(int(gpu_index))
            self.mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            bits = [(name, getattr(nv, attr)) for name, attr in self.REASONS]

            def run():
                while not self.stop_flag.is_set():
                    try:
                        self.sm.append(float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)))
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.reasons.update(name for name, bit in bits if r & bit)
                    except nv.NVMLError:
                        return
                    self.stop_flag.wait(0.005)

            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            return
        except Exception:  # noqa: BLE001 - no NVML: fall back to nvidia-smi
            self.thread = None
        try:
            import tempfile

            self.fh = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-i", gpu_index], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.thread is not None:
            self.stop_flag.set()
            self.thread.join(timeout=5)
        elif self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.fh.flush()
            self.fh.seek(0)
            names = [nm for nm, _ in self.REASONS]
            for r in (x.split(",") for x in self.fh.read().splitlines() if x.strip()):
                r = [x.strip() for x in r]
                if len(r) < 9:
                    continue
                try:
                    self.sm.append(float(r[1]))
                    self.mx = float(r[2])
                except ValueError:
                    continue
                self.reasons.update(nm for nm, v in zip(names, r[5:9]) if v.lower().startswith("active"))
            self.fh.close()
            os.unlink(self.fh.name)
        else:
            return None
        if not self.sm:
            return None
        return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": self.mx, "reasons": sorted(self.reasons),
                "samples": len(self.sm), "source": "nvml" if self.thread is not None else "nvidia-smi"}


# --------------------------------------------------------------------------
# CPU baseline (the FP64 CPU oracle; test infrastructure, timed as the baseline)
# --------------------------------------------------------------------------

def cpu_baseline(mh, mesh, dofs, omegas, betas, columns: int):
    sys.path.insert(0, str(ROOT))
    import oracle
    import scipy.linalg as sla

    oracle.lib()
    n = mesh.nfaces
    w = float(omegas[len(omegas) // 2])
    k = w * w / 9.81
    mask = oracle.GF_RANKINE | oracle.GF_RANKINE_REFLECTED | oracle.GF_DELHOMMEAU
    t0 = time.perf_counter()
    S, D = oracle.assemble(mesh, k, mask, True, columns=(0, columns))
    t_asm = (time.perf_counter() - t0) * n / columns
    # LU and solves on a full FP64 matrix of the same size (Wu assembly is cheap)
    S, D = oracle.assemble(mesh, k, oracle.GF_RANKINE | oracle.GF_RANKINE_REFLECTED | oracle.GF_WU,
                           True)
    t0 = time.perf_counter()
    lu = sla.lu_factor(D, check_finite=False)
    bcs = [oracle.radiation_bc(mesh.normals, d, w) for d in dofs]
    bcs += [oracle.airy_bc(mesh.centers, mesh.normals, w, b) for b in betas]
    phi = sla.lu_solve(lu, S @ np.stack(bcs, axis=1), check_finite=False)
    for q in range(phi.shape[1]):
        for d in dofs:
            oracle.integrate_pressure(mesh.normals, mesh.areas, 1j * 1000.0 * w * phi[:, q], d)
    t_lu = time.perf_counter() - t0
    per_solve = t_asm + t_lu
    return {"value": 1.0 / per_solve, "unit": "solves/s", "cores": oracle.max_threads(),
            "kind": "port",
            "sample": (f"1 frequency (omega={w:.3f}): exact-quadrature Delhommeau assembly of "
                       f"{columns} of {n} columns scaled x{n / columns:g} ({t_asm:.2f} s), plus "
                       f"LAPACK zgetrf/zgetrs + 3 right-hand sides + forces ({t_lu:.3f} s)")}


# --------------------------------------------------------------------------
# reference arm: the CPU implementation of the path (oracle port)
# --------------------------------------------------------------------------

def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    mh = load_package()
    mesh, dofs, omegas, betas, gfs = workload(mh, args.res, args.n_omega)
    times = []
    base = None
    for step in range(args.warmup + args.steps):
        base = cpu_baseline(mh, mesh, dofs, omegas, betas, args.cpu_columns)
        if step >= args.warmup:
            times.append(1.0 / base["value"])
    per = float(np.mean(times))
    v = 1.0 / per
    line = {"metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_dict(mesh, omegas, args), "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": base["cores"],
                             "kind": "port", "sample": base["sample"]},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------------------
# our arm
# --------------------------------------------------------------------------

def _pinned(a: np.ndarray, torch):
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t


def e2e_step(mh, ctx, host, omegas_p, dofs_p, betas_p, out_p, args, mask, info):
    """Mesh upload + batch + outputs to host through the C ABI."""
    N = mh.native
    L = N.lib()
    h = N._P()
    dp = lambda t: ctypes.cast(t.data_ptr(), N._D)
    N.check(L.mh_mesh_create(ctx.handle, host["n"], host["nv"], dp(host["vertices"]),
                             ctypes.cast(host["faces"].data_ptr(), N._I64), dp(host["centers"]),
                             dp(host["normals"]), dp(host["areas"]), dp(host["radii"]),
                             ctypes.byref(h)), ctx.handle)
    try:
        N.check(L.mh_hydro_batch(ctx.handle, h, omegas_p.numel(), dp(omegas_p), args.n_dof,
                                 dp(dofs_p), betas_p.numel(), dp(betas_p), 1000.0, 9.81, mask, 1,
                                 N.MH_PRECISION_MIXED, args.tol, args.max_iter, dp(out_p[0]),
                                 dp(out_p[1]), dp(out_p[2]), dp(out_p[3]), ctypes.byref(info)),
                ctx.handle)
    finally:
        L.mh_mesh_destroy(ctx.handle, h)


def e2e_grad_step(mh, ctx, host, omegas_p, dofs_p, betas_p, bars_p, grads_p, args, mask, info):
    """Mesh upload + forward/adjoint batch + cotangents to host through the C ABI."""
    N = mh.native
    L = N.lib()
    h = N._P()
    dp = lambda t: ctypes.cast(t.data_ptr(), N._D) if t is not None else None
    N.check(L.mh_mesh_create(ctx.handle, host["n"], host["nv"], dp(host["vertices"]),
                             ctypes.cast(host["faces"].data_ptr(), N._I64), dp(host["centers"]),
                             dp(host["normals"]), dp(host["areas"]), dp(host["radii"]),
                             ctypes.byref(h)), ctx.handle)
    try:
        N.check(L.mh_hydro_batch_vjp(
            ctx.handle, h, omegas_p.numel(), dp(omegas_p), args.n_dof, dp(dofs_p), betas_p.numel(),
            dp(betas_p), 1000.0, 9.81, mask, 1, N.MH_PRECISION_MIXED, args.tol, args.max_iter,
            dp(bars_p[0]), dp(bars_p[1]), dp(bars_p[2]), None, None, None, None, None,
            dp(grads_p[0]), dp(grads_p[1]), dp(grads_p[2]), dp(grads_p[3]), None, dp(grads_p[4]),
            None, ctypes.byref(info)), ctx.handle)
    finally:
        L.mh_mesh_destroy(ctx.handle, h)


def grad_weights(nd, nw, nb):
    rng = np.random.default_rng(2024)
    return (rng.normal(size=(nd, nd, nw)), rng.normal(size=(nd, nd, nw)),
            rng.normal(size=(nd, nw, nb)) + 1j * rng.normal(size=(nd, nw, nb)))


def run_grads(mh, ctx, mesh, dofs, omegas, betas, gfs, args, stream, barrier, dist, world, torch):
    """Adjoint grads/s (mixed) with the FP64 GPU path and the agreement of
    the two; each step one mh_hydro_batch_vjp over all frequencies."""
    nd, nw, nb = len(dofs), len(omegas), len(betas)
    wA, wB, wF = grad_weights(nd, nw, nb)
    tan = mh.hemisphere_tangents(1.0, (0.0, 0.0, 0.0), tuple(args.res))["radius"]

    def gstep():
        r = mh.hydro_batch_vjp(mesh, omegas, dofs, betas, wA, wB, wF, None, green_functions=gfs,
                               precision="mixed", tol=args.tol, max_iter=args.max_iter, ctx=ctx)
        return r, r.mesh.dot(tan)

    for _ in range(args.warmup):
        r, dR = gstep()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ctx.set_profiling(True)
    l0 = ctx.kernel_launches()
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        r, dR = gstep()
    ev1.record(stream)
    barrier()
    launches = ctx.kernel_launches() - l0
    phases = ctx.phase_times()
    ctx.set_profiling(False)
    ms = ev0.elapsed_time(ev1)
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    out = {"value": world * nw * args.steps / (ms / 1e3), "unit": "grads/s",
           "ms_per_step": ms / args.steps, "gpu_launches": launches,
           "objective": "J = sum(wA A) + sum(wB B) + Re sum(conj(wF) Fd), seeded weights",
           "outputs": "cotangents of vertices, centers, normals, areas, radii, omegas; dJ/dR",
           "dJ_dR": dR, "phases_ms_per_step": {k: v[0] / args.steps for k, v in phases.items() if v[1]}}
    # e2e through the C ABI
    host = host_mesh(mesh, torch)
    omegas_p = _pinned(omegas, torch)
    betas_p = _pinned(np.asarray(betas, dtype=np.float64), torch)
    dofs_p = _pinned(np.concatenate([np.asfortranarray(d).reshape(-1, order="F") for d in dofs]), torch)
    bars_p = [_pinned(np.asfortranarray(wA).reshape(-1, order="F"), torch),
              _pinned(np.asfortranarray(wB).reshape(-1, order="F"), torch),
              _pinned(np.asfortranarray(wF).reshape(-1, order="F").view(np.float64), torch)]
    grads_p = [torch.zeros(3 * mesh.nvertices, dtype=torch.float64).pin_memory(),
               torch.zeros(3 * mesh.nfaces, dtype=torch.float64).pin_memory(),
               torch.zeros(3 * mesh.nfaces, dtype=torch.float64).pin_memory(),
               torch.zeros(mesh.nfaces, dtype=torch.float64).pin_memory(),
               torch.zeros(nw, dtype=torch.float64).pin_memory()]
    cinfo = mh.bodies._Info()
    mask = mh.gf_mask(gfs)
    e2e_grad_step(mh, ctx, host, omegas_p, dofs_p, betas_p, bars_p, grads_p, args, mask, cinfo)
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        e2e_grad_step(mh, ctx, host, omegas_p, dofs_p, betas_p, bars_p, grads_p, args, mask, cinfo)
    ev1.record(stream)
    barrier()
    ms_e2e = ev0.elapsed_time(ev1)
    if dist is not None:
        t = torch.tensor([ms_e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    h2d = sum(int(v.numel() * v.element_size()) for k, v in host.items() if k not in ("n", "nv"))
    h2d += int(omegas_p.numel() * 8 + betas_p.numel() * 8 + dofs_p.numel() * 8)
    h2d += sum(int(t.numel() * t.element_size()) for t in bars_p)
    out["e2e"] = {"value": world * nw * args.steps / (ms_e2e / 1e3), "unit": "grads/s",
                  "h2d_bytes_per_step": h2d,
                  "d2h_bytes_per_step": sum(int(t.numel() * t.element_size()) for t in grads_p),
                  "ms_per_step": ms_e2e / args.steps}
    if args.no_fp64:
        return out
    # FP64 GPU path: per-call cost a + b * n_omega fitted on two subsample sizes
    sub = np.arange(0, nw, max(1, nw // args.fp64_omegas))[:args.fp64_omegas]
    mh.hydro_batch_vjp(mesh, omegas[sub[:1]], dofs, betas, wA[:, :, sub[:1]], wB[:, :, sub[:1]],
                       wF[:, sub[:1]], None, green_functions=gfs, precision="fp64", ctx=ctx)  # warm-up
    times = {}
    res64 = resmx = None
    for cnt in (2, len(sub)):
        s_ = sub[:cnt]
        call = lambda prec: mh.hydro_batch_vjp(mesh, omegas[s_], dofs, betas, wA[:, :, s_], wB[:, :, s_],
                                               wF[:, s_], None, green_functions=gfs, precision=prec,
                                               tol=args.tol, max_iter=args.max_iter, ctx=ctx)
        torch.cuda.synchronize()
        ev0.record(stream)
        r64 = call("fp64")
        ev1.record(stream)
        torch.cuda.synchronize()
        times[cnt] = ev0.elapsed_time(ev1)
        if cnt == len(sub):
            res64, resmx = r64, call("mixed")
    b = (times[len(sub)] - times[2]) / (len(sub) - 2)
    a = times[2] - 2 * b
    per = (a + nw * b) / nw
    out["fp64_gpu"] = {"value": 1e3 / per, "unit": "grads/s", "ms_per_grad_at_n_omega": per,
                       "fit_ms": {"per_call": a, "per_omega": b}, "omegas_timed": [2, int(len(sub))]}
    out["speedup_vs_fp64_gpu"] = out["value"] / out["fp64_gpu"]["value"]
    acc = {}
    for f in ("vertices", "centers", "normals", "areas"):
        x, y = getattr(resmx.mesh, f), getattr(res64.mesh, f)
        acc[f] = float(np.max(np.abs(x - y)) / np.max(np.abs(y)))
    acc["omegas"] = float(np.max(np.abs(resmx.omegas - res64.omegas)) / np.max(np.abs(res64.omegas)))
    acc["dJ_dR"] = abs(resmx.mesh.dot(tan) - res64.mesh.dot(tan)) / abs(res64.mesh.dot(tan))
    acc["note"] = "max abs difference / max abs value, mixed vs FP64 GPU gradients, same frequencies"
    out["accuracy"] = acc
    return out


def host_mesh(mesh, torch):
    return {"n": mesh.nfaces, "nv": mesh.nvertices,
            "vertices": _pinned(np.asfortranarray(mesh.vertices).reshape(-1, order="F"), torch),
            "faces": _pinned(np.asfortranarray(mesh.faces).reshape(-1, order="F"), torch),
            "centers": _pinned(np.asfortranarray(mesh.centers).reshape(-1, order="F"), torch),
            "normals": _pinned(np.asfortranarray(mesh.normals).reshape(-1, order="F"), torch),
            "areas": _pinned(mesh.areas, torch), "radii": _pinned(mesh.radii, torch)}


def run_ours(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    mh = load_package()
    ctx = mh.Context(local)
    ctx.set_lu_backend(args.lu)
    stream = torch.cuda.ExternalStream(ctx.stream())
    mesh, dofs, omegas, betas, gfs = workload(mh, args.res, args.n_omega)
    mask = mh.gf_mask(gfs)
    args.n_dof = len(dofs)
    dm = mh.device_mesh(mesh, ctx)

    def step():
        return mh.hydro_batch(mesh, omegas, dofs, betas, green_functions=gfs, precision="mixed",
                              tol=args.tol, max_iter=args.max_iter, ctx=ctx)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        out = step()
    # ---- timed region (resident inputs) ----
    vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
    gpu_index = vis.split(",")[local] if vis and vis.split(",")[local].strip().isdigit() else str(local)
    sampler = ClockSampler(gpu_index, local)
    ctx.set_profiling(True)
    launches0 = ctx.kernel_launches()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        out = step()
    ev1.record(stream)
    barrier()
    launches = ctx.kernel_launches() - launches0
    phases = ctx.phase_times()
    ctx.set_profiling(False)
    clocks = sampler.stop()
    ms = ev0.elapsed_time(ev1)
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    value = world * args.n_omega * args.steps / (ms / 1e3)
    A, B, Fd, Fk, info = out

    # ---- e2e through the C ABI from pinned host buffers ----
    host = host_mesh(mesh, torch)
    omegas_p = _pinned(omegas, torch)
    betas_p = _pinned(np.asarray(betas, dtype=np.float64), torch)
    dofs_p = _pinned(np.concatenate([np.asfortranarray(d).reshape(-1, order="F") for d in dofs]),
                     torch)
    nd, nw, nb = len(dofs), len(omegas), len(betas)
    out_p = [torch.zeros(nd * nd * nw, dtype=torch.float64).pin_memory(),
             torch.zeros(nd * nd * nw, dtype=torch.float64).pin_memory(),
             torch.zeros(2 * nd * nw * nb, dtype=torch.float64).pin_memory(),
             torch.zeros(2 * nd * nw * nb, dtype=torch.float64).pin_memory()]
    cinfo = mh.bodies._Info()
    e2e_step(mh, ctx, host, omegas_p, dofs_p, betas_p, out_p, args, mask, cinfo)
    barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        e2e_step(mh, ctx, host, omegas_p, dofs_p, betas_p, out_p, args, mask, cinfo)
    ev1.record(stream)
    barrier()
    ms_e2e = ev0.elapsed_time(ev1)
    if dist is not None:
        t = torch.tensor([ms_e2e], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_e2e = float(t.item())
    h2d = sum(int(v.numel() * v.element_size()) for k, v in host.items() if k not in ("n", "nv"))
    h2d += int(omegas_p.numel() * 8 * 2 + betas_p.numel() * 8 + dofs_p.numel() * 8)
    d2h = sum(int(t.numel() * t.element_size()) for t in out_p)
    e2e = {"value": world * args.n_omega * args.steps / (ms_e2e / 1e3), "unit": "solves/s",
           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
           "ms_per_step": ms_e2e / args.steps}

    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": ("f64+f32+f16 (FP64 matrices and residuals, FP32 LU panels, FP16 tensor-core "
                      "updates)" if args.lu == "tcgen05" else "f64+f32"), "data": "synthetic",
            "config": config_dict(mesh, omegas, args), "e2e": e2e, "gpu_launches": launches,
            "refinement": {"iterations": info.refine_iterations, "fallbacks": info.n_fallback,
                           "max_rel_residual": info.max_rel_residual}}
    if clocks:
        line["clocks"] = clocks
    per_phase = {k: v[0] / args.steps for k, v in phases.items() if v[1]}
    line["phases_ms_per_step"] = per_phase
    line["roofline"] = roofline(per_phase, mesh.nfaces, args)

    if not args.no_grads:
        line["grads"] = run_grads(mh, ctx, mesh, dofs, omegas, betas, gfs, args, stream, barrier, dist,
                                  world, torch)
    if rank == 0 and not args.no_fp64:
        line["fp64_gpu"], line["accuracy"] = fp64_baseline(mh, ctx, mesh, dofs, omegas, betas, gfs,
                                                           (A, B, Fd), args)
        if line["fp64_gpu"]["table"]["value"] > 0:
            line["speedup_vs_fp64_gpu"] = value / line["fp64_gpu"]["table"]["value"]
    if rank == 0 and not args.no_cpu:
        line["cpu_baseline"] = cpu_baseline(mh, mesh, dofs, omegas, betas, args.cpu_columns)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    ctx.close()
    return 0


def _peaks():
    try:
        peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return peaks, "measured"
    except (OSError, ValueError):
        return {}, "fallback"


# DRAM bytes (read + write) per pair-frequency of k_wave_delh_allw from an
# ncu capture (hemisphere 1024 panels, 64 frequencies, the solve step's
# launch without tape: (dram__bytes_read.sum + dram__bytes_write.sum) /
# (n^2 * 64)); traffic grows with the pairs and frequencies a launch
# processes, so it is scaled by them.
WAVE_DRAM_BYTES_PER_PAIR_FREQ = 39.4


def roofline(per_phase, n, args):
    """Dominant kernel of the solve step: the frequency-batched wave pass
    k_wave_delh_allw (one launch per step, timed alone by its phase events).
    Algorithmic bytes per launch: the FP64 Rankine parts of S and D read once
    per pair (16 B), S and D written in FP64 complex and the FP32 LU copy of D
    per pair and frequency (40 B).  The LU phase is given beside it against
    the dense tensor peak, (8/3) n^3 real flops per matrix."""
    peaks, src = _peaks()
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    tensor = float(peaks.get("bf16_tflops", 1590.0))
    if "wave" not in per_phase:
        return None
    ms = per_phase["wave"]
    nn = float(n) * n
    alg = nn * (16.0 + 40.0 * args.n_omega)
    achieved = alg / (ms / 1e3) / 1e9
    traffic = None
    if WAVE_DRAM_BYTES_PER_PAIR_FREQ is not None:
        traffic = WAVE_DRAM_BYTES_PER_PAIR_FREQ * nn * args.n_omega
    out = {"kernel": "k_wave_delh_allw", "bound": "hbm", "achieved": achieved, "peak": hbm,
           "unit": "GB/s", "frac": achieved / hbm, "peak_source": src, "traffic": traffic,
           "ms_per_launch": ms, "algorithmic_bytes_per_launch": alg,
           "note": ("FP64-issue bound (alpha contraction of the polar table per pair, Horner series "
                    "in R and complex arithmetic per pair and frequency; ncu at 1024 panels x 64 "
                    "frequencies: FP64 pipe 64% active at 15% warps active, no spills); the HBM "
                    "fraction shows the writes are not the limit")}
    if "lu" in per_phase:
        fl = 8.0 / 3.0 * float(n) ** 3 * args.n_omega
        ach = fl / (per_phase["lu"] / 1e3) / 1e12
        out["lu"] = {"kernels": "k_lu_diag64 + k_lu_trsm_tc + k_lu_update_tc", "bound": "tensor",
                     "achieved": ach, "peak": tensor, "unit": "TFLOP/s", "frac": ach / tensor,
                     "ms_per_step": per_phase["lu"], "algorithmic_flops_per_step": fl}
    return out


def fp64_baseline(mh, ctx, mesh, dofs, omegas, betas, gfs, mixed, args):
    """Plain FP64 GPU path on a frequency subsample: FP64 assembly (table and
    exact quadrature), cuSOLVER zgetrf/zgetrs, one frequency at a time; timed
    with CUDA events on the library's stream."""
    import torch

    stream = torch.cuda.ExternalStream(ctx.stream())
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    sub = np.arange(0, len(omegas), max(1, len(omegas) // args.fp64_omegas))[:args.fp64_omegas]
    res = {}
    out64 = None
    for method in ("table", "exact"):
        ctx.set_delhommeau_method(method)
        om = omegas[sub] if method == "table" else omegas[sub[:2]]
        mh.hydro_batch(mesh, om[:1], dofs, betas, green_functions=gfs, precision="fp64", ctx=ctx)
        torch.cuda.synchronize()
        ev0.record(stream)
        o = mh.hydro_batch(mesh, om, dofs, betas, green_functions=gfs, precision="fp64", ctx=ctx)
        ev1.record(stream)
        torch.cuda.synchronize()
        dt = ev0.elapsed_time(ev1) / 1e3
        res[method] = {"value": len(om) / dt, "unit": "solves/s", "omegas": int(len(om)),
                       "ms_per_solve": dt / len(om) * 1e3}
        if method == "table":
            out64 = o
    ctx.set_delhommeau_method("table")
    A, B, Fd = mixed
    acc = {}
    for name, a, b in (("A", A[:, :, sub], out64[0]), ("B", B[:, :, sub], out64[1]),
                       ("F", Fd[:, sub], out64[2])):
        acc[name] = float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
    acc["note"] = "max abs difference / max abs value, mixed vs FP64 GPU path, same frequencies"
    return res, acc


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--res", type=int, nargs=2, default=[64, 64])
    ap.add_argument("--n-omega", type=int, default=64)
    # relative residual of the FP64 refinement; 1e-8 takes two sweeps and leaves A, B, F within
    # 4e-10 and the gradients within 2e-8 of the FP64 path (the metric asks 1e-6 and 1e-5)
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--max-iter", type=int, default=30)
    ap.add_argument("--fp64-omegas", type=int, default=8)
    ap.add_argument("--cpu-columns", type=int, default=64)
    ap.add_argument("--lu", default="tcgen05", choices=["tcgen05", "simt"])
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-grads", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
