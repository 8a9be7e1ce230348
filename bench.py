"""Benchmark: GF bank cells/s on the graded-soil workload.

One step = one full Green's-function bank of the graded-soil workload
(10 finite layers over a half-space, 2048 frequencies x 16384 wavenumbers x
1024 ranges, complex Dunkin propagators in FP64, shared-grid quadrature),
recomputed from the medium: layer constants, static coefficients, the
propagator over every (f, k) and the wavenumber sum. The Hankel (J0) weights
depend only on the plan's grid and ranges and are built by its first execute;
the e2e leg builds a new plan, weights included, every step.

  value  cells/s with the medium already on the device (gfk_plan_execute),
         timed with CUDA events on the plan's stream, L2 flushed between steps
  e2e    cells/s through the host C ABI (gfk_bank_spectra): host medium and
         grids in, the FP64 bank read back to pinned host memory, every step

Multi-GPU (torchrun): every rank builds its own bank (weak scaling, no
collective on the data path); the timing is the max over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import ctypes
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "GF bank cells/s at relL2≤1e-6 vs FP64; surrogate speedup at ≤1% error"
UNIT = "cells/s"


def dist_init(args):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch
        import torch.distributed as dist
        if dist.get_backend() == "nccl":
            dist.barrier(device_ids=[torch.cuda.current_device()])
        else:
            dist.barrier()


def allmax(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled every 10 ms through
    NVML while the timed region runs (read-only queries)."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "hw_power_brake_slowdown": 0x80, "sw_power_cap": 0x4}

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.stop_flag = threading.Event()
        self.thread = None

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = None
            try:
                import torch
                prop = torch.cuda.get_device_properties(self.device)
                bus = f"{prop.pci_domain_id:08x}:{prop.pci_bus_id:02x}:{prop.pci_device_id:02x}.0"
                h = pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            self.nv, self.h = pynvml, h
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None
            return
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()

    def _run(self):
        nv, h = self.nv, self.h
        while not self.stop_flag.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((sm, reasons))
            except Exception:
                pass
            time.sleep(0.01)

    def stop(self):
        if not self.thread:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.stop_flag.set()
        self.thread.join(timeout=2)
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        reasons = sorted({name for _, r in self.rows for name, bit in self.REASONS.items() if r & bit})
        return {"sm_mhz": statistics.median(r[0] for r in self.rows), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.rows)}


# Used when MEASURED_PEAKS.json is absent: an earlier measurement on the same
# B200 pool (STREAM-style copy; cuBLAS BF16 GEMM burst and sustained).
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}


def measured_peaks():
    """The roofline denominators: MEASURED_PEAKS.json when present (source
    "measured"), else FALLBACK_PEAKS (source "fallback")."""
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        if isinstance(d, dict):
            return {**d, "source": "measured"}
    except (OSError, ValueError):
        pass
    return {**FALLBACK_PEAKS, "source": "fallback"}


def fp64_gemm_peak(torch):
    """cuBLAS FP64 GEMM throughput (TFLOP/s), best of 5, as the FP64 denominator."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2 * n ** 3 / (best * 1e-3) / 1e12


def propagated_layers(stack, freqs, omega_imag, k, ref_freq=30.0, default_q=0.0):
    """Mean number of finite layers the Dunkin solve propagates per
    (frequency, wavenumber) once it starts at the shallowest layer thick enough
    to isolate the ones beneath (start_layer in csrc/gfk_solver.cuh: both
    Re(1 - c^2/v^2) (k h)^2 above kThick^2 = 23^2), evaluated on the given
    sample grid.
    The propagator's algorithmic count assumes every finite layer."""
    wc2 = (2 * np.pi * np.asarray(freqs) - 1j * omega_imag) ** 2
    c2 = wc2[:, None] / (np.asarray(k) ** 2)[None, :]
    fin = stack[:-1]
    top = np.full(c2.shape, len(fin), dtype=np.int64)
    open_ = np.ones(c2.shape, dtype=bool)

    def velocity(v, q, f):  # the Kjartansson velocity at the complex frequency (fk.go:96-110)
        if q <= 0:
            return np.full(f.shape, v, dtype=np.complex128)
        gam = np.arctan(1.0 / q) / np.pi
        z = (omega_imag + 2j * np.pi * f) / (2 * np.pi * ref_freq)
        return v * np.cos(np.pi * gam / 2) * np.exp(gam * np.log(z))

    f = np.asarray(freqs, dtype=np.float64)
    for i, lay in enumerate(fin):
        q = lay.qs if lay.qs > 0 else (default_q if default_q > 0 else 30.0)
        qp = lay.qp if lay.qp > 0 else 2.25 * q
        a, b = velocity(lay.vp, qp, f), velocity(lay.vs, q, f)
        pa = 1.0 - np.real(c2 / (a * a)[:, None])
        pb = 1.0 - np.real(c2 / (b * b)[:, None])
        zeta = np.asarray(k)[None, :] * lay.thickness
        thick = open_ & (np.minimum(pa, pb) * zeta * zeta > 23.0 ** 2)
        top[thick] = i
        open_ &= ~thick
    return float(top.mean())


def cpu_baseline(gfk, wl, threads, target_s=15.0):
    """The oracle's restatement of the reference algorithm (reference-direct:
    Qp = 2.25 Qs, real frequency, guard), compiled -O3 -march=native for this
    host, on a bounded sample of the workload: all ranges, the full wavenumber
    grid, frequencies from the band the reference answers, on `threads` host
    threads (one frequency per thread at a time, as geobank's goroutines)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    timed, flags = O.timed_lib()
    st = [(l.thickness, l.vp, l.vs, l.density, l.qs, 0.0) for l in wl.stack]
    m = O.OracleMedium(st)
    answered = np.array([O.check_layer_phase(m, f) == 0 for f in wl.freqs])
    band = wl.freqs[answered]
    # one probe frequency per thread to size the sample
    probe = band[np.linspace(0, len(band) - 1, threads).astype(int)]
    t0 = time.perf_counter()
    O.bank_spectra(m, wl.ranges, probe, samples=wl.samples, kmax=wl.kmax, threads=threads, library=timed)
    per_round = time.perf_counter() - t0
    rounds = max(1, int(target_s / max(per_round, 1e-3)))
    sample = band[np.linspace(0, len(band) - 1, min(len(band), rounds * threads)).astype(int)]
    t0 = time.perf_counter()
    _, status = O.bank_spectra(m, wl.ranges, sample, samples=wl.samples, kmax=wl.kmax, threads=threads,
                               library=timed)
    dt = time.perf_counter() - t0
    cells = len(sample) * len(wl.ranges)
    return {"value": cells / dt, "unit": UNIT, "cores": threads, "threads": threads, "kind": "port",
            "flags": flags, "bins_sampled": int(len(sample)), "bins_answered": int(len(band)),
            "band": "reference parity band: the bins the reference's MaxLayerPhase guard answers "
                    f"({band.min():.2f}-{band.max():.2f} Hz of {wl.freqs.min():.2f}-{wl.freqs.max():.2f} Hz)",
            "sample": f"{len(sample)} of the {len(band)} bins the reference answers (<= guard), all "
                      f"{len(wl.ranges)} ranges, {wl.samples} wavenumbers, reference-direct restatement "
                      f"(oracle/gfk_oracle.c built {flags}), {dt:.1f} s on {threads} threads",
            "status_ok": bool((status == 0).all())}


def cpu_baseline_batched(soils, ranges, nk, kmax, threads, target_s=12.0, nsample=8):
    """The same restatement on the uneven soils: `nsample` soils spread over
    the seeded list, for each the bins the reference's guard answers, sampled
    so the whole leg takes about target_s on `threads` host threads."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    timed, flags = O.timed_lib()
    picks = [soils[i] for i in np.linspace(0, len(soils) - 1, nsample).astype(int)]
    cases = []
    for st, fr in picks:
        m = O.OracleMedium([(l.thickness, l.vp, l.vs, l.density, l.qs, 0.0) for l in st])
        band = fr[np.array([O.check_layer_phase(m, f) == 0 for f in fr])]
        if len(band):
            cases.append((m, band))
    # size the sample with one round of `threads` bins of the first soil
    m0, b0 = cases[0]
    probe = b0[np.linspace(0, len(b0) - 1, threads).astype(int)]
    t0 = time.perf_counter()
    O.bank_spectra(m0, ranges, probe, samples=nk, kmax=kmax, threads=threads, library=timed)
    per_bin = (time.perf_counter() - t0) / len(probe) * threads
    per_soil = max(threads, int(target_s / max(per_bin, 1e-6) * threads / len(cases)))
    cells, bins, dt, ok = 0, 0, 0.0, True
    for m, band in cases:
        sample = band[np.linspace(0, len(band) - 1, min(len(band), per_soil)).astype(int)]
        t0 = time.perf_counter()
        _, status = O.bank_spectra(m, ranges, sample, samples=nk, kmax=kmax, threads=threads, library=timed)
        dt += time.perf_counter() - t0
        cells += len(sample) * len(ranges)
        bins += len(sample)
        ok &= bool((status == 0).all())
    return {"value": cells / dt, "unit": UNIT, "cores": threads, "threads": threads, "kind": "port",
            "flags": flags, "bins_sampled": bins, "soils_sampled": len(cases),
            "band": "reference parity band per soil: the bins the reference's MaxLayerPhase guard answers",
            "sample": f"{bins} bins of {len(cases)} of the soils (evenly spread over the seeded list), all "
                      f"{len(ranges)} ranges, {nk} wavenumbers, reference-direct restatement "
                      f"(oracle/gfk_oracle.c built {flags}), {dt:.1f} s on {threads} threads",
            "status_ok": ok}


def run_reference(args):
    rank, world, local = dist_init(args)
    if rank != 0:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    import __graft_entry__
    gfk = __graft_entry__.load_package()
    wl = gfk.workloads.single_soil() if args.workload == "single" else gfk.workloads.graded_soil()
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_baseline(gfk, wl, threads, target_s=2.0)
    vals = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        cb = cpu_baseline(gfk, wl, threads, target_s=8.0)
        vals.append(cb["value"])
    dt = time.perf_counter() - t0
    value = statistics.mean(vals)
    out = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * dt / max(args.steps, 1),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic", "config": config_of(wl, "reference-direct restatement on host cores"),
           "cpu_baseline": dict(cb, value=value),
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def config_of(wl, note):
    if wl.name == "single_soil":
        soil = ("0.5 m (Vs 150, Vp 300, rho 1700, Qs 15, Qp 30) and 2 m (250, 500, 1800, 25, 50) layers over a "
                "half-space (400, 800, 2000, 40, 80)")
        l2 = "L2 flushed (256 MiB write) between timed steps; the 32 MB integrand fits in L2"
    else:
        soil = ("10 finite 0.8 m layers (Vs 120->600 m/s, Vp=2Vs, rho 1600->2100, Qs 10->60, Qp=2Qs) over a "
                "half-space")
        l2 = ("intermediates (537 MB integrand, 268 MB int8 digit planes; 134 MB J0 table on the FP64 path) exceed L2; "
              "L2 also flushed (256 MiB write) between timed steps")
    return {"workload": f"{wl.name}: {soil}; {len(wl.freqs)} bins 0-500 Hz (fs 1 kHz), "
                        f"{wl.samples} wavenumbers to {wl.kmax:.1f} rad/m, {len(wl.ranges)} ranges "
                        f"{wl.ranges[0]:g}-{wl.ranges[-1]:g} m, w_I = pi/T",
            "soils": 1, "frequencies": len(wl.freqs), "wavenumbers": wl.samples, "ranges": len(wl.ranges),
            "cells_per_step": wl.cells(), "l2": l2, "note": note}


# DRAM traffic of one graded-soil propagator launch per frequency it
# processes (dram__bytes_read.sum + dram__bytes_write.sum of an ncu capture,
# divided by the captured launch's frequencies).
PROP_TRAFFIC_BYTES_PER_FREQ = (1305600 + 231434496 + 1118208 + 228752896) / 2 / 1024
PROP_TRAFFIC_SOURCE = ("ncu capture (dram__bytes_read.sum + dram__bytes_write.sum, 2 launches) of k_prop on every "
                       "other frequency of the graded soil (1024 x 16384, a 268 MB integrand > L2), scaled by "
                       "frequencies")


def dev_view(torch, ptr, count, local):
    """A float64 torch tensor over `count` doubles of libgfk device memory
    (no copy)."""
    class _Buf:
        __cuda_array_interface__ = {"shape": (count,), "typestr": "<f8", "data": (ptr, False), "version": 3}
    return torch.as_tensor(_Buf(), device=f"cuda:{local}")


def abi_bank_spectra(gfk, eng, med, wl, out_host, status_host):
    """The call geobank would make: gfk_bank_spectra through the C ABI, host
    medium and grids in, the [nf][nr] complex128 bank into the pinned
    `out_host` (a torch tensor of nf x 2 nr float64)."""
    from gfk_b200.fk import _c_medium
    N = gfk._native
    r = np.ascontiguousarray(wl.ranges)
    f = np.ascontiguousarray(wl.freqs)
    with _c_medium(med) as cm:
        st = N.lib().gfk_bank_spectra(eng.ctx, ctypes.byref(cm), ctypes.byref(med._solve()),
                                      r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(r),
                                      f.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(f),
                                      wl.integration().c(),
                                      ctypes.cast(out_host.data_ptr(), ctypes.POINTER(ctypes.c_double)),
                                      ctypes.cast(status_host.data_ptr(), ctypes.POINTER(ctypes.c_int32)))
    eng.check(st)


def abi_bank_payload(gfk, eng, med, wl, bins, out_host, status_host):
    """geobank's own output through the C ABI: gfk_bank_payload, the bank
    file's float32 range-major payload packed on the device and downloaded
    into the pinned `out_host` (2 nr bins float32)."""
    from gfk_b200.fk import _c_medium
    N = gfk._native
    r = np.ascontiguousarray(wl.ranges)
    f = np.ascontiguousarray(wl.freqs)
    with _c_medium(med) as cm:
        st = N.lib().gfk_bank_payload(eng.ctx, ctypes.byref(cm), ctypes.byref(med._solve()),
                                      r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(r),
                                      f.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(f),
                                      wl.integration().c(), 1, bins,
                                      ctypes.cast(out_host.data_ptr(), ctypes.POINTER(ctypes.c_float)),
                                      ctypes.cast(status_host.data_ptr(), ctypes.POINTER(ctypes.c_int32)))
    eng.check(st)


def single_leg(gfk, torch, eng, local, world, fp64_peak, steps=20, warmup=5, cpu=True):
    """The single-soil workload (2 layers over a half-space, 512 bins x 64
    ranges, 4096 wavenumbers) for the default bench line, in the plain FP64
    form (the reference's complex128 bank, computed by the FP64 propagator
    and the FP64 tensor-core sum) with the split sum beside it: device-resident
    stream span (L2 flushed between steps), end to end through gfk_bank_spectra
    into pinned host memory, the propagator's roofline, and the CPU baseline
    on the bins the reference answers."""
    wl = gfk.workloads.single_soil()
    gstream = torch.cuda.ExternalStream(eng.stream(), device=f"cuda:{local}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    out = {"workload": "single_soil: 0.5 m (Vs 150, Vp 300, rho 1700, Qs 15, Qp 30) and 2 m (250, 500, 1800, 25, 50) "
                       "layers over a half-space (400, 800, 2000, 40, 80); 512 bins 0-500 Hz (fs 1 kHz), 4096 "
                       f"wavenumbers to {wl.kmax:.1f} rad/m, 64 ranges 1-64 m, w_I = pi/T",
           "cells_per_step": wl.cells() * world}
    got = {}
    for name, quad in (("plain_fp64", gfk.PLAIN_FP64), ("split", gfk.SPLIT_INT8)):
        med = wl.medium(gfk.DUNKIN, engine=eng, quadrature=quad)
        plan = gfk.Plan(med, wl.ranges, wl.freqs, wl.integration(), engine=eng)
        for _ in range(warmup):
            plan.execute()
        got[name], st = plan.download()
        assert (st == 0).all()
        plan.kernel_times(reset=True)
        spans = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        launches0 = eng.kernel_launches()
        with torch.cuda.stream(gstream):
            for a, b in spans:
                flush.fill_(1)
                a.record(gstream)
                plan.execute()
                b.record(gstream)
        torch.cuda.synchronize()
        launches = eng.kernel_launches() - launches0
        prop_ms, quad_ms, other_ms = plan.kernel_times(reset=True)
        ms = allmax(sum(a.elapsed_time(b) for a, b in spans) / steps, world)
        plan.close()
        host = torch.empty((len(wl.freqs), 2 * len(wl.ranges)), dtype=torch.float64, pin_memory=True)
        hstat = torch.zeros(len(wl.freqs), dtype=torch.int32, pin_memory=True)
        abi_bank_spectra(gfk, eng, med, wl, host, hstat)
        t0 = time.perf_counter()
        for _ in range(steps):
            abi_bank_spectra(gfk, eng, med, wl, host, hstat)
        e2e_s = allmax((time.perf_counter() - t0) / steps, world)
        kgrid = np.arange(1, wl.samples + 1) * (wl.kmax / wl.samples)
        lx = propagated_layers(wl.stack, wl.freqs[::4], wl.omega_imag, kgrid[::4])
        f_exec = len(wl.freqs) * wl.samples * (700 * lx + 300)
        f_fixed = len(wl.freqs) * wl.samples * (700 * (len(wl.stack) - 1) + 300)
        out[name] = {"value": wl.cells() * world / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms, "steps": steps,
                     "warmup": warmup, "gpu_launches": launches,
                     "kernel_ms": {"propagator": prop_ms, "quadrature": quad_ms, "other": other_ms},
                     "e2e": {"value": wl.cells() * world / e2e_s, "unit": UNIT, "ms_per_step": e2e_s * 1e3,
                             "h2d_bytes_per_step": len(wl.stack) * 48 + len(wl.ranges) * 8 + len(wl.freqs) * 36,
                             "d2h_bytes_per_step": wl.cells() * 16 + len(wl.freqs) * 4},
                     "roofline": {"bound": "fp64", "kernel": "k_prop (Dunkin propagator)",
                                  "achieved": f_exec / (prop_ms * 1e-3) / 1e12, "peak": fp64_peak, "unit": "TFLOP/s",
                                  "frac": f_exec / (prop_ms * 1e-3) / 1e12 / fp64_peak,
                                  "mean_layers_propagated": lx,
                                  "fixed_count_frac": f_fixed / (prop_ms * 1e-3) / 1e12 / fp64_peak}}
    a, b = got["plain_fp64"], got["split"]
    out["split"]["relL2_split_vs_fp64"] = float(np.linalg.norm(b - a) / np.linalg.norm(a))
    out["value"], out["unit"], out["ms_per_step"] = out["plain_fp64"]["value"], UNIT, out["plain_fp64"]["ms_per_step"]
    out["timing"] = "stream span of each execute on libgfk's stream, L2 flushed (256 MiB write) between steps"
    if cpu:
        cb = cpu_baseline(gfk, wl, os.cpu_count() or 1, target_s=8.0)
        cb.pop("status_ok", None)
        out["cpu_baseline"] = cb
    del flush
    return out


def learned_leg(gfk, torch, eng, world, steps=200, warmup=10):
    """The learned part at a size that fits the default bench run.

    Training throughput (config 4's network and batch): FP64 labels for 8192
    soils of the 11-scalar family from the batched solver, then `steps`
    timed AdamW steps of the BF16 6 x 512 network (batch 8192, one CUDA graph
    per step). Surrogate gain (config 5's sweep at N = 256): three members
    trained 20,000 steps on 16,384 Sobol-box soils at the sensor range answer
    the 2560-soil Saltelli sweep; the row gate re-solves disputed and
    energetic rows with the plain f-k solve; reported against the all-plain
    run: rows solved, wall time of both runs, and Sobol index errors."""
    U, S = gfk.surrogate, gfk.sobol
    out = {}
    params = U.draw(8192, 20240611)
    t0 = time.perf_counter()
    ds = U.Dataset(params, U.LabelGrid(), floor_rel=1e-6, engine=eng).fill(batch_soils=8192)
    label_s = time.perf_counter() - t0
    train, _ = U.split_soils(len(params), 0.05, 0)
    net = U.Net(U.NetConfig(total_steps=warmup + steps, loss_mode=gfk._native.LOSS_PLAIN), eng)
    net.scales_from(ds)
    net.train(ds, train, warmup)
    launches0 = eng.kernel_launches()
    t0 = time.perf_counter()
    net.train(ds, train, steps)  # returns after the stream is synchronised
    dt = allmax(time.perf_counter() - t0, world)
    launches = eng.kernel_launches() - launches0
    B = net.config.batch
    flops = 2 * B * (128 * 512 + 4 * 512 * 512 + 2 * 512) * 3 - 2 * B * 128 * 512  # fwd + dX + dW, no dX0
    ms = 1e3 * dt / steps
    pk = measured_peaks()
    out["train"] = {"workload": "surrogate training: 8192 3-layer soils x 64 ranges x 512 bins of FP64 labels "
                                f"({label_s:.1f} s), batch 8192, 128 features -> 5 x 512 SiLU -> 2, AdamW",
                    "value": B * steps * world / dt, "unit": "samples/s", "ms_per_step": ms, "steps": steps,
                    "warmup": warmup, "gpu_launches": int(launches), "dtype": "bf16",
                    "roofline": {"bound": "tensor", "achieved": flops / (ms * 1e-3) / 1e12,
                                 "peak": pk.get("bf16_tflops"), "unit": "TFLOP/s",
                                 "frac": flops / (ms * 1e-3) / 1e12 / pk["bf16_tflops"] if pk.get("bf16_tflops") else None,
                                 "peak_source": pk["source"]}}
    net.close()
    ds.close()
    rng = np.random.default_rng(20240611)
    p11 = U.from_sobol(S.unit_to_params(rng.random((16384, 8))))
    ds = U.Dataset(p11, U.LabelGrid(), floor_rel=1e-6, engine=eng).fill(batch_soils=8192)
    train, _ = U.split_soils(len(p11), 0.05, 0)
    t0 = time.perf_counter()
    cfg = U.NetConfig(total_steps=20000, lr_max=1e-3, warmup_steps=200)
    nets = U.train_ensemble(ds, train, members=3, steps=20000, config=cfg, engine=eng, ranges=(9, 10))
    train_s = time.perf_counter() - t0
    ds.close()
    S.run_plain(eng, n=256, seed=0)  # warm-up of both paths (allocator, first launches)
    S.run_surrogate(eng, nets, n=256, seed=0, threshold=0.01, gate="rows", amp_threshold=0.001)
    plain = S.run_plain(eng, n=256, seed=0)
    sur = S.run_surrogate(eng, nets, n=256, seed=0, threshold=0.01, gate="rows", amp_threshold=0.001)
    for n_ in nets:
        n_.close()
    err = max(abs(getattr(sur, kind)[o][q] - getattr(plain, kind)[o][q])
              for kind in ("s1", "st") for o in ("peak", "centroid") for q in getattr(sur, kind)[o])
    out["surrogate"] = {"workload": "Saltelli N=256, d=8 (2560 soils x 512 bins at 10 m); 3 members trained 20,000 "
                                    f"steps on 16,384 Sobol-box soils at the sensor range ({train_s:.1f} s, not counted); "
                                    "row gate: members disagree by > 1% of the trace-spectrum peak or predicted "
                                    "|G S| > 0.1% of it",
                        "fk_rows_fraction": sur.seconds["fallback_fraction"],
                        "speedup_wall": plain.seconds["total"] / sur.seconds["total"],
                        "timing": "wall time of each whole run after one untimed run of each",
                        "plain_s": plain.seconds["total"], "surrogate_s": sur.seconds["total"],
                        "max_index_abs_error": err,
                        "peak_metric_rel_error_p90": float(np.percentile(
                            np.abs(sur.metrics["peak"] / plain.metrics["peak"] - 1), 90))}
    return out


def batched_leg(gfk, torch, eng, local, rank, world, fp64_peak, steps=3, cpu=True):
    """The 4096 seeded uneven soils (256-2048 bins each, 8192 wavenumbers, 128
    ranges; this rank's share) as one batch plan with the split sum, for the
    default bench line: device-resident throughput (one CUDA graph per
    execute, stream span), end to end from host media into pinned host
    memory, the split sum's rel-L2 against the FP64 sum of the same bank per
    soil, the propagator's roofline and a CPU baseline on a sample."""
    soils, ranges, nk, kmax = gfk.workloads.batched_soils()
    mine = gfk.workloads.shard(soils, rank, world)
    opt = gfk.Integration(nk, 0.0, kmax)
    freqs = [fr for _, fr in mine]
    rows = [len(fr) for fr in freqs]
    nrows = sum(rows)
    nr = len(ranges)
    cells = nrows * nr

    def media(quad):
        return [gfk.Medium(st, formulation=gfk.DUNKIN, quadrature=quad, engine=eng) for st, _ in mine]

    gstream = torch.cuda.ExternalStream(eng.stream(), device=f"cuda:{local}")
    t0 = time.perf_counter()
    plan = gfk.Batch(media(gfk.SPLIT_INT8), freqs, ranges, opt, engine=eng)
    build_s = time.perf_counter() - t0
    plan.execute()  # first execute: launch-shape and tile-shape tuning, the Hankel weights
    prop_shape = plan.tuning()
    tc_shape = plan.quad_shape()
    plan.kernel_times(reset=True)
    plan.execute()  # one execute timed kernel by kernel
    prop_ms, quad_ms, other_ms = plan.kernel_times(reset=True)
    plan.use_graph(True)
    plan.execute()  # captures the graph
    torch.cuda.synchronize()
    launches0 = eng.kernel_launches()
    spans = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    barrier(world)
    with torch.cuda.stream(gstream):
        for a, b in spans:
            a.record(gstream)
            plan.execute()
            b.record(gstream)
    torch.cuda.synchronize()
    launches = eng.kernel_launches() - launches0
    step_ms = allmax(sum(a.elapsed_time(b) for a, b in spans) / steps, world)
    cells_all = cells * world
    value = cells_all / (step_ms * 1e-3)

    # the split sum against the FP64 sum of the same integrand, per soil, on the device
    pp = gfk.Batch(media(gfk.PLAIN_FP64), freqs, ranges, opt, engine=eng)
    pp.execute()
    st_split, st_plain = plan.statuses(), pp.statuses()
    torch.cuda.synchronize()
    gs = dev_view(torch, plan.result_device_ptr(), nrows * nr * 2, local).view(nrows, nr * 2)
    gp = dev_view(torch, pp.result_device_ptr(), nrows * nr * 2, local).view(nrows, nr * 2)
    num = torch.empty(nrows, dtype=torch.float64, device=gs.device)
    den = torch.empty_like(num)
    for r0 in range(0, nrows, 1 << 18):
        r1 = min(nrows, r0 + (1 << 18))
        num[r0:r1] = (gs[r0:r1] - gp[r0:r1]).square().sum(1)
        den[r0:r1] = gp[r0:r1].square().sum(1)
    soil_of = torch.as_tensor(np.repeat(np.arange(len(rows)), rows), device=gs.device)
    snum = torch.zeros(len(rows), dtype=torch.float64, device=gs.device).index_add_(0, soil_of, num)
    sden = torch.zeros_like(snum).index_add_(0, soil_of, den)
    per_soil = (snum / sden).sqrt().cpu().numpy()
    per_row = (num / den).sqrt()
    accuracy = {"relL2_split_vs_fp64_per_soil": {"max": float(per_soil.max()),
                                                  "median": float(np.median(per_soil)),
                                                  "worst_soil": int(np.argmax(per_soil))},
                "relL2_whole_bank": float((num.sum() / den.sum()).sqrt()),
                "max_row_relL2": float(per_row.max()),
                "soils_over_1e-6": int((per_soil > 1e-6).sum()),
                "statuses_ok": bool((st_split == 0).all() and (st_plain == 0).all())}
    del gs, gp, num, den, per_row
    pp.close()

    # end to end: host media and grids in, the FP64 rows back into pinned host memory
    host_rows = torch.empty(nrows * nr * 2, dtype=torch.float64, pin_memory=True).numpy()
    host_rows = host_rows.view(np.complex128).reshape(nrows, nr)
    barrier(world)
    t0 = time.perf_counter()
    e2e_plan = gfk.Batch(media(gfk.SPLIT_INT8), freqs, ranges, opt, engine=eng)
    e2e_plan.execute_download(out=host_rows)  # each chunk's rows copied out while the next computes
    e2e_s = allmax(time.perf_counter() - t0, world)
    e2e_plan.close()
    layers = sum(len(st) for st, _ in mine)
    plan.close()

    # the propagator's roofline: fixed count (every finite layer) and the
    # layers actually propagated, sampled on every 16th soil's grid
    flops = sum(len(fr) * nk * (700 * (len(st) - 1) + 300) for st, fr in mine)
    kgrid = np.arange(1, nk + 1) * (kmax / nk)
    en = ed = 0.0
    for st, fr in mine[::16]:
        lx = propagated_layers(st, fr[::8], 0.0, kgrid[::32])
        en += len(fr) * (700 * lx + 300)
        ed += len(fr) * (700 * (len(st) - 1) + 300)
    exec_ratio = en / ed if ed else 1.0
    ach = flops * exec_ratio / (prop_ms * 1e-3) / 1e12
    out = {"workload": f"batched_soils: {len(soils)} seeded soils (2-12 entries, Vs log-U 80-600, Vp/Vs U 1.7-3.0, "
                       f"rho U 1500-2200, Qs U 10-60, Qp 2Qs, h log-U 0.2-5 m), 256-2048 bins each over 0-500 Hz, "
                       f"{nk} wavenumbers to {kmax:.1f} rad/m, {nr} ranges 1-128 m, real frequencies; split sum; "
                       "one CUDA graph per execute",
           "value": value, "unit": UNIT, "ms_per_step": step_ms, "steps": steps, "warmup": 3,
           "timing": "stream span of each graph launch (CUDA events on libgfk's stream), mean over the steps, max "
                     "over ranks; the 9.7 GB result and the 4 GB integrand chunks exceed L2, so no flush",
           "soils_per_rank": len(mine), "rows_per_rank": nrows, "cells_per_step": cells_all,
           "plan_build_s": build_s, "gpu_launches": launches,
           "autotuned": {"propagator_launch_shape": gfk.prop_shape(prop_shape[0]),
                         "propagator_tuning_ms": prop_shape[1],
                         "tensor_core_tile": {"ranges_per_cta": tc_shape[0], "stages": tc_shape[1],
                                              "tuning_ms_per_shape": tc_shape[2]}},
           "kernel_ms": {"propagator": prop_ms, "quadrature": quad_ms, "other": other_ms},
           "e2e": {"value": cells_all / e2e_s, "unit": UNIT, "s_per_step": e2e_s, "steps": 1,
                   "h2d_bytes_per_step": layers * 48 + nrows * 8,
                   "d2h_bytes_per_step": nrows * nr * 16 + nrows * 4,
                   "note": "plan build from host media, execute with each row chunk downloaded into pinned host "
                           "memory while the next computes (gfk_plan_execute_download)"},
           "accuracy": accuracy,
           "roofline": {"bound": "fp64", "kernel": "k_prop (Dunkin propagator)", "achieved": ach,
                        "peak": fp64_peak, "unit": "TFLOP/s", "frac": ach / fp64_peak, "traffic": None,
                        "work": "executed: 700 flops per finite layer actually propagated + 300 per (f, k), the "
                                "propagated share sampled on every 16th soil",
                        "executed_share_of_fixed_count": exec_ratio,
                        "fixed_count": {"tflops": flops / (prop_ms * 1e-3) / 1e12,
                                        "frac": flops / (prop_ms * 1e-3) / 1e12 / fp64_peak}}}
    if cpu:
        cb = cpu_baseline_batched(soils, ranges, nk, kmax, os.cpu_count() or 1)
        cb.pop("status_ok", None)
        out["cpu_baseline"] = cb
    return out


def run_batched(args, gfk, torch, rank, world, local):
    """The seeded uneven soils: every rank builds its own share of the soils
    (round-robin by cost, no collective on the data path); one CUDA-graph
    execute per step."""
    soils, ranges, nk, kmax = gfk.workloads.batched_soils(count=args.soils)
    mine = gfk.workloads.shard(soils, rank, world)
    eng = gfk.Engine(local)
    quad = gfk.PLAIN_FP64 if args.quadrature == "fp64" else gfk.SPLIT_INT8
    media = [gfk.Medium(st, formulation=gfk.DUNKIN, quadrature=quad, engine=eng) for st, _ in mine]
    freqs = [fr for _, fr in mine]
    opt = gfk.Integration(nk, 0.0, kmax)
    cells = sum(len(f) for f in freqs) * len(ranges)
    t0 = time.perf_counter()
    plan = gfk.Batch(media, freqs, ranges, opt, engine=eng)
    build_s = time.perf_counter() - t0
    for _ in range(max(args.warmup, 1)):
        plan.execute()
    got, status = plan.download()
    assert (status == 0).all() and np.isfinite(got).all()
    plan.use_graph(True)
    plan.execute()  # capture
    plan.kernel_times(reset=True)
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = eng.kernel_launches()
    barrier(world)
    torch.cuda.synchronize()
    t_wall = time.perf_counter()
    for _ in range(args.steps):
        plan.execute()
    torch.cuda.synchronize()
    barrier(world)
    wall = time.perf_counter() - t_wall
    launches = eng.kernel_launches() - launches0
    _, _, graph_ms = plan.kernel_times(reset=True)
    clk = clocks.stop()
    step_ms = allmax(graph_ms, world)
    prop_choice, prop_tune_ms = plan.tuning()
    tc_tn, tc_stages, tc_tune_ms = plan.quad_shape()
    cells_all = int(allmax(cells, world) if world == 1 else cells * world)
    value = cells_all / (step_ms * 1e-3)
    # end to end: host media and grids in, the FP64 rows back into pinned host memory
    nrows_mine = sum(len(f) for f in freqs)
    host_rows = torch.empty(nrows_mine * len(ranges) * 2, dtype=torch.float64, pin_memory=True).numpy()
    host_rows = host_rows.view(np.complex128).reshape(nrows_mine, len(ranges))
    t0 = time.perf_counter()
    e2e_plan = gfk.Batch(media, freqs, ranges, opt, engine=eng)
    rows, st = e2e_plan.execute_download(out=host_rows)
    e2e_s = allmax(time.perf_counter() - t0, world)
    e2e_plan.close()
    nrows = sum(len(f) for f in freqs)
    layers = sum(len(m.stack) for m in media)
    flops = sum(len(fr) * nk * (700 * (len(stk) - 1) + 300) for stk, fr in mine)
    # layers actually propagated (thick-layer start), on every 16th soil's sampled grid
    kgrid = np.arange(1, nk + 1) * (kmax / nk)
    num = den = 0.0
    for stk, fr in mine[::16]:
        lx = propagated_layers(stk, fr[::8], media[0].omega_imag, kgrid[::32])
        num += len(fr) * (700 * lx + 300)
        den += len(fr) * (700 * (len(stk) - 1) + 300)
    exec_ratio = num / den if den else 1.0
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": f"batched_soils: {args.soils} seeded soils (2-12 entries, Vs log-U 80-600, "
                                      f"Vp/Vs U 1.7-3.0, rho U 1500-2200, Qs U 10-60, Qp 2Qs, h log-U 0.2-5 m), "
                                      f"256-2048 bins each over 0-500 Hz, {nk} wavenumbers to {kmax:.1f} rad/m, "
                                      f"{len(ranges)} ranges 1-128 m; one CUDA graph per execute",
                          "soils_per_rank": len(mine), "rows_per_rank": nrows, "cells_per_step": cells_all,
                          "quadrature": args.quadrature},
               "e2e": {"value": cells_all / e2e_s, "unit": UNIT, "h2d_bytes_per_step": layers * 48 + nrows * 8,
                       "d2h_bytes_per_step": nrows * len(ranges) * 16 + nrows * 4, "s_per_step": e2e_s},
               "gpu_launches": launches, "clocks": clk, "plan_build_s": build_s,
               "autotuned": {"propagator_launch_shape": gfk.prop_shape(prop_choice),
                             "propagator_tuning_ms": prop_tune_ms,
                             "tensor_core_tile": {"ranges_per_cta": tc_tn, "stages": tc_stages,
                                                  "tuning_ms_per_shape": tc_tune_ms}},
               "propagator_fp64_tflops_algorithmic": flops / (step_ms * 1e-3) / 1e12,
               "propagator_executed": {
                   "note": "the fixed count above assumes every finite layer; the solve starts at the shallowest "
                           "layer thick enough to isolate the ones beneath (sampled on every 16th soil)",
                   "flops_fraction": exec_ratio, "tflops": flops * exec_ratio / (step_ms * 1e-3) / 1e12},
               "wall_s_timed_region": wall}
        print(json.dumps(out))
    plan.close()
    eng.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_sobol(args, gfk, torch, rank, world, local):
    """The all-plain Sobol run: N(d+2) soils, each through the GPU f-k solve at
    10 m (512 bins, 8192 wavenumbers), traces, metrics, indices. One step is
    the whole run; ranks would split the soils (weak scaling in soils)."""
    S = gfk.sobol
    eng = gfk.Engine(local)
    t0 = time.perf_counter()
    res = S.run_plain(eng, n=args.sobol_n, seed=0)
    wall = time.perf_counter() - t0
    eng.close()
    if rank == 0:
        cells = res.seconds["rows"]
        out = {"metric": METRIC, "value": cells / res.seconds["solve_gpu"], "unit": UNIT, "n_gpus": world,
               "steps": 1, "warmup": 0, "ms_per_step": 1e3 * res.seconds["solve_gpu"], "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": {"workload": f"sobol plain: Saltelli N={args.sobol_n}, d=8 soil parameters, "
                                      f"{res.seconds['soils']} soils x 512 bins at 10 m, 8192 wavenumbers, "
                                      "75 kg footstep through an SM-24-like geophone (10 Hz, 0.7)",
                          "soils": res.seconds["soils"], "rows": cells},
               "e2e": {"value": cells / wall, "unit": UNIT, "s_per_run": wall,
                       "h2d_bytes_per_step": res.seconds["soils"] * 3 * 48 + 513 * 16,
                       "d2h_bytes_per_step": res.seconds["soils"] * 2 * 8 + cells * 4},
               "sobol": {"S1": res.s1, "ST": res.st,
                         "seconds": {k: v for k, v in res.seconds.items() if k not in ("rows", "soils")}}}
        print(json.dumps(out))


def run_fdtd(args, gfk, torch, rank, world, local):
    """The finite-difference validator on a grid far larger than L2: a lossy
    (SLS, Q 25 at 30 Hz) two-layer model 60 m x 40 m at 2 cm spacing
    (3021 x 2021 cells with the absorbing layers), K time steps after W
    warm-up steps, two kernels per step."""
    F = gfk.fdtd
    eng = gfk.Engine(local)
    st = gfk.Stack([gfk.Layer(2.0, 350.0, 140.0, 1600.0, 0, 0), gfk.Layer(0.0, 800.0, 320.0, 2000.0, 0, 0)])
    md = F.Model(st, relax=gfk.SLS.fit(25.0, 30.0), ref_freq=30, max_range=60, depth=40, spacing=0.02,
                 dominant_freq=25)
    dt, nr, nz = md.grid()
    force = F.ricker(1000, 25, dt, args.warmup + args.steps)
    F.run(F.Shot(md, force, [5.0], max(args.warmup, 3)), engine=eng)  # warm the allocator and kernels
    barrier(world)
    t0 = time.perf_counter()
    res = F.run(F.Shot(md, force, [5.0, 20.0], args.steps), engine=eng)
    dt_wall = time.perf_counter() - t0  # run() returns after the stream is synchronised
    t = allmax(dt_wall, world)
    cells = nr * nz
    # algorithmic bytes per cell-step (lossy interior): velocities read 6 fields, write 2;
    # stresses read 10 (4 stresses, 2 velocities, 4 memory variables), write 8
    bytes_per = (6 + 2 + 10 + 8) * 8
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import fdtd_oracle as FO
        sim = FO.Sim([(2.0, 350.0, 140.0, 1600.0), (0.0, 800.0, 320.0, 2000.0)], FO.SLS.fit(25.0, 30.0), 30,
                     60, 40, 0.02, dominant_freq=25)
        sim.force = force
        c0 = time.perf_counter()
        ns = 0
        while time.perf_counter() - c0 < 10.0:
            sim.do_step()
            ns += 1
        cs = time.perf_counter() - c0
        cpu = {"value": cells * ns / cs, "unit": "cell-updates/s", "cores": 1, "kind": "port",
               "sample": f"{ns} steps of the same grid through the numpy restatement (oracle/fdtd_oracle.py)"}
    eng.close()
    if rank == 0:
        ms = 1e3 * t / args.steps
        ach = cells * bytes_per / (ms * 1e-3) / 1e9
        pks = measured_peaks()
        peak = pks.get("hbm_gbs")
        out = {"metric": "FDTD cell-updates/s (axisymmetric velocity-stress, SLS, C-PML)",
               "value": cells * args.steps * world / t, "unit": "cell-updates/s", "n_gpus": world,
               "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "gpu_launches": 2 * args.steps + (args.steps + 255) // 256,
               "config": {"workload": f"fdtd: 2-layer lossy soil 60 m x 40 m at 2 cm ({nr} x {nz} cells), "
                                      "Ricker 25 Hz vertical force, 2 receivers", "inputs_vs_l2": "fields, memory variables and C-PML state 0.9 GB > L2"},
               "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                            "frac": ach / peak if peak else None, "traffic": None, "peak_source": pks["source"]},
               "cpu_baseline": cpu, "peak_speed": res.peak}
        print(json.dumps(out))


def run_consume(args, gfk, torch, rank, world, local):
    """Bank consumption (internal/sensing's use of a bank): the graded-soil
    bank (2049 bins x 1024 ranges, fs 1 kHz, 4096-sample transform) built by
    the solver and opened on the device once (payload and Bank.prepare
    tables resident); per step the causal velocity impulse responses of 8192
    query ranges (1024 samples each): bracket, Bank.Response interpolation,
    i w, taper and inverse FFT on the device. `value` writes the responses to
    device memory; `e2e` returns them to pinned host memory."""
    eng = gfk.Engine(local)
    wl = gfk.workloads.graded_soil()
    med = wl.medium(gfk.DUNKIN, engine=eng, quadrature=gfk.SPLIT_INT8)
    spectra, st = med.bank_spectra(wl.ranges, wl.freqs, wl.integration())
    h = gfk.Header(gfk.Provenance("gfk-b200 fk"), wl.stack, wl.fs, wl.transform_samples,
                   gfk.RangeGrid(0.5, 512.0, 1024),
                   "vertical surface displacement per unit vertical surface point force", "m/N")
    b = gfk.Bank.new(h)
    b.data[:, 1:len(wl.freqs) + 1, 0] = spectra.T.real
    b.data[:, 1:len(wl.freqs) + 1, 1] = spectra.T.imag
    nq, length = 8192, 1024
    q = np.random.default_rng(5).uniform(0.5, 512.0, nq)
    t_open = time.perf_counter()
    db = b.device(eng)
    t_open = time.perf_counter() - t_open
    dev = torch.empty((nq, length), dtype=torch.float64, device=f"cuda:{local}")
    host = torch.empty((nq, length), dtype=torch.float64, pin_memory=True).numpy()
    for _ in range(max(args.warmup, 3)):
        db.impulse_responses(q, length, out_device_ptr=dev.data_ptr())
        db.impulse_responses(q, length, out=host)
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        db.impulse_responses(q, length, out_device_ptr=dev.data_ptr())  # returns with the responses written
    t = allmax(time.perf_counter() - t0, world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        db.impulse_responses(q, length, out=host)
    t_e2e = allmax(time.perf_counter() - t0, world)
    clk = clocks.stop()
    t_one = time.perf_counter()
    one = b.impulse_responses(q[:1024], length, engine=eng)  # the one-shot call: payload up, tables, responses
    t_one = time.perf_counter() - t_one
    assert np.isfinite(host).all() and np.array_equal(one, host[:1024])
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import bank_oracle as BO
        c0 = time.perf_counter()
        BO.prepare(b.data)
        c_prep = time.perf_counter() - c0
        ns = 32
        c0 = time.perf_counter()
        want = BO.impulse_responses(b.data, (0.5, 512.0), wl.fs, wl.transform_samples, q[:ns], length)
        c_all = time.perf_counter() - c0  # includes one more prepare
        per_q = max(c_all - c_prep, 1e-9) / ns
        rel = float(np.linalg.norm(host[:ns] - want) / np.linalg.norm(want))
        cpu = {"value": 1.0 / per_q, "unit": "impulse responses/s", "cores": 1, "kind": "port",
               "sample": f"{ns} queries ({per_q * 1e3:.1f} ms each) through the numpy restatement "
                         f"(oracle/bank_oracle.py) after its Bank.prepare ({c_prep:.1f} s, not counted, as the "
                         f"device bank's one-off open is not)",
               "relL2_gpu_vs_oracle_on_sample": rel}
    db.close()
    eng.close()
    if rank == 0:
        ms = 1e3 * t / args.steps
        out_bytes = nq * length * 8
        print(json.dumps({
            "metric": "bank impulse responses/s (internal/sensing from a device-resident bank)",
            "value": nq * args.steps * world / t, "unit": "impulse responses/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"consume: graded-soil bank 2049 bins x 1024 ranges (0.5-512 m) opened on the "
                                   f"device once ({1e3 * t_open:.1f} ms), {nq} query ranges per step, velocity "
                                   f"responses of {length} samples (4096-point transform)"},
            "e2e": {"value": nq * args.steps * world / t_e2e, "unit": "impulse responses/s",
                    "h2d_bytes_per_step": nq * 12, "d2h_bytes_per_step": out_bytes,
                    "ms_per_step": 1e3 * t_e2e / args.steps},
            "one_shot_call": {"queries": 1024, "ms": 1e3 * t_one,
                              "note": "gfk_bank_impulse_responses: pageable payload upload, tables, responses"},
            "gpu_launches": 2 * args.steps, "clocks": clk, "cpu_baseline": cpu}))


def run_disp(args, gfk, torch, rank, world, local):
    """Rayleigh dispersion curves (internal/disp over propmat.Secular): every
    mode of the 10-layer graded soil at 512 frequencies 2-200 Hz per step, one
    gfk_dispersion_modes call (a 2000-sample velocity scan per frequency, then
    one bisection per bracket, one block per frequency)."""
    D = gfk.disp
    eng = gfk.Engine(local)
    wl = gfk.workloads.graded_soil()
    stack = wl.stack
    freqs = np.linspace(2.0, 200.0, 512)
    for _ in range(max(args.warmup, 3)):
        res = D.modes_many(stack, freqs, engine=eng)
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        res = D.modes_many(stack, freqs, engine=eng)
    t = allmax(time.perf_counter() - t0, world)
    clk = clocks.stop()
    roots = sum(len(r) for r in res)
    samples, lfin = 2000, len(stack) - 1
    # secular evaluations per step: the scan (samples + 1 per frequency) plus
    # ~22 bisection halvings per root (bracket (hi - lo)/2000 down to 1e-10 relative)
    evals = len(freqs) * (samples + 1) + 22 * roots
    flops_eval = 3000 * lfin + 200  # per finite layer: 4x4 exponential, 6x6 compound, minor update
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import disp_oracle as DO
        tup = [(l.thickness, l.vp, l.vs, l.density) for l in stack]
        c0 = time.perf_counter()
        ns = 0
        worst = 0.0
        while ns < 2 or (time.perf_counter() - c0 < 10.0 and ns < len(freqs)):
            i = (ns * 97) % len(freqs)
            want = DO.modes(tup, freqs[i])
            got = res[i]
            if len(want) == len(got) and want:
                worst = max(worst, max(abs(a - b) / b for a, b in zip(got, want)))
            ns += 1
        cs = time.perf_counter() - c0
        cpu = {"value": ns / cs, "unit": "frequencies/s", "cores": 1, "kind": "port",
               "sample": f"{ns} of the frequencies through the numpy/scipy restatement (oracle/disp_oracle.py)",
               "max_rel_root_diff_gpu_vs_oracle_on_sample": worst}
    eng.close()
    if rank == 0:
        ms = 1e3 * t / args.steps
        ach = evals * flops_eval / (ms * 1e-3) / 1e12
        fp64_peak = fp64_gemm_peak(torch)
        print(json.dumps({
            "metric": "dispersion frequencies/s (all Rayleigh modes per frequency)",
            "value": len(freqs) * args.steps * world / t, "unit": "frequencies/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"disp: graded soil (10 layers over a half-space), {len(freqs)} frequencies "
                                   f"2-200 Hz, 2000-sample scan, tolerance 1e-10; {roots} roots per step"},
            "e2e": {"value": len(freqs) * args.steps * world / t, "unit": "frequencies/s",
                    "h2d_bytes_per_step": len(freqs) * 8 + len(stack) * 48,
                    "d2h_bytes_per_step": len(freqs) * (64 * 8 + 4)},  # modes_many's [nf][64] roots + counts
            "gpu_launches": args.steps,
            "roofline": {"bound": "fp64", "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s",
                         "frac": ach / fp64_peak, "traffic": None,
                         "note": "end-to-end call time; evaluations estimated as the scan plus ~22 bisection "
                                 "steps per root, each counted at 3000 flops per finite layer + 200"},
            "clocks": clk, "cpu_baseline": cpu}))


def run_train(args, gfk, torch, rank, world, local):
    """Surrogate training throughput: labels for --sur-soils family soils
    from the batched FP64 solver, then W warm-up and K timed AdamW steps of
    the BF16 network (batch 8192, one CUDA graph per step: batch gather,
    5 forward GEMMs, head/loss, 4 backward-data GEMMs, 5 weight-gradient
    GEMMs, bias sums, loss record, AdamW)."""
    U = gfk.surrogate
    eng = gfk.Engine(local)
    params = U.draw(args.sur_soils, 20240611)
    ds = U.Dataset(params, U.LabelGrid(), floor_rel=1e-6, engine=eng).fill(batch_soils=8192)
    train, _ = U.split_soils(args.sur_soils, 0.05, 0)
    net = U.Net(U.NetConfig(total_steps=args.warmup + args.steps, loss_mode=gfk._native.LOSS_PLAIN), eng)
    net.scales_from(ds)
    net.train(ds, train, max(args.warmup, 3))
    launches0 = eng.kernel_launches()
    barrier(world)
    t0 = time.perf_counter()
    loss = net.train(ds, train, args.steps)
    dt = time.perf_counter() - t0  # train() returns after the stream is synchronised
    launches = eng.kernel_launches() - launches0
    B = net.config.batch
    flops = 2 * B * (128 * 512 + 4 * 512 * 512 + 2 * 512) * 3 - 2 * B * 128 * 512  # fwd + dX + dW, no dX0
    t = allmax(dt, world)
    net.close()
    ds.close()
    eng.close()
    if rank == 0:
        ms = 1e3 * t / args.steps
        out = {"metric": "surrogate training samples/s (BF16 MLP 6x512, AdamW)", "value": B * args.steps * world / t,
               "unit": "samples/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
               "data": "synthetic", "gpu_launches": int(launches),
               "config": {"workload": f"surrogate training: {args.sur_soils} 3-layer soils x 64 ranges x 512 bins "
                                      "labels, batch 8192, 128 features -> 5 x 512 SiLU -> 2"},
               "roofline": {"bound": "tensor", "achieved": flops / (ms * 1e-3) / 1e12,
                            "peak": measured_peaks().get("bf16_tflops"), "unit": "TFLOP/s",
                            "frac": None, "traffic": None, "peak_source": measured_peaks()["source"]},
               "final_loss": loss[-100:].mean(axis=0).tolist()}
        pk = out["roofline"]["peak"]
        if pk:
            out["roofline"]["frac"] = out["roofline"]["achieved"] / pk
        print(json.dumps(out))


def run_surrogate(args, gfk, torch, rank, world, local):
    """The learned part end to end on one GPU: labels for the 3-layer soil
    family from the batched FP64 solver, an ensemble of BF16 networks trained
    by libgfk's kernels, held-out error, then the Sobol run with the
    surrogate answering and the plain f-k solve as fallback, against the
    all-plain Sobol run. One step is the whole pipeline."""
    S, U = gfk.sobol, gfk.surrogate
    eng = gfk.Engine(local)
    log = (lambda m: print(m, file=sys.stderr, flush=True)) if rank == 0 else (lambda m: None)
    t0 = time.perf_counter()
    if args.sur_family == "sobol":
        # the Sobol soils' own 8-parameter box, as members of the 11-scalar family
        params = U.from_sobol(S.unit_to_params(np.random.default_rng(20240611).random((args.sur_soils, 8))))
    else:
        params = U.draw(args.sur_soils, 20240611)
    ds = U.Dataset(params, U.LabelGrid(), floor_rel=1e-6, engine=eng).fill(batch_soils=8192)
    t_data = time.perf_counter() - t0
    m0, s0, m1, s1, frac = ds.stats()
    log(f"labels: {args.sur_soils} soils in {t_data:.1f} s (solver {ds.solve_ms / 1e3:.1f} s GPU); "
        f"t0 {m0:.3f}+-{s0:.3f}, t1 {m1:.3e}+-{s1:.3e}, phase cells {frac:.3f}")
    train, held = U.split_soils(args.sur_soils, 0.05, 0)
    cfg = U.NetConfig(total_steps=args.sur_steps, lr_max=args.sur_lr, fourier_sigma=args.sur_sigma)
    t1 = time.perf_counter()
    ranges = tuple(int(x) for x in args.sur_ranges.split(",")) if args.sur_ranges else None
    nets = U.train_ensemble(ds, train, members=args.members, steps=args.sur_steps, config=cfg, engine=eng, log=log,
                            ranges=ranges)
    t_train = time.perf_counter() - t1
    evals = [n.evaluate(ds, held) for n in nets]
    for i, e in enumerate(evals):
        log(f"member {i} held-out: " + ", ".join(f"{k} {v:.4g}" for k, v in e.items()))
    if args.save_nets:
        pathlib.Path(args.save_nets).mkdir(parents=True, exist_ok=True)
        for i, n in enumerate(nets):
            n.save(pathlib.Path(args.save_nets) / f"member{i}.npz")
    ds.close()
    res_p = S.run_plain(eng, n=args.sobol_n, seed=0)
    log(f"plain sobol: {res_p.seconds}")
    res_s = S.run_surrogate(eng, nets, n=args.sobol_n, seed=0, threshold=args.threshold, gate="rows",
                            amp_threshold=args.amp_threshold)
    log(f"surrogate sobol (row gate): {res_s.seconds}")
    res_g = S.run_surrogate(eng, nets, n=args.sobol_n, seed=0, threshold=args.threshold, gate="soil")
    log(f"surrogate sobol (soil gate): {res_g.seconds}")

    def index_errors(res):
        err = {}
        for kind, a, b in (("S1", res.s1, res_p.s1), ("ST", res.st, res_p.st)):
            for out in ("peak", "centroid"):
                err[f"{kind}_{out}"] = max(abs(a[out][k] - b[out][k]) for k in a[out])
        return err

    def metric_errors(res):
        return {out: np.percentile(np.abs(res.metrics[out] / res_p.metrics[out] - 1), [50, 90, 99]).tolist()
                for out in ("peak", "centroid")}

    err = index_errors(res_s)
    rel = metric_errors(res_s)
    eng.close()
    if rank == 0:
        speed = res_p.seconds["total"] / res_s.seconds["total"]
        out = {"metric": "surrogate speedup at <=1% error (Sobol indices, surrogate+fallback vs all-plain GPU)",
               "value": speed, "unit": "x", "n_gpus": world, "steps": 1, "warmup": 0,
               "ms_per_step": 1e3 * res_s.seconds["total"], "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "bf16", "data": "synthetic",
               "config": {"workload": f"surrogate: {args.sur_soils} 3-layer soils ({args.sur_family} box) x 64 ranges "
                                      f"x 512 bins labels (training ranges {args.sur_ranges or 'all'}), "
                                      f"{args.members} x MLP 6x512 SiLU BF16 {args.sur_steps} steps batch 8192; "
                                      f"Sobol N={args.sobol_n} d=8 at 10 m; f-k fallback on the rows where the "
                                      f"ensemble spread exceeds {args.threshold:.0%} of the trace-spectrum peak "
                                      f"or the predicted |G S| exceeds {args.amp_threshold:.1%} of it"},
               "index_abs_error": err, "metric_rel_error_p50_p90_p99": rel,
               "soil_gate": {"speedup": res_p.seconds["total"] / res_g.seconds["total"],
                             "index_abs_error": index_errors(res_g), "metric_rel_error_p50_p90_p99":
                             metric_errors(res_g), "seconds": res_g.seconds},
               "held_out": evals, "seconds": {"labels": t_data, "train": t_train,
                                             "plain_sobol": res_p.seconds, "surrogate_sobol": res_s.seconds},
               "sobol": {"surrogate": {"S1": res_s.s1, "ST": res_s.st}, "plain": {"S1": res_p.s1, "ST": res_p.st}}}
        print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gfk", choices=["gfk", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--freq-stride", type=int, default=1,
                    help="profiling only: keep every n-th frequency (a smaller case of the same kernels)")
    ap.add_argument("--workload", default="graded", choices=["graded", "single", "batched", "sobol", "surrogate", "train",
                                                              "fdtd", "consume", "disp"],
                    help="graded: the 10-layer graded soil (default); batched: seeded uneven soils; "
                         "sobol: the all-plain Sobol run")
    ap.add_argument("--sobol-n", type=int, default=16384, help="sobol workload: Saltelli base size N")
    ap.add_argument("--soils", type=int, default=4096, help="batched workload: number of soils")
    ap.add_argument("--sur-soils", type=int, default=65536, help="surrogate workload: labelled soils")
    ap.add_argument("--sur-steps", type=int, default=150000, help="surrogate workload: steps per member")
    ap.add_argument("--sur-lr", type=float, default=3e-4)
    ap.add_argument("--sur-sigma", type=float, default=8.0, help="Fourier feature frequency std")
    ap.add_argument("--members", type=int, default=4, help="surrogate ensemble size")
    ap.add_argument("--sur-family", default="box", choices=["box", "sobol"],
                    help="surrogate training soils: box = the 11-scalar family's box; sobol = the Sobol "
                         "soils' 8-parameter box inside it")
    ap.add_argument("--sur-ranges", default="", help="surrogate training range indices r0,r1 (default: all)")
    ap.add_argument("--threshold", type=float, default=0.01, help="ensemble spread above which soils fall back")
    ap.add_argument("--amp-threshold", type=float, default=0.001,
                    help="row gate: also re-solve rows whose predicted |G S| exceeds this share of the soil's peak")
    ap.add_argument("--save-nets", default="", help="directory to save the trained members")
    ap.add_argument("--quadrature", default="split", choices=["split", "fp64"],
                    help="split: exact int8-slice tensor-core sum (default); fp64: the plain FP64 sum")
    ap.add_argument("--no-batched", action="store_true",
                    help="default workload: skip the single-soil, batched, training and surrogate objects in the line")
    ap.add_argument("--profile", action="store_true",
                    help="profiling only: skip the e2e leg, the FP64 peak probe and the CPU baseline")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    rank, world, local = dist_init(args)
    torch.cuda.set_device(local)
    import __graft_entry__
    gfk = __graft_entry__.load_package()
    if args.workload == "batched":
        return run_batched(args, gfk, torch, rank, world, local)
    if args.workload == "sobol":
        return run_sobol(args, gfk, torch, rank, world, local)
    if args.workload == "surrogate":
        return run_surrogate(args, gfk, torch, rank, world, local)
    if args.workload == "consume":
        return run_consume(args, gfk, torch, rank, world, local)
    if args.workload == "disp":
        return run_disp(args, gfk, torch, rank, world, local)
    if args.workload == "train":
        return run_train(args, gfk, torch, rank, world, local)
    if args.workload == "fdtd":
        return run_fdtd(args, gfk, torch, rank, world, local)
    wl = gfk.workloads.single_soil() if args.workload == "single" else gfk.workloads.graded_soil()
    if args.freq_stride > 1:
        wl.freqs = wl.freqs[::args.freq_stride].copy()
    eng = gfk.Engine(local)
    quad = gfk.PLAIN_FP64 if args.quadrature == "fp64" else gfk.SPLIT_INT8
    med = wl.medium(gfk.DUNKIN, engine=eng, quadrature=quad)
    plan = gfk.Plan(med, wl.ranges, wl.freqs, wl.integration(), engine=eng)
    # libgfk queues its work on its own (non-blocking) stream: the L2 flush
    # and the span events go on that stream, in order with the kernels
    gstream = torch.cuda.ExternalStream(eng.stream(), device=f"cuda:{local}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    for _ in range(max(args.warmup, 0)):
        plan.execute()
    got, status = plan.download()
    assert (status == 0).all() and np.isfinite(got).all()
    plan.kernel_times(reset=True)
    variant, tune_ms = plan.tuning()
    tc_tn, tc_stages, tc_tune_ms = plan.quad_shape()

    # --- device-resident timing: the stream span of each execute ----------
    clocks = ClockSampler(local)
    clocks.start()
    launches0 = eng.kernel_launches()
    spans = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier(world)
    torch.cuda.synchronize()
    t_wall = time.perf_counter()
    with torch.cuda.stream(gstream):
        for a, b in spans:
            flush.fill_(1)
            a.record(gstream)
            plan.execute()
            b.record(gstream)
    torch.cuda.synchronize()
    barrier(world)
    wall = time.perf_counter() - t_wall
    launches = eng.kernel_launches() - launches0
    prop_ms, quad_ms, other_ms = plan.kernel_times(reset=True)
    kernel_sum_ms = prop_ms + quad_ms + other_ms
    span_ms = sum(a.elapsed_time(b) for a, b in spans) / max(args.steps, 1)
    clk = clocks.stop()
    step_ms = allmax(span_ms, world)
    cells_all = wl.cells() * world
    value = cells_all / (step_ms * 1e-3)

    # --- end-to-end through the host C ABI ------------------------------
    out_host = torch.empty((len(wl.freqs), 2 * len(wl.ranges)), dtype=torch.float64, pin_memory=True)
    status_host = torch.zeros(len(wl.freqs), dtype=torch.int32, pin_memory=True)
    N = gfk._native
    r = np.ascontiguousarray(wl.ranges)
    f = np.ascontiguousarray(wl.freqs)

    def e2e_call():
        abi_bank_spectra(gfk, eng, med, wl, out_host, status_host)

    if args.profile:
        plan.close()
        eng.close()
        print(json.dumps({"profile_run": True, "ms_per_step": step_ms, "kernel_ms": [prop_ms, quad_ms, other_ms],
                          "prop_variant": variant, "tune_ms": tune_ms}))
        return
    e2e_call()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_call()
    e2e_s = allmax((time.perf_counter() - t0) / max(args.steps, 1), world)
    e2e_value = cells_all / e2e_s
    bins = wl.transform_samples // 2 + 1
    pay_host = torch.empty(2 * len(wl.ranges) * bins, dtype=torch.float32, pin_memory=True)
    abi_bank_payload(gfk, eng, med, wl, bins, pay_host, status_host)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        abi_bank_payload(gfk, eng, med, wl, bins, pay_host, status_host)
    pay_s = allmax((time.perf_counter() - t0) / max(args.steps, 1), world)
    nl = len(wl.stack)
    h2d = nl * 48 + len(r) * 8 + len(f) * (8 + 8 + 8 + 4 + 8)
    d2h = len(f) * len(r) * 16 + len(f) * 4

    # --- the plain FP64 path on the same bank: accuracy bar and speed ratio ---
    plain_leg = None
    if quad == gfk.SPLIT_INT8:
        mp = wl.medium(gfk.DUNKIN, engine=eng)
        pp = gfk.Plan(mp, wl.ranges, wl.freqs, wl.integration(), engine=eng)
        for _ in range(max(args.warmup, 1)):
            pp.execute()
        ref, rst = pp.download()
        rel = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        per_bin = float(np.max(np.linalg.norm(got - ref, axis=1) / np.linalg.norm(ref, axis=1)))
        pp.kernel_times(reset=True)
        pspans = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(args.steps)]
        with torch.cuda.stream(gstream):
            for a, b in pspans:
                flush.fill_(1)
                a.record(gstream)
                pp.execute()
                b.record(gstream)
        torch.cuda.synchronize()
        pprop, pquad, pother = pp.kernel_times(reset=True)
        pms = allmax(sum(a.elapsed_time(b) for a, b in pspans) / max(args.steps, 1), world)
        plain_leg = {"value": cells_all / (pms * 1e-3), "unit": UNIT, "ms_per_step": pms,
                     "kernel_ms": {"propagator": pprop, "quadrature": pquad, "other": pother},
                     "split_over_plain": pms / step_ms,
                     "relL2_split_vs_fp64": rel, "max_bin_relL2_split_vs_fp64": per_bin}
        pp.close()

    # --- roofline of the dominant kernel --------------------------------
    peaks = measured_peaks()
    fp64_peak = fp64_gemm_peak(torch)
    lfin = nl - 1
    f_prop = len(f) * wl.samples * (700 * lfin + 300)   # algorithmic FP64 flops per propagator launch
    f_quad = 4 * len(f) * wl.samples * len(r)           # complex x real MAC, per quadrature launch
    kgrid = np.arange(1, wl.samples + 1) * (wl.kmax / wl.samples)
    l_exec = propagated_layers(wl.stack, wl.freqs[::8], wl.omega_imag, kgrid[::8])
    f_exec = len(f) * wl.samples * (700 * l_exec + 300)
    if prop_ms >= quad_ms:
        dom, ach = "k_prop (Dunkin propagator)", f_exec / (prop_ms * 1e-3) / 1e12
    else:
        dom, ach = ("k_quad_gemm (FP64 wavenumber sum)" if quad == gfk.PLAIN_FP64 else
                    "k_quad_tc (tensor-core wavenumber sum)"), f_quad / (quad_ms * 1e-3) / 1e12
    # DRAM bytes of one propagator launch, from an ncu capture of the graded
    # soil's every-other-frequency case (its 268 MB integrand exceeds L2),
    # scaled by the frequencies one full launch processes
    traffic, traffic_src = None, None
    if args.workload != "single" and args.freq_stride == 1 and prop_ms >= quad_ms:
        traffic = PROP_TRAFFIC_BYTES_PER_FREQ * len(f)
        traffic_src = PROP_TRAFFIC_SOURCE
    roof_time = (f_prop + f_quad) / (fp64_peak * 1e12)
    roofline = {"bound": "fp64", "kernel": dom, "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": ach / fp64_peak, "traffic": traffic, "traffic_source": traffic_src,
                "work": "executed: 700 flops per finite layer actually propagated (the thick-layer start skips "
                        "layers beneath the shallowest isolating one) + 300 per (f, k)",
                "peak_source": "measured here: cuBLAS FP64 GEMM 8192^3 best of 5 (MEASURED_PEAKS.json has no FP64 "
                               "figure)",
                "algorithmic_flops": {"propagator_fixed": f_prop, "propagator_executed": f_exec,
                                      "quadrature": f_quad},
                "mean_layers_propagated": l_exec, "finite_layers": lfin,
                "fixed_count": {"note": "the same launch credited with every finite layer (700 flops each) + 300 per (f, k)",
                                "tflops": f_prop / (prop_ms * 1e-3) / 1e12,
                                "frac": f_prop / (prop_ms * 1e-3) / 1e12 / fp64_peak},
                "step_frac_of_fp64_roofline": roof_time / (step_ms * 1e-3),
                "kernel_ms": {"propagator": prop_ms, "quadrature": quad_ms, "other": other_ms},
                "propagator_launch_shape": {"chosen": variant, "shape": gfk.prop_shape(variant),
                                            "tuning_ms": tune_ms},
                "quadrature": {"path": "split int8 slices on tcgen05 (10 slice GEMMs)" if quad == gfk.SPLIT_INT8
                               else "plain FP64 on the FP64 tensor cores", "ms": quad_ms,
                               "tile_shape": {"ranges_per_cta": tc_tn, "stages": tc_stages,
                                              "tuning_ms_per_shape": tc_tune_ms,
                                              "shapes": "(128, 3), (128, 2), (64, 4), (64, 3)"}
                               if quad == gfk.SPLIT_INT8 else None,
                               "useful_tflops": f_quad / (quad_ms * 1e-3) / 1e12,
                               "int8_tops_executed": (10 * 2 * 2 * len(f) * len(r) * wl.samples) / (quad_ms * 1e-3) / 1e12
                               if quad == gfk.SPLIT_INT8 else None},
                "hbm_gbs_peak": peaks.get("hbm_gbs"), "hbm_peak_source": peaks["source"]}
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(gfk, wl, os.cpu_count() or 1)
        cb.pop("status_ok", None)
    plan.close()
    del flush
    single = batched = learned = None
    if not args.no_batched and args.workload == "graded" and args.freq_stride == 1:
        learned = learned_leg(gfk, torch, eng, world)
        single = single_leg(gfk, torch, eng, local, world, fp64_peak,
                            cpu=(rank == 0 and world == 1 and not args.no_cpu_baseline))
        batched = batched_leg(gfk, torch, eng, local, rank, world, fp64_peak,
                              steps=min(args.steps, 3), cpu=(rank == 0 and world == 1 and not args.no_cpu_baseline))
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f64", "data": "synthetic",
               "config": dict(config_of(wl, "Dunkin formulation, FP64 propagators; " +
                                        ("wavenumber sum as exact int8 slices on the tcgen05 tensor cores, FP64 "
                                         "recombination" if quad == gfk.SPLIT_INT8 else "FP64 wavenumber sum")),
                              parallelism=f"replicas{world}" if world > 1 else "single"),
               "timing": {"value_is": "stream span of each execute (CUDA events on libgfk's stream around it, the "
                                      "L2 flush outside), mean over the timed steps, max over ranks",
                          "kernel_sum_ms_per_step": kernel_sum_ms},
               "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                       "ms_per_step": e2e_s * 1e3},
               "e2e_bank_payload": {"value": cells_all / pay_s, "unit": UNIT, "ms_per_step": pay_s * 1e3,
                                    "h2d_bytes_per_step": h2d,
                                    "d2h_bytes_per_step": 8 * len(wl.ranges) * bins + 4 * len(wl.freqs),
                                    "note": "geobank's output: gfk_bank_payload packs the bank file's float32 "
                                            "range-major payload on the device and downloads only that"},
               "gpu_launches": launches, "clocks": clk, "roofline": roofline,
               "wall_s_timed_region": wall}
        if cb:
            out["cpu_baseline"] = cb
        if plain_leg:
            out["plain_fp64"] = plain_leg
        if learned:
            out.update(learned)
        if single:
            out["single"] = single
        if batched:
            out["batched"] = batched
        print(json.dumps(out))
    eng.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
