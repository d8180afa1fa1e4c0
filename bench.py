"""Benchmark of the multislice hot path: multislice steps/s on 512^2 waves.

Workload (one line of the headline STEM scan, see jmultislicelib_b200/synthetic.py
SCAN_512): 512x512 complex64 waves, 200 slices over 4 slice types with 16
frozen-phonon variants each, 300 kV / 22 mrad / Cs 1 um probe, Fresnel
propagator with 2/3 band limit, 3 annular detectors read every 20 slices plus
the 128x128 binned exit diffraction pattern.  One bench step = one raster row
of 64 probe positions x 16 phonon passes x 200 slices = 204,800 multislice
steps (the full scan is 64 such rows).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torch.distributed.run, one rank per GPU; each rank takes its
own raster rows (weak scaling, no data-path collective); timing is the max
over ranks.  --impl reference times the reference's own CPU path
(CJMultiSlice::CPUMultislice on MKL, compiled from the reference sources into
oracle/_ref) on the host cores with the same workload, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "multislice steps/s (512² wave)"
UNIT = "steps/s"
# tensor-core forms reported beside the FP32 headline: (JMS_SetPrecision mode, name)
TC_FORMS = ((1, "bf16"), (2, "fp16"))
# tensor FLOPs per point of one 512-point pass: 4 radix stages (32, 16, 16, 32),
# 5 hi/lo products of 8 R flops per point each
TC_FLOP_PER_POINT = 5 * 8 * (32 + 16 + 16 + 32)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while running."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) >= 9:
                for k, nm in enumerate(names):
                    if r[5 + k].lower().startswith("active"):
                        reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


# ---------------------------------------------------------------------------
# reference CPU path (oracle/_ref): the reported baseline and the reference arm
# ---------------------------------------------------------------------------
def reference_cpu(cfg, sp, probe, pro, dets, pos, nthreads, npos_sample, npass_sample=1):
    """Times CJMultiSlice::CPUMultislice of the reference on nthreads host
    threads over npos_sample positions x npass_sample passes; returns steps/s."""
    from oracle import ref

    if not ref.available():
        raise RuntimeError("oracle/_ref/libjms_ref.so is not built")
    objs = []
    objslc = np.arange(cfg["nobj"]) % cfg["nslice_types"]
    for t in range(nthreads):
        R = ref.RefJMS()
        R.set_high_tension(cfg["kv"])
        R.set_grid(cfg["nx"], cfg["ny"], sp.a, sp.b, 0.19525)
        R.setup(ref.CODE_CPU, [cfg["nvar"]] * cfg["nslice_types"], objslc, [0] * cfg["nslice_types"],
                cfg["ndetper"], len(dets), 1, 1)
        for s, gr in enumerate(sp.gratings):
            R.set_phase_grating(ref.CODE_CPU, s, gr)
        R.set_propagator(ref.CODE_CPU, 0, pro)
        for i, (d, m) in enumerate(dets):
            R.set_detector(ref.CODE_CPU, i, d, m)
        R.init_core(ref.CODE_CPU, 1)
        R.set_incident_wave(ref.CODE_CPU, probe)
        R.seed(1000 + t)
        objs.append(R)
    nd = objs[0].num_det_planes()
    sample = pos[:npos_sample]
    t0 = time.perf_counter()
    out, e = ref.cpu_scan(objs, sample, npass_sample, nd * len(dets))
    dt = time.perf_counter() - t0
    assert e == 0, e
    for R in objs:
        R.close()
    steps = npos_sample * npass_sample * cfg["nobj"]
    return steps / dt, dt, out


def reference_gpu(cfg, sp, probe, pro, dets, pos, ours, ours_e2e, npos=4):
    """Times the reference's own GPU path on this GPU: CJMultiSlice::
    GPUMultislice (src/JMultiSlice.cpp:4513-4677, cuFFT + the ArrayOps kernels,
    compiled for sm_100a in oracle/_ref), driven per probe position as the
    reference benchmark drives it, over npos positions x the workload's passes."""
    from oracle import ref

    if not ref.available():
        raise RuntimeError("oracle/_ref/libjms_ref.so is not built")
    npass = cfg["nvar"]
    objslc = np.arange(cfg["nobj"]) % cfg["nslice_types"]
    R = ref.RefJMS()
    try:
        R.set_high_tension(cfg["kv"])
        R.set_grid(cfg["nx"], cfg["ny"], sp.a, sp.b, 0.19525)
        # the wrappers check the reference's return codes themselves
        R.setup(ref.CODE_GPU, [cfg["nvar"]] * cfg["nslice_types"], objslc, [0] * cfg["nslice_types"],
                cfg["ndetper"], len(dets), 1, 1)
        for s_, gr in enumerate(sp.gratings):
            R.set_phase_grating(ref.CODE_GPU, s_, gr)
        R.set_propagator(ref.CODE_GPU, 0, pro)
        for i, (d, m) in enumerate(dets):
            R.set_detector(ref.CODE_GPU, i, d, m)
        R.init_core(ref.CODE_GPU)
        R.set_incident_wave(ref.CODE_GPU, probe)
        R.seed(77)
        nout = R.num_det_planes() * len(dets)
        _, _, e = ref.gpu_scan(R, pos[:1], 1, nout)            # warm-up: cuFFT plans, first launches
        assert e == 0, e
        _, sec, e = ref.gpu_scan(R, pos[:npos], npass, nout)
        assert e == 0, e
    finally:
        R.close()
    steps = npos * npass * cfg["nobj"]
    v = steps / sec
    return {"value": v, "unit": UNIT, "kind": "reference",
            "path": "CJMultiSlice::GPUMultislice (cuFFT + ArrayOps kernels, built for sm_100a), one call per "
                    "position-pass with OffsetIncomingWave and GetResult per position, as JMSBench1 drives it",
            "sample": f"{npos} probe positions x {npass} phonon passes x {cfg['nobj']} slices ({sec:.2f} s)",
            "speedup_value": ours / v, "speedup_e2e": ours_e2e / v}


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from jmultislicelib_b200 import synthetic as S

    cfg = S.SCAN_512
    try:
        from oracle import ref
        if not ref.available():
            raise RuntimeError("reference library oracle/_ref/libjms_ref.so missing")
    except Exception as ex:
        print(json.dumps({"impl": "reference", "unavailable": str(ex)}))
        return 0
    sp = S.make_specimen(cfg["nx"], cfg["ny"], cfg["ncell"], cfg["ncell"], cfg["nslice_types"], cfg["nvar"],
                         cfg["seed"], cfg["kv"])
    # the reference's own generators provide probe, propagator and detectors
    R = ref.RefJMS()
    R.set_high_tension(cfg["kv"])
    R.set_grid(cfg["nx"], cfg["ny"], sp.a, sp.b, 0.19525)
    pro = R.calc_propagator(0.19525, 0.0, 0.0, cfg["ntype"])
    dets = [R.calc_ring_detector(b0, b1) for (b0, b1) in cfg["dets"]]
    ab = np.zeros(48, np.float32)
    ab[10] = cfg["cs"]
    probe = R.calc_probe(cfg["alpha"], abrr=ab)
    R.close()
    mid = (cfg["ncell"] // 2) * S.A_CELL
    pos = S.scan_positions(cfg["nscan"], mid, mid, S.A_CELL)
    nt = host_threads()
    per_step = nt  # one position-pass per thread per step
    rates, times = [], []
    for it in range(args.warmup + args.steps):
        sel = pos[(it * per_step) % len(pos):][:per_step]
        if len(sel) < per_step:
            sel = pos[:per_step]
        r, dt, _ = reference_cpu(cfg, sp, probe, pro, dets, sel, nt, per_step)
        if it >= args.warmup:
            rates.append(r)
            times.append(dt)
    value = per_step * cfg["nobj"] * len(times) / sum(times)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": "STEM scan 512^2, 200 slices, 4 slice types x 16 phonon variants; "
                                   f"bench step = {per_step} position-passes on the host threads",
                       "grid": 512, "slices": cfg["nobj"]},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nt, "kind": "reference",
                             "sample": f"{per_step} probe positions x 1 phonon pass x 200 slices per step "
                                       "(CJMultiSlice::CPUMultislice on MKL DFTI, one thread per position)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# product arm
# ---------------------------------------------------------------------------
def run_ours(args):
    import torch

    import jmultislicelib_b200 as jb
    from jmultislicelib_b200 import synthetic as S

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    cfg = S.SCAN_512
    J = jb.JMS()
    J.L.SetCurrentGPU(local)
    stream = torch.cuda.Stream()
    J.set_stream(stream.cuda_stream)
    J.L.JMS_SetScanBatch(args.batch)
    sp, probe, pro, dets, pos = S.setup_library(J, cfg)
    J.seed(4242 + rank)
    nd = J.num_det_planes()
    ndet = len(dets)
    npos_step = cfg["nscan"]            # one raster row
    npass = cfg["nvar"]
    bin_ = cfg["bin"]
    nbx, nby = cfg["nx"] // bin_, cfg["ny"] // bin_
    steps_per_bench_step = npos_step * npass * cfg["nobj"]
    # waves per launch: with a batch larger than the row, the library puts
    # batch // 64 phonon configurations of the row's positions into each launch
    kp = min(npass, max(1, args.batch // npos_step)) if args.batch > npos_step else 1
    waves = kp * npos_step if args.batch > npos_step else min(args.batch, npos_step)
    dev = torch.device("cuda", local)
    d_pos = torch.from_numpy(pos).to(dev)
    d_int = torch.zeros((len(pos), nd, ndet), dtype=torch.float64, device=dev)
    d_bin = torch.zeros((npos_step, nby, nbx), dtype=torch.float32, device=dev)

    from jmultislicelib_b200 import shard

    my_rows = shard.rows_for_rank(cfg["nscan"], rank, world)

    def row_of(k):
        return my_rows[k % len(my_rows)]

    # FFT plan choice by the library's autotuner (outside the timed region)
    import ctypes as C
    ms_r, ms_c = C.c_float(0), C.c_float(0)
    ir, ic = C.c_int(0), C.c_int(0)
    if J.L.JMS_Autotune(waves, 20, C.byref(ms_r), C.byref(ms_c), C.byref(ir), C.byref(ic)):
        raise RuntimeError("autotune failed")
    print(f"# library kernel launches before the warm-up: {J.L.JMS_KernelLaunches()}", file=sys.stderr)
    names = []
    for axis in (0, 1):
        buf = C.create_string_buffer(64)
        J.L.JMS_PlanName(axis, buf, 64)
        names.append(buf.value.decode())

    def step(k):
        r = row_of(k)
        p = d_pos[r * npos_step:(r + 1) * npos_step]
        o = d_int[r * npos_step:(r + 1) * npos_step]
        e = J.L.JMS_ScanGPUDevice(npos_step, p.data_ptr(), 0.0, npass, None, o.data_ptr(), d_bin.data_ptr(), bin_)
        if e != 0:
            raise RuntimeError(f"JMS_ScanGPUDevice returned {e}")

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    with torch.cuda.stream(stream):
        for k in range(args.warmup):
            step(k)
    torch.cuda.synchronize()
    barrier()
    l0 = J.L.JMS_KernelLaunches()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for k in range(args.steps):
                step(args.warmup + k)
            ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = J.L.JMS_KernelLaunches() - l0
    barrier()
    # per-pass durations: one more bench step with CUDA events around every
    # pass launch (kept out of the headline region above)
    J.L.JMS_SetPassTiming(1)
    with torch.cuda.stream(stream):
        step(args.warmup + args.steps)
    torch.cuda.synchronize()
    mc, mr = C.c_double(0), C.c_double(0)
    nc, nr = C.c_longlong(0), C.c_longlong(0)
    J.L.JMS_PassTiming(C.byref(mc), C.byref(nc), C.byref(mr), C.byref(nr))
    J.L.JMS_SetPassTiming(0)
    barrier()
    # tensor-core forms of the same step (JMS_SetPrecision), reported beside
    # the FP32 headline: steps/s and per-pass device times
    tc_forms = {}
    if world == 1 and not args.no_tc:
        N_ = cfg["nx"] * cfg["ny"]
        for mode, form in TC_FORMS:
            if J.set_precision(mode) != 0:
                tc_forms[form] = {"value": None, "note": "JMS_SetPrecision failed"}
                continue
            tc0 = J.L.JMS_TcLaunches()
            with torch.cuda.stream(stream):
                step(0)
            torch.cuda.synchronize()
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                t0.record(stream)
                for k in range(2):
                    step(1 + k)
                t1.record(stream)
            torch.cuda.synchronize()
            ms_tc = t0.elapsed_time(t1) / 2
            J.L.JMS_SetPassTiming(1)
            with torch.cuda.stream(stream):
                step(3)
            torch.cuda.synchronize()
            tmc, tmr = C.c_double(0), C.c_double(0)
            tnc, tnr = C.c_longlong(0), C.c_longlong(0)
            J.L.JMS_PassTiming(C.byref(tmc), C.byref(tnc), C.byref(tmr), C.byref(tnr))
            J.L.JMS_SetPassTiming(0)
            status = J.tc_status()
            ntc = J.L.JMS_TcLaunches() - tc0
            J.set_precision(0)
            col_us = 1e3 * tmc.value / max(tnc.value, 1)
            flops = waves * N_ * TC_FLOP_PER_POINT   # one column-pass launch, 5 products per radix stage
            tc_forms[form] = {"value": steps_per_bench_step / (ms_tc / 1e3), "unit": UNIT, "ms_per_step": ms_tc,
                              "col_pass_us": col_us, "row_pass_us": 1e3 * tmr.value / max(tnr.value, 1),
                              "col_pass_tflops": flops / (col_us * 1e-6) / 1e12,
                              "col_pass_hbm_frac": waves * 24 * N_ / (col_us * 1e-6) / 1e9 / peaks()[0],
                              "tc_launches": int(ntc), "tc_status": int(status)}
    if world > 1:
        t = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    value = world * args.steps * steps_per_bench_step / (ms / 1e3)

    # the chosen form of the scan (multi-fidelity control variate) against the
    # plain one, same rows and configurations (rank 0 of a single-GPU run)
    chosen_form = None
    if world == 1 and not args.no_chosen:
        try:
            chosen_form = measure_multifidelity(J, cfg, stream, d_pos, npos_step, rows=max(2, args.steps), warmup=1)
        except Exception as ex:
            chosen_form = {"form": None, "note": f"not run: {ex}"}

    # e2e through the host-buffer entry point (pinned host memory)
    h_pos = torch.from_numpy(pos[:npos_step].copy()).pin_memory()
    h_int = torch.zeros((npos_step, nd, ndet), dtype=torch.float32).pin_memory()
    h_bin = torch.zeros((npos_step, nby, nbx), dtype=torch.float32).pin_memory()
    fp = C.POINTER(C.c_float)

    def e2e_step():  # noqa: E306
        e = J.L.JMS_ScanGPU(npos_step, C.cast(h_pos.data_ptr(), fp), 0.0, npass, None,
                            C.cast(h_int.data_ptr(), fp), C.cast(h_bin.data_ptr(), fp), bin_)
        if e != 0:
            raise RuntimeError(f"JMS_ScanGPU returned {e}")

    e2e_steps = max(1, args.steps)
    e2e_step()
    torch.cuda.synchronize()
    barrier()
    e2e_each, e2e_dev = [], []
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(e2e_steps)]
    with ClockSampler(local) as clk_e2e:
        t0 = time.perf_counter()
        for k in range(e2e_steps):
            t1 = time.perf_counter()
            evs[k][0].record(stream)
            e2e_step()            # returns after its device work and the result copy
            evs[k][1].record(stream)
            e2e_each.append(1e3 * (time.perf_counter() - t1))
        torch.cuda.synchronize()
        e2e_s = time.perf_counter() - t0
    e2e_dev = [a.elapsed_time(b) for a, b in evs]
    if world > 1:
        t = torch.tensor([e2e_s], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_value = world * e2e_steps * steps_per_bench_step / e2e_s
    gen = measure_grating_generation(J, cfg) if rank == 0 else None
    multi = None
    if world > 1:   # every rank takes the same collective steps
        try:
            multi = multirank_results(J, cfg, d_pos, npos_step, bin_, nby, nbx, stream, rank, world)
        except Exception as ex:
            multi = {"note": f"not run: {ex}"}

    if rank == 0:
        N = cfg["nx"] * cfg["ny"]
        hbm, src = peaks()
        # dominant pass: algorithmic bytes per launch = waves x 24 N (8N wave
        # read + 8N wave write + 8N grating or propagator read)
        kind, t_ms, n = ("row", mr.value, nr.value) if mr.value >= mc.value else ("column", mc.value, nc.value)
        plan = names[0] if kind == "row" else names[1]
        avg_s = (t_ms / max(n, 1)) / 1e3
        algo = waves * 24 * N
        achieved = algo / avg_s / 1e9
        roof = {"bound": "hbm", "kernel": f"k_{kind[:3]}_pass plan {plan} ({waves} waves)", "achieved": achieved,
                "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_source": f"{src} hbm_gbs",
                "traffic": traffic_from_profiles(kind, waves), "bytes_per_launch": algo,
                "avg_launch_us": avg_s * 1e6, "col_pass_us": 1e3 * mc.value / max(nc.value, 1),
                "row_pass_us": 1e3 * mr.value / max(nr.value, 1)}
        # the bytes the band-pruned design must move per slice of the whole step:
        # each wave's live rows (rows where the propagator is nonzero) read and
        # written once by each of the two passes, each configuration's grating
        # and the propagator read once per launch
        live = float(np.count_nonzero(np.abs(pro).max(axis=1) > 0)) / cfg["ny"]
        pruned = waves * 32 * N * live + kp * 8 * N + 8 * N
        slice_s = (ms / args.steps) / 1e3 / cfg["nobj"] * (waves / (npos_step * npass))
        roof["pruned"] = {"bytes_per_slice": pruned, "live_row_fraction": live,
                          "achieved": pruned / slice_s / 1e9, "frac": pruned / slice_s / 1e9 / hbm,
                          "note": f"one slice of {waves} waves in the timed step (all launches of the slice, "
                                  "readout planes included) against the bytes a band-pruned two-pass step must "
                                  "move; the pass rows above count 24 N per wave and pass"}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": "STEM scan row: 64 probe positions x 16 frozen-phonon passes x 200 slices, "
                                       "512x512 complex64, 3 annular detectors every 20 slices + 128x128 binned "
                                       "exit diffraction",
                           "grid": 512, "slices": cfg["nobj"], "positions_per_step": npos_step, "passes": npass,
                           "batch_waves": waves, "configurations_per_launch": kp, "parallelism": f"probe positions sharded over {world} GPU(s)",
                           "fft_plans": {"row": names[0], "column": names[1], "tuned_row_us": 1e3 * ms_r.value,
                                         "tuned_col_us": 1e3 * ms_c.value},
                           "l2": f"inputs larger than L2 (128 MiB grating pool, {2 * waves} MiB of waves per "
                                 "batch, 126 MB L2)"},
                "e2e": {"value": e2e_value, "unit": UNIT, "ms_each": [round(v, 2) for v in e2e_each],
                        "device_ms_each": [round(v, 2) for v in e2e_dev], "clocks": clk_e2e.summary(),
                        "h2d_bytes_per_step": int(h_pos.numel() * 4),
                        "d2h_bytes_per_step": int(h_int.numel() * 4 + h_bin.numel() * 4)},
                "gpu_launches": int(launches), "roofline": roof, "clocks": clk.summary(),
                "grating_generation": gen}
        if chosen_form is not None:
            line["chosen_form"] = chosen_form
        if multi is not None:
            line["multi_gpu_results"] = multi
        if tc_forms:
            line["tensor_core"] = {"forms": tc_forms,
                                   "note": "same step with the tensor-core passes (JMS_SetPrecision 1 = BF16 hi+lo, "
                                           "2 = FP16 hi+lo; readout slices keep the FP32 passes); "
                                           "col_pass_tflops counts 5 MMA products per radix stage"}
        if world == 1 and not args.no_cpu:
            try:
                gen["cpu_reference"] = reference_grating_cpu(cfg)
            except Exception as ex:
                gen["cpu_reference"] = {"value": None, "sample": f"not run: {ex}"}
            try:
                nt = host_threads()
                sample = 8 * nt
                r, dt, _ = reference_cpu(cfg, sp, probe, pro, dets, pos, nt, sample)
                line["cpu_baseline"] = {"value": r, "unit": UNIT, "cores": nt, "kind": "reference",
                                        "sample": f"{sample} probe positions x 1 phonon pass x 200 slices "
                                                  f"({dt:.1f} s, CJMultiSlice::CPUMultislice on MKL, "
                                                  "one thread per position)"}
            except Exception as ex:
                line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                                        "sample": f"not run: {ex}"}
        if world == 1 and not args.no_ref_gpu:
            try:
                line["reference_gpu"] = reference_gpu(cfg, sp, probe, pro, dets, pos, value, e2e_value)
            except Exception as ex:
                line["reference_gpu"] = {"value": None, "unit": UNIT, "note": f"not run: {type(ex).__name__}: {ex}"}
        if world == 1 and not args.no_err:
            ee = error_vs_oracle(J, cfg, sp, probe, pro, dets, pos, tc_forms=() if args.no_tc else TC_FORMS)
            ee["criterion"] = ("per detector: max |error| over positions and planes relative to the detector's "
                               f"largest signal (det_rel) and to max(largest signal, {DET_FLOOR} of the beam) "
                               "(floored, the bar the tests hold to 1e-4)")
            ee.update(subset_errors(J, cfg, sp, probe, pro, dets, pos, () if args.no_tc else TC_FORMS))
            line["err_vs_fp64"] = ee
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def measure_grating_generation(J, cfg):
    """On-device phase gratings (JMS_PgrCalculate) for the workload's specimen:
    4 slice types x 16 QEP variants of 512^2 gratings (6x6 cells, 72 / 108
    atoms per slice, Gaussian form factors, sigma 0.08 A displacements,
    2/3 band limit), written to the generator's own buffer.  Wall-clock time of
    the host calls (site linking and uploads included), after a warm-up."""
    import torch

    from jmultislicelib_b200 import synthetic as S

    nx, ny = cfg["nx"], cfg["ny"]
    a = b = cfg["ncell"] * S.A_CELL
    ff, sk = S.form_factor_tables(nx, ny, a, b, cfg["seed"], cfg["kv"])
    if J.pgr_setup(nx, ny, a, b, cfg["kv"], 2, 0, 1) or J.pgr_set_form_factors(ff, sk, [S.BISO_PHONON] * 3):
        return {"value": None, "unit": "gratings/s", "sample": "generator setup failed"}
    layers = [S.layer_atoms(cfg["ncell"], cfg["ncell"], st % 2) for st in range(cfg["nslice_types"])]

    def specimen(seed):
        for st, at in enumerate(layers):
            e, _ = J.pgr_calculate(at, S.DZ_SLICE, ngr=cfg["nvar"], seed=seed + st, want=False)
            if e:
                raise RuntimeError(f"JMS_PgrCalculate returned {e}")

    specimen(1)
    torch.cuda.synchronize()
    reps = 5
    t0 = time.perf_counter()
    for r in range(reps):
        specimen(100 * (r + 2))
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / reps
    ngr = cfg["nslice_types"] * cfg["nvar"]
    return {"value": ngr / dt, "unit": "gratings/s", "ms_per_specimen": 1e3 * dt,
            "sample": f"{ngr} gratings of {nx}x{ny} ({cfg['nslice_types']} slice types x {cfg['nvar']} QEP "
                      f"variants, {len(layers[0])}/{len(layers[1])} atoms per slice) per specimen, {reps} specimens"}


def reference_grating_cpu(cfg):
    """The reference's CJEElaSca::CalculatePhasegratingCPU (one thread, MKL)
    on slices of the same size and atom count (SrTiO3 6x6 cells: Sr + O and
    Ti + 2 O layers, Weickenmeier-Kohl form factors)."""
    from oracle import ref

    from jmultislicelib_b200 import synthetic as S

    if not ref.available():
        raise RuntimeError("oracle/_ref/libjms_ref.so is not built")
    n = cfg["ncell"]
    a = n * S.A_CELL
    total, count = 0.0, 0
    for layer in ({(38, 0.0, 0.0), (8, 0.5, 0.5)}, {(22, 0.5, 0.5), (8, 0.5, 0.0), (8, 0.0, 0.5)}):
        Z, pos = [], []
        for i in range(n):
            for j in range(n):
                for (z, fx, fy) in sorted(layer):
                    Z.append(z)
                    pos.append(((i + fx) / n, (j + fy) / n, 0.0))
        bi = np.full(len(Z), S.BISO_PHONON, np.float32)
        _, _, _, _, sec = ref.pgr(cfg["nx"], cfg["ny"], a, a, S.DZ_SLICE, cfg["kv"], Z, bi, np.ones(len(Z)), pos,
                                  thermal=2, nrep=2, seed=5)
        total += sec
        count += 2
    return {"value": count / total, "unit": "gratings/s", "cores": 1, "kind": "reference",
            "sample": f"{count} gratings of {cfg['nx']}x{cfg['ny']} (72 and 108 atoms), "
                      f"CJEElaSca::CalculatePhasegratingCPU, {total:.2f} s"}


# Uneven batch: 12 specimens cycling through 256, 384, 512, 720 and 1024 grid
# points, 50-400 slices, 1-16 phonon variants, scans of 16x16 to 64x64
# (numpy PCG64, seed 20261206); ABO3 supercells of n / 64 cells, gratings
# made on the device (JMS_PgrCalculate, QEP variants).  A step is one raster
# row of every specimen (one phonon pass), i.e. sum(nscan * nobj) multislice
# steps over all 12 grids.
UNEVEN_SEED = 20261206


def uneven_specimens():
    rng = np.random.default_rng(UNEVEN_SEED)
    out = []
    for i in range(12):
        n = (256, 384, 512, 720, 1024)[i % 5]
        out.append({"n": n, "nobj": int(rng.integers(50, 401)), "nvar": int(rng.integers(1, 17)),
                    "nscan": int(rng.choice([16, 32, 48, 64])), "ncell": n // 64})
    return out


def run_uneven(args):
    import ctypes as C

    import torch

    import jmultislicelib_b200 as jb
    from jmultislicelib_b200 import synthetic as S

    torch.cuda.set_device(0)
    J = jb.JMS()
    specs = uneven_specimens()
    ctxs, rows = [], []
    t_gen = 0.0
    for k, sp in enumerate(specs):
        cid = J.L.JMS_CreateContext()
        ctxs.append(cid)
        J.L.JMS_SelectContext(cid)
        n, nc = sp["n"], sp["ncell"]
        a = nc * S.A_CELL
        J.set_high_tension(300.0)
        J.set_grid(n, n, a, a, S.DZ_SLICE)
        pro = J.calc_propagator(S.DZ_SLICE, 0.0, 0.0, 1)
        dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in ((0, 10), (20, 50), (80, 200))]
        abrr = np.zeros(48, np.float32)
        abrr[10] = 1000.0
        probe = J.calc_probe(22.0, abrr=abrr)
        objslc = np.arange(sp["nobj"]) % 2
        assert J.setup(2, [sp["nvar"]] * 2, objslc, [0, 0], 20, 3, 1) == [0, 0, 0, 0]
        ff, sk = S.form_factor_tables(n, n, a, a, UNEVEN_SEED + k)
        assert J.pgr_setup(n, n, a, a, 300.0, 2, 0, 1) == 0
        assert J.pgr_set_form_factors(ff, sk, [S.BISO_PHONON] * 3) == 0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for s_ in range(2):
            e, _ = J.pgr_calculate(S.layer_atoms(nc, nc, s_), S.DZ_SLICE, ngr=sp["nvar"], seed=k * 10 + s_,
                                   islc=s_, ivar0=0, want=False)
            assert e == 0, e
        torch.cuda.synchronize()
        t_gen += time.perf_counter() - t0
        assert J.set_propagator(2, 0, pro) == 0
        for i, (d, m) in enumerate(dets):
            assert J.set_detector(2, i, d, m) == 0
        assert J.init_core(2) == 0
        assert J.set_incident_wave(2, probe) == 0
        J.seed(100 + k)
        J.L.JMS_SetScanBatch(64)
        mid = (nc // 2) * S.A_CELL
        pos = S.scan_positions(sp["nscan"], mid, mid, S.A_CELL)[:sp["nscan"]]   # one raster row
        d_pos = torch.from_numpy(np.ascontiguousarray(pos)).cuda()
        d_out = torch.zeros((len(pos), J.num_det_planes(), 3), dtype=torch.float64, device="cuda")
        rows.append((d_pos, d_out))
    steps = sum(sp["nscan"] * sp["nobj"] for sp in specs)

    def enqueue(k):
        J.L.JMS_SelectContext(ctxs[k])
        d_pos, d_out = rows[k]
        e = J.L.JMS_ScanGPUDevice(d_pos.shape[0], d_pos.data_ptr(), 0.0, 1, None, d_out.data_ptr(), None, 0)
        assert e == 0, e

    def sequential():
        for k in range(len(specs)):
            enqueue(k)
            torch.cuda.synchronize()

    def concurrent():
        for k in range(len(specs)):
            enqueue(k)
        torch.cuda.synchronize()

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        torch.cuda.synchronize()
        return (time.perf_counter() - t0) / reps

    reps = max(1, args.steps)
    res = {}
    for cid in ctxs:                       # fixed schedule: each length's default plan
        J.L.JMS_SelectContext(cid)
        J.L.JMS_SelectPlans(0, 0)
    res["fixed_sequential"] = timed(sequential, reps)
    tuned = {}
    for k, cid in enumerate(ctxs):         # autotuned plans per grid
        J.L.JMS_SelectContext(cid)
        ir, ic = C.c_int(0), C.c_int(0)
        assert J.L.JMS_Autotune(min(64, specs[k]["nscan"]), 10, None, None, C.byref(ir), C.byref(ic)) == 0
        buf = C.create_string_buffer(64)
        J.L.JMS_PlanName(0, buf, 64)
        tuned[specs[k]["n"]] = buf.value.decode()
    res["tuned_sequential"] = timed(sequential, reps)
    res["tuned_concurrent"] = timed(concurrent, reps)
    arr = np.array(ctxs, np.int32)
    assert J.L.JMS_GraphBegin(len(ctxs), arr.ctypes.data_as(C.POINTER(C.c_int))) == 0
    for k in range(len(specs)):
        enqueue(k)
    h = J.L.JMS_GraphEnd()
    assert h >= 1, h
    res["tuned_graph"] = timed(lambda: J.L.JMS_GraphLaunch(h, None, 1), reps)
    J.L.JMS_GraphDestroy(h)
    # all specimens in order on one stream, without a host synchronisation
    # between them, and that sequence captured once as one CUDA graph
    one = torch.cuda.Stream()
    for cid in ctxs:
        J.L.JMS_SelectContext(cid)
        J.L.JMS_SetStream(C.c_void_p(one.cuda_stream))
    res["tuned_one_stream"] = timed(concurrent, reps)
    first = np.array(ctxs[:1], np.int32)
    assert J.L.JMS_GraphBegin(1, first.ctypes.data_as(C.POINTER(C.c_int))) == 0
    for k in range(len(specs)):
        enqueue(k)
    h1 = J.L.JMS_GraphEnd()
    assert h1 >= 1, h1
    res["tuned_one_stream_graph"] = timed(lambda: J.L.JMS_GraphLaunch(h1, None, 1), reps)
    J.L.JMS_GraphDestroy(h1)
    J.L.JMS_SelectContext(0)
    for cid in ctxs:
        J.L.JMS_DestroyContext(cid)
    line = {"metric": "uneven batch multislice steps/s", "value": steps / res["tuned_one_stream_graph"],
            "unit": "steps/s",
            "n_gpus": 1, "steps": reps, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "12 specimens (256-1024 grid points, 50-400 slices, 1-16 QEP variants), "
                                   "one raster row each, one phonon pass", "specimens": specs,
                       "multislice_steps_per_step": steps, "tuned_row_plans": tuned},
            "mode_of_value": "tuned plans, the 12 specimens in order on one stream, captured once as one CUDA graph",
            "modes_steps_per_s": {k: steps / v for k, v in res.items()},
            "ms_per_step": {k: 1e3 * v for k, v in res.items()},
            "grating_generation_s": t_gen}
    print(json.dumps(line))
    return 0


# Control-variate frozen-phonon averaging on the headline scan's specimen:
# ground truth = the mean over 64 phonon configurations at an 8x8 subset of
# the 64x64 raster; estimator = 4 full configurations + the surrogate on all
# 64; surrogate trained on pairs from separate configurations and positions.
def run_cv(args):
    import torch

    import jmultislicelib_b200 as jb
    from jmultislicelib_b200 import surrogate as SG
    from jmultislicelib_b200 import synthetic as S

    torch.cuda.set_device(0)
    cfg = S.SCAN_512
    J = jb.JMS()
    t_spec = time.perf_counter()
    sp = S.make_specimen(cfg["nx"], cfg["ny"], cfg["ncell"], cfg["ncell"], cfg["nslice_types"], cfg["nvar"],
                         cfg["seed"], cfg["kv"], keep_potential=True)
    t_spec = time.perf_counter() - t_spec
    J.L.JMS_SetScanBatch(64)
    _, probe, pro, dets, raster = S.setup_library(J, cfg, specimen=sp)
    nd = J.num_det_planes()
    planes = list(range(1, nd))                 # the 10 readout thicknesses after the entrance plane
    nout = len(planes) * len(dets)
    cell0 = (cfg["ncell"] // 2) * S.A_CELL
    rng = np.random.default_rng(20261207)

    def configs(n):
        """n phonon configurations: a random variant of its structure slice per object slice."""
        return rng.integers(0, cfg["nvar"], (n, cfg["nobj"])).astype(np.int32)

    # training pairs: separate configurations and random positions in the scanned cell
    tr_cfg = configs(args.cv_train_configs)
    tr_pos = (cell0 + rng.uniform(0, S.A_CELL, (args.cv_train_positions, 2))).astype(np.float32)
    d_tr = torch.from_numpy(tr_pos).cuda()
    # surrogate input: one channel per readout interval of the depth, a 64 x 64-
    # pixel window around the probe averaged to 16 x 16
    nbins, pool = args.cv_bins, args.cv_pool
    size = SG.PATCH // pool
    X, Y = [], []
    t_gen = 0.0
    tr_patches = SG.DevicePatches(sp, cfg["nobj"], cfg["nslice_types"], tr_pos, nbins, pool=pool)
    for v in tr_cfg:
        X.append(tr_patches(v)[0].cpu().numpy())
        y, dt = SG.timed(lambda: SG.signals(J, d_tr, len(tr_pos), v, planes))
        Y.append(y)
        t_gen += dt
    # the surrogate learns the phonon fluctuation at a fixed position: inputs
    # and targets are deviations from their mean over the configurations
    X = np.stack(X)                    # [config, position, nbins, size, size]
    Y = np.stack(Y)                    # [config, position, nout]
    X -= X.mean(axis=0, keepdims=True)
    Y -= Y.mean(axis=0, keepdims=True)
    nval = max(2, len(tr_cfg) // 8)    # held-out configurations: early stopping and beta
    Xt, Yt = X[nval:].reshape(-1, *X.shape[2:]), Y[nval:].reshape(-1, nout)
    Xv, Yv = X[:nval].reshape(-1, *X.shape[2:]), Y[:nval].reshape(-1, nout)
    cv = SG.ControlVariate(nout, batch=256, seed=1, cin=nbins, size=size, relu=args.cv_relu)
    hist, t_train = SG.timed(lambda: cv.fit(Xt, Yt, Xv, Yv, epochs=args.cv_epochs))
    # evaluation: 8x8 subset of the raster, 64 fresh configurations
    ev_pos = np.ascontiguousarray(raster.reshape(64, 64, 2)[::8, ::8].reshape(-1, 2))
    d_ev = torch.from_numpy(ev_pos).cuda()
    ev_cfg = configs(64)
    F = np.zeros((64, len(ev_pos), nout))
    G = np.zeros_like(F)
    P = np.zeros((64, len(ev_pos), nbins, size, size), np.float32)
    t_full = t_sur = t_patch = 0.0
    for k, v in enumerate(ev_cfg):
        F[k], dt = SG.timed(lambda: SG.signals(J, d_ev, len(ev_pos), v, planes))
        t_full += dt
    ev_patches = SG.DevicePatches(sp, cfg["nobj"], cfg["nslice_types"], ev_pos, nbins, pool=pool)
    Pd, t_patch = SG.timed(lambda: ev_patches(ev_cfg))          # all 64 configurations in one launch
    P[:] = Pd.cpu().numpy()
    P -= P.mean(axis=0, keepdims=True)
    G, t_sur = SG.timed(lambda: cv.predict(P.reshape(-1, *P.shape[2:])).reshape(F.shape))
    truth = F.mean(axis=0)
    n_few = 4
    plain = F[:n_few].mean(axis=0)
    est = SG.cv_estimate(F[:n_few], G[:n_few], G, cv.beta)
    scale = np.abs(truth).mean(axis=0)[None, :]
    e_plain = np.sqrt((((plain - truth) / scale) ** 2).mean(axis=0)).reshape(len(planes), len(dets))
    e_cv = np.sqrt((((est - truth) / scale) ** 2).mean(axis=0)).reshape(len(planes), len(dets))
    var_f = F.var(axis=0).mean(axis=0)
    var_r = (F - cv.beta * G).var(axis=0).mean(axis=0)
    ratio = (var_r / np.maximum(var_f, 1e-300)).reshape(len(planes), len(dets))
    line = {"metric": "control-variate frozen-phonon estimate", "unit": "relative RMS error", "n_gpus": 1,
            "data": "synthetic",
            "config": {"workload": "512^2 scan specimen, 8x8 positions, 64 phonon configurations as ground truth, "
                                   "estimator 4 full + surrogate on 64",
                       "input": f"{nbins} depth bins x {size} x {size} (64 x 64-pixel window averaged "
                                f"{pool} x {pool})", "relu": bool(args.cv_relu),
                       "train_configs": int(args.cv_train_configs),
                       "train_pairs": int(Xt.shape[0]), "validation_pairs": int(Xv.shape[0]),
                       "epochs": args.cv_epochs, "outputs": nout},
            "err_plain4_per_det": [float(v) for v in e_plain.mean(axis=0)],
            "err_cv4_per_det": [float(v) for v in e_cv.mean(axis=0)],
            "var_ratio_per_det": [float(v) for v in ratio.mean(axis=0)],
            "var_ratio_by_thickness": ratio.tolist(),
            "plain_configs_for_same_error": [float(n_few * (a / max(b, 1e-30)) ** 2)
                                             for a, b in zip(e_plain.mean(axis=0), e_cv.mean(axis=0))],
            "loss_train_val_first_last": [hist[0], hist[-1]], "beta_mean": float(np.mean(cv.beta)),
            "seconds": {"specimen_potentials": t_spec, "training_signals": t_gen, "training": t_train,
                        "full_multislice_64": t_full, "full_multislice_4": t_full * n_few / 64,
                        "surrogate_inference_64": t_sur, "patch_inputs_64_device": t_patch}}
    print(json.dumps(line))
    return 0


# The headline scan in the quantum-excitation-of-phonons form: every phonon
# pass gets its own configuration, i.e. 200 freshly displaced gratings (one
# per object slice) made on the device, instead of draws from a fixed pool
# of 16 variants per slice type.  The grating store holds one slot per object
# slice (variant k of type s = the k-th object slice of that type).
def run_qep(args):
    import ctypes as C

    import torch

    import jmultislicelib_b200 as jb
    from jmultislicelib_b200 import synthetic as S

    torch.cuda.set_device(0)
    cfg = dict(S.SCAN_512)
    J = jb.JMS()
    stream = torch.cuda.Stream(priority=-1)        # scans; grating generation runs on a lower-priority stream
    J.set_stream(stream.cuda_stream)
    J.L.JMS_SetScanBatch(args.batch)
    nobj, nst = cfg["nobj"], cfg["nslice_types"]
    objslc = np.arange(nobj) % nst
    count = [int((objslc == s_).sum()) for s_ in range(nst)]
    rank = np.zeros(nobj, np.int32)
    for s_ in range(nst):
        rank[objslc == s_] = np.arange(count[s_])
    nx, ny, nc = cfg["nx"], cfg["ny"], cfg["ncell"]
    a = nc * S.A_CELL
    J.cleanup()
    J.set_high_tension(cfg["kv"])
    J.set_grid(nx, ny, a, a, S.DZ_SLICE)
    pro = J.calc_propagator(S.DZ_SLICE, 0.0, 0.0, cfg["ntype"])
    dets = [J.calc_ring_detector(b0, b1) for (b0, b1) in cfg["dets"]]
    abrr = np.zeros(48, np.float32)
    abrr[10] = cfg["cs"]
    probe = J.calc_probe(cfg["alpha"], abrr=abrr)
    # the grating store holds every configuration of a step, twice (two halves
    # that alternate between steps): structure slice s has count[s] x nconf x 2
    # variants, variant (h nconf + k) count[s] + r being the r-th object slice
    # of type s in configuration k of half h
    nconf, nhalf = cfg["nvar"], 2
    assert J.setup(2, [c * nconf * nhalf for c in count], objslc, [0] * nst, cfg["ndetper"], len(dets),
                   1) == [0, 0, 0, 0]
    assert J.set_propagator(2, 0, pro) == 0
    for i, (d, m) in enumerate(dets):
        assert J.set_detector(2, i, d, m) == 0
    assert J.init_core(2) == 0
    assert J.set_incident_wave(2, probe) == 0
    ff, sk = S.form_factor_tables(nx, ny, a, a, cfg["seed"], cfg["kv"])
    assert J.pgr_setup(nx, ny, a, a, cfg["kv"], 2, 0, 1) == 0
    assert J.pgr_set_form_factors(ff, sk, [S.BISO_PHONON] * 3) == 0
    layers = [S.layer_atoms(nc, nc, s_ % 2) for s_ in range(nst)]
    mid = (nc // 2) * S.A_CELL
    pos = S.scan_positions(cfg["nscan"], mid, mid, S.A_CELL)
    npos = cfg["nscan"]
    d_pos = torch.from_numpy(pos[:npos].copy()).cuda()
    d_int = torch.zeros((npos, J.num_det_planes(), len(dets)), dtype=torch.float64, device="cuda")
    # FFT plan choice by the library's autotuner, for launches of the fused
    # configurations (outside the timed region)
    ir, ic = C.c_int(0), C.c_int(0)
    assert J.L.JMS_Autotune(min(args.batch, npos * nconf), 20, None, None, C.byref(ir), C.byref(ic)) == 0
    cnt = np.asarray(count, np.int32)[objslc]
    vs = [np.ascontiguousarray(np.stack([(h * nconf + k) * cnt + rank for k in range(nconf)]), np.int32)
          for h in range(nhalf)]
    gstream = torch.cuda.Stream(priority=0)        # generation; the scan stream has the higher priority

    def generate(k):
        # nconf fresh configurations of step k (count[s] new gratings per slice type each) into half k % 2
        h = k % nhalf
        for p in range(nconf):
            for s_ in range(nst):
                e, _ = J.pgr_calculate(layers[s_], S.DZ_SLICE, ngr=count[s_], seed=(1000 * k + p) * 16 + s_,
                                       islc=s_, ivar0=(h * nconf + p) * count[s_], want=False)
                assert e == 0, e

    def scan(k):
        # one scan over the nconf configurations of step k (their waves share the launches)
        v = vs[k % nhalf]
        e = J.L.JMS_ScanGPUDevice(npos, d_pos.data_ptr(), 0.0, nconf, v.ctypes.data_as(C.POINTER(C.c_int)),
                                  d_int.data_ptr(), None, 0)
        assert e == 0, e

    def serial(k0, n, evs):
        # generation and scan of each step in turn on the scan stream
        J.pgr_set_stream(0)
        for k in range(k0, k0 + n):
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            generate(k)
            e1.record(stream)
            scan(k)
            e2.record(stream)
            evs.append((e0, e1, e2))

    def overlapped(k0, n):
        # generation of step k + 1 (generator stream) runs during the scan of
        # step k (scan stream): a scan waits for its gratings, a generation
        # for the scan that last read its half
        J.pgr_set_stream(gstream.cuda_stream)
        gstream.wait_stream(stream)
        ev_gen, ev_scan = {}, {}
        with torch.cuda.stream(gstream):
            generate(k0)
        ev_gen[k0] = torch.cuda.Event()
        ev_gen[k0].record(gstream)
        for k in range(k0, k0 + n):
            if k + 1 < k0 + n:
                if k - 1 in ev_scan:
                    gstream.wait_event(ev_scan[k - 1])
                with torch.cuda.stream(gstream):
                    generate(k + 1)
                ev_gen[k + 1] = torch.cuda.Event()
                ev_gen[k + 1].record(gstream)
            stream.wait_event(ev_gen[k])
            scan(k)
            ev_scan[k] = torch.cuda.Event()
            ev_scan[k].record(stream)
        J.pgr_set_stream(0)

    def timed(fn, k0, *extra):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(0) as clk:
            with torch.cuda.stream(stream):
                ev0.record(stream)
                fn(k0, args.steps, *extra)
                ev1.record(stream)
            torch.cuda.synchronize()
        return ev0.elapsed_time(ev1), clk.summary()

    with torch.cuda.stream(stream):
        serial(0, args.warmup, [])
        overlapped(args.warmup, args.warmup)
    torch.cuda.synchronize()
    all_ev = []
    ms_serial, _ = timed(serial, 2 * args.warmup, all_ev)
    ms, clocks = timed(overlapped, 2 * args.warmup + args.steps)
    gen_ms = sum(a.elapsed_time(b) for a, b, _ in all_ev)
    scan_ms = sum(b.elapsed_time(c) for _, b, c in all_ev)
    steps_per = npos * cfg["nvar"] * nobj
    line = {"metric": "multislice steps/s (512² wave), fresh QEP gratings every pass", "unit": "steps/s",
            "value": args.steps * steps_per / (ms / 1e3), "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "STEM scan row: 64 positions x 16 phonon passes x 200 slices, 512x512; every "
                                   "pass a new QEP configuration: 200 gratings generated on the device "
                                   "(sigma 0.08 A, Gaussian form factors, 2/3 band limit); the 16 configurations "
                                   "of a step (3,200 gratings) are generated into one half of a double grating "
                                   "store while the previous step's half is scanned (generator stream of its own, "
                                   "JMS_PgrSetStream; the scan stream has the higher priority)",
                       "batch_waves": min(args.batch, 64 * nconf)},
            "serial": {"value": args.steps * steps_per / (ms_serial / 1e3), "ms_per_step": ms_serial / args.steps,
                       "grating_generation_share": gen_ms / ms_serial,
                       "scan_only_steps_per_s": args.steps * steps_per / (scan_ms / 1e3),
                       "note": "generation, then scan, on one stream"},
            "clocks": clocks}
    print(json.dumps(line))
    return 0


def coarse_grid(cfg, beta_mrad, lengths=(128, 160, 192, 240, 256, 320, 384)):
    """Smallest supported grid length whose 2/3 band limit reaches beta_mrad
    (same supercell): 2/3 * n / (2 a) * lambda >= beta."""
    from jmultislicelib_b200 import synthetic as S

    a = cfg["ncell"] * S.A_CELL                             # nm
    v = cfg["kv"] * 1e3
    lam = 1.2264262862 / np.sqrt(v * (1.0 + 9.7847538e-7 * v))   # relativistic electron wavelength, nm
    for n in lengths:
        if (2.0 / 3.0) * n / (2.0 * a) * lam * 1e3 >= beta_mrad:
            return n
    return cfg["nx"]


def measure_multifidelity(J, cfg, stream, d_pos, npos_step, rows, warmup, n_low=None, group=4):
    """The chosen form of the scan (JMS_ScanMultiFidelityDevice) against the plain
    one on the same raster rows and the same 16 phonon configurations: plain =
    16 full-grid passes per position; chosen = 1 full-grid pass + 16 passes on a
    n_low^2 grid of the same specimen (control variate, coefficient 1), n_low
    the coarsest grid among the candidates whose band limit covers the 20-50 mrad
    detector (192 at 300 kV on the 23.43 A cell: 54 mrad; 180 would reach
    50.4 mrad, but its 12 x 15 line plan runs 1.6x slower per point, so the
    chosen form took 100.6 ms per raster row with it against 77.8 with 192).  The chosen form takes
    `group` raster rows per call, so that the coarse grid's launches carry
    group x 64 waves (its 192^2 waves are small); the plain form takes one row
    per call (64 waves of 512^2 already fill a launch).  Times per raster row
    with CUDA events (inputs on the device) and the relative difference of the
    estimate from the plain average, per detector."""
    if n_low is None:
        n_low = coarse_grid(cfg, cfg["dets"][1][1])
    rows = group * ((rows + group - 1) // group)
    import ctypes as C

    import torch

    from jmultislicelib_b200 import synthetic as S

    npass = cfg["nvar"]
    varseq = np.random.default_rng(20261209).integers(0, cfg["nvar"], (npass, cfg["nobj"])).astype(np.int32)
    vs = varseq.ctypes.data_as(C.POINTER(C.c_int))
    lo = J.L.JMS_CreateContext()
    try:
        J.L.JMS_SelectContext(lo)
        c_lo = dict(cfg, nx=n_low, ny=n_low)
        sp_lo = S.make_specimen(n_low, n_low, c_lo["ncell"], c_lo["ncell"], c_lo["nslice_types"], c_lo["nvar"],
                                c_lo["seed"], c_lo["kv"])
        S.setup_library(J, c_lo, specimen=sp_lo)
        J.L.JMS_SetScanBatch(1024)          # 4 configurations x 256 positions per coarse launch
        J.L.JMS_SelectContext(0)
        nd, ndet = J.L.GetDetetionSliceNum(), J.L.GetDetNum()
        dev = d_pos.device
        o_plain = torch.zeros((rows, npos_step, nd, ndet), dtype=torch.float64, device=dev)
        o_cv = torch.zeros_like(o_plain)

        def plain(r):
            p = d_pos[r * npos_step:(r + 1) * npos_step]
            e = J.L.JMS_ScanGPUDevice(npos_step, p.data_ptr(), 0.0, npass, vs, o_plain[r].data_ptr(), None, 0)
            if e:
                raise RuntimeError(f"JMS_ScanGPUDevice returned {e}")

        def chosen(r):
            # rows r .. r + group - 1 in one call (r a multiple of group)
            if r % group:
                return
            n = group * npos_step
            p = d_pos[r * npos_step:r * npos_step + n]
            e = J.L.JMS_ScanMultiFidelityDevice(0, lo, n, p.data_ptr(), 0.0, npass, vs, o_cv[r].data_ptr())
            if e:
                raise RuntimeError(f"JMS_ScanMultiFidelityDevice returned {e}")

        res = {}
        for name, fn in (("plain", plain), ("chosen", chosen)):
            with torch.cuda.stream(stream):
                for k in range(warmup):
                    fn((k * group) % rows)
            torch.cuda.synchronize()
            if name == "plain":
                o_plain.zero_()        # the plain scan accumulates into its output
                torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                e0.record(stream)
                for r in range(rows):
                    fn(r)
                e1.record(stream)      # the full-grid stream waits for the coarse one inside each chosen call
            torch.cuda.synchronize()
            res[name] = e0.elapsed_time(e1) / rows
        truth = o_plain.cpu().numpy()
        est = o_cv.cpu().numpy()
        big = np.abs(truth).max(axis=(0, 1, 2))
        err = np.abs(est - truth).max(axis=(0, 1, 2)) / np.maximum(big, 1e-300)
        return {"form": f"control variate: 1 pass on the 512^2 grid + {npass} passes on {n_low}^2 (coefficient 1), "
                        f"JMS_ScanMultiFidelityDevice",
                "plain_form": f"{npass} passes on the 512^2 grid (JMS_ScanGPUDevice, same configurations)",
                "ms_per_row": res["chosen"], "plain_ms_per_row": res["plain"],
                "speedup_vs_plain": res["plain"] / res["chosen"],
                "scan_s": 64 * res["chosen"] / 1e3, "plain_scan_s": 64 * res["plain"] / 1e3,
                "rows_timed": rows, "rows_per_chosen_call": group,
                "err_vs_plain_per_det": [float(x) for x in err],
                "note": "error relative to each detector's largest signal; the 80-200 mrad detector lies outside "
                        f"the {n_low}^2 band limit, so its estimate is the single full pass (its signal is 2e-10 "
                        "of the beam, below the FP32 noise of every form)"}
    finally:
        J.L.JMS_SelectContext(0)
        J.L.JMS_DestroyContext(lo)


def traffic_from_profiles(kind, waves):
    """DRAM bytes per launch of the pass with `waves` waves, from the committed
    ncu summary (line "traffic_bytes_per_launch_<waves>_waves: <bytes>")."""
    p = os.path.join(ROOT, "profiles", f"{kind}_pass_512.md")
    try:
        for line in open(p):
            if line.startswith(f"traffic_bytes_per_launch_{waves}_waves:"):
                return float(line.split(":")[1])
    except Exception:
        pass
    return None


def error_vs_oracle(J, cfg, sp, probe, pro, dets, pos, tc_forms=()):
    """Relative error of the integrated detector signals of one probe position
    (one phonon pass, 200 slices) against the FP64 oracle, per detector (max
    over the 11 readout planes, relative to that detector's largest signal),
    next to the error of the reference's own FP32 CPU path on the same input
    and of the tensor-core forms tc_forms ((JMS_SetPrecision mode, name), ...)."""
    try:
        from oracle import oracle as OR
    except Exception as ex:
        return {"det_rel": None, "sample": f"oracle unavailable: {ex}"}
    objslc = np.arange(cfg["nobj"]) % cfg["nslice_types"]
    nvar = [cfg["nvar"]] * cfg["nslice_types"]
    var = OR.Rng(99).variant_sequence(nvar, objslc)
    p = pos[len(pos) // 2:len(pos) // 2 + 1]
    e, out, _ = J.scan(p, 1, varseq=var[None, :])
    assert e == 0
    n, hsh = OR.detection_planes(cfg["ndetper"], cfg["nobj"])
    wl = J.L.GetWaveLength()
    w0 = OR.offset(probe, sp.a, sp.b, wl, float(p[0, 0]), float(p[0, 1]))
    res = OR.multislice(w0, np.concatenate(sp.gratings), objslc * cfg["nvar"] + var, pro[None],
                        np.zeros(cfg["nobj"], np.int32), hsh, n, det=np.stack([d for d, _ in dets]),
                        masks=[m for _, m in dets], imagedet=1)
    ref_fp64 = res["det_int"]
    den = np.maximum(np.abs(ref_fp64).max(axis=0), 1e-300)

    def rel(x):
        return [float(v) for v in np.abs(x - ref_fp64).max(axis=0) / den]

    tc_rel = {}
    for mode, form in tc_forms:
        J.set_precision(mode)
        e, out_tc, _ = J.scan(p, 1, varseq=var[None, :])
        J.set_precision(0)
        tc_rel[form] = rel(out_tc[0]) if e == 0 else f"scan returned {e}"
    out_d = {"det_rel": rel(out[0]), "abs_vs_beam": float(np.abs(out[0] - ref_fp64).max()),
             "signal_max": [float(v) for v in np.abs(ref_fp64).max(axis=0)],
             "sample": "1 position x 1 phonon pass x 200 slices, 11 planes x 3 detectors; "
                       "det_rel per detector (0-10, 20-50, 80-200 mrad)"}
    try:  # the reference's own FP32 path (CPUMultislice on MKL) on the same input and variants
        from oracle import ref
        R = ref.RefJMS()
        R.set_high_tension(cfg["kv"])
        R.set_grid(cfg["nx"], cfg["ny"], sp.a, sp.b, 0.19525)
        R.setup(ref.CODE_CPU, nvar, objslc, [0] * cfg["nslice_types"], cfg["ndetper"], len(dets), 1, 1)
        for s_, gr in enumerate(sp.gratings):
            R.set_phase_grating(ref.CODE_CPU, s_, gr)
        R.set_propagator(ref.CODE_CPU, 0, pro)
        for i, (d, m) in enumerate(dets):
            R.set_detector(ref.CODE_CPU, i, d, m)
        R.init_core(ref.CODE_CPU, 1)
        R.set_incident_wave(ref.CODE_CPU, probe)
        R.seed(99)
        R.offset(ref.CODE_CPU, float(p[0, 0]), float(p[0, 1]), 0.0)
        R.cpu_multislice(0, 0, 1.0, 0)
        rd = R.get_result(ref.CODE_CPU, 1, n * len(dets)).reshape(n, len(dets))
        R.close()
        out_d["reference_fp32_det_rel"] = rel(rd)
    except Exception as ex:
        out_d["reference_fp32_det_rel"] = f"not run: {ex}"
    if tc_rel:
        out_d["tensor_core_det_rel"] = tc_rel
    return out_d


def multirank_results(J, cfg, d_pos, npos_step, bin_, nby, nbx, stream, rank, world):
    """The result path of a sharded scan (N > 1 ranks): every rank scans its
    raster rows of a small scan (2 rows per rank, 2 fixed phonon
    configurations, JMS_ScanGPUDevice), the integrated detectors of all rows
    are all-gathered and the binned exit patterns summed over ranks with an
    all-reduce (the position-averaged pattern), both over NCCL.  Rank 0 reruns
    the last rank's rows and reports the largest difference from the gathered
    copy, and the all-reduced pattern against the sum of the gathered partial
    patterns."""
    import ctypes as C

    import torch

    from jmultislicelib_b200 import shard

    nd, ndet = J.L.GetDetetionSliceNum(), J.L.GetDetNum()
    varseq = np.ascontiguousarray(np.random.default_rng(4243).integers(0, cfg["nvar"], (2, cfg["nobj"])), np.int32)
    vs = varseq.ctypes.data_as(C.POINTER(C.c_int))
    dev = d_pos.device
    d_o = torch.zeros((npos_step, nd, ndet), dtype=torch.float64, device=dev)
    d_b = torch.zeros((npos_step, nby, nbx), dtype=torch.float32, device=dev)

    def scan_row(r):
        with torch.cuda.stream(stream):
            d_o.zero_()
            d_b.zero_()
            p = d_pos[r * npos_step:(r + 1) * npos_step]
            e = J.L.JMS_ScanGPUDevice(npos_step, p.data_ptr(), 0.0, 2, vs, d_o.data_ptr(), d_b.data_ptr(), bin_)
        torch.cuda.synchronize()
        if e:
            raise RuntimeError(f"JMS_ScanGPUDevice returned {e}")
        return d_o.cpu().numpy(), d_b.sum(dim=0).double().cpu().numpy()

    _, _, rep = shard.check_sharded_scan(scan_row, rank, world, rows_each=2)
    rep["workload"] = (f"{2 * world} raster rows x {npos_step} positions x 2 phonon configurations; gather of "
                       f"[row][{npos_step}][{nd}][{ndet}] float64 and all-reduce of the summed {nby}x{nbx} "
                       "binned exit patterns over NCCL")
    return rep


# 4 x 4 subset of the 64 x 64 raster pinned to the FP64 oracle: raster rows and
# columns 8, 24, 40 and 56
SUBSET_IDX = [iy * 64 + ix for iy in (8, 24, 40, 56) for ix in (8, 24, 40, 56)]
DET_FLOOR = 1e-3   # of the beam intensity (the probe is normalised to 1)


def _err_metrics(got, truth):
    """Per detector: max |got - truth| over positions and planes, relative to
    the detector's largest signal (det_rel) and to max(largest signal,
    DET_FLOOR) (floored), with the absolute error and the largest signal."""
    ax = tuple(range(truth.ndim - 1))
    d = np.abs(got - truth).max(axis=ax)
    big = np.abs(truth).max(axis=ax)
    return {"det_rel": [float(x) for x in d / np.maximum(big, 1e-300)],
            "floored": [float(x) for x in d / np.maximum(big, DET_FLOOR)],
            "abs": [float(x) for x in d], "signal_max": [float(x) for x in big]}


def coarse_context(J, cfg, n_low, specimen_kw=None):
    """A library context holding the workload's specimen on an n_low^2 grid of
    the same supercell (the coarse grid of the chosen form); returns its id,
    with context 0 selected again."""
    from jmultislicelib_b200 import synthetic as S

    lo = J.L.JMS_CreateContext()
    J.L.JMS_SelectContext(lo)
    c_lo = dict(cfg, nx=n_low, ny=n_low)
    sp_lo = S.make_specimen(n_low, n_low, c_lo["ncell"], c_lo["ncell"], c_lo["nslice_types"], c_lo["nvar"],
                            c_lo["seed"], c_lo["kv"], **(specimen_kw or {}))
    S.setup_library(J, c_lo, specimen=sp_lo)
    J.L.JMS_SetScanBatch(1024)
    J.L.JMS_SelectContext(0)
    return lo


def fp64_subset(J, ctx, lo, cfg, sp, probe, pro, dets, pos, tc_forms=(), threads=None, seed=99):
    """The headline scan as benched, pinned to the FP64 oracle on the 4 x 4
    position subset.  One call scans 64 positions (the 16 subset positions and
    48 others of the raster) x 16 frozen-phonon configurations, i.e. the
    benched 1024-wave launches, through JMS_ScanGPU on context ctx.  The 16
    configurations alternate two variant sequences drawn as GPUMultislice draws
    them (c0, c1, c0, c1, ...), so the scan's 16-configuration average equals
    the 2-configuration average that the FP64 oracle computes for each subset
    position (32 oracle runs of 200 slices, in a thread pool).  The chosen form
    (JMS_ScanMultiFidelity, coarse context lo) and the tensor-core forms run on
    the same positions and configurations."""
    import concurrent.futures as cf
    import ctypes as C

    from oracle import oracle as OR

    nobj, nt, nvar = cfg["nobj"], cfg["nslice_types"], cfg["nvar"]
    objslc = np.arange(nobj) % nt
    rng = OR.Rng(seed)
    v = [rng.variant_sequence([nvar] * nt, objslc) for _ in range(2)]
    npass = nvar
    varseq = np.ascontiguousarray(np.stack([v[k % 2] for k in range(npass)]), np.int32)
    rest = [i for i in range(32 * 64, 33 * 64) if i not in SUBSET_IDX][:48]
    p64 = np.ascontiguousarray(np.concatenate([pos[SUBSET_IDX], pos[rest]]), np.float32)
    t0 = time.perf_counter()
    J.L.JMS_SelectContext(ctx)
    try:
        e, out, _ = J.scan(p64, npass, varseq=varseq)
        assert e == 0, e
        forms = {"plain": out[:16]}
        for mode, form in tc_forms:
            J.set_precision(mode)
            e, o_tc, _ = J.scan(p64, npass, varseq=varseq)
            J.set_precision(0)
            forms[form] = o_tc[:16] if e == 0 else None
        nd, ndet = J.L.GetDetetionSliceNum(), J.L.GetDetNum()
    finally:
        J.L.JMS_SelectContext(0)
    if lo is not None:
        o_cv = np.zeros((64, nd, ndet), np.float32)
        fp = C.POINTER(C.c_float)
        e = J.L.JMS_ScanMultiFidelity(ctx, lo, 64, p64.ctypes.data_as(fp), 0.0, npass,
                                      varseq.ctypes.data_as(C.POINTER(C.c_int)), o_cv.ctypes.data_as(fp))
        forms["chosen"] = o_cv[:16] if e == 0 else None
    t_gpu = time.perf_counter() - t0
    n, hsh = OR.detection_planes(cfg["ndetper"], nobj)
    wl = J.L.GetWaveLength()
    pool_ = np.concatenate(sp.gratings)
    detf = np.stack([d for d, _ in dets])
    masks = [m for _, m in dets]

    def job(pk):
        p, k = pk
        w0 = OR.offset(probe, sp.a, sp.b, wl, float(p64[p, 0]), float(p64[p, 1]))
        res = OR.multislice(w0, pool_, (objslc * nvar + v[k]).astype(np.int32), pro[None],
                            np.zeros(nobj, np.int32), hsh, n, det=detf, masks=masks, imagedet=1)
        return p, k, res["det_int"]

    t0 = time.perf_counter()
    truth = np.zeros((16, n, len(dets)))
    nthr = threads or host_threads()
    with cf.ThreadPoolExecutor(max(1, min(32, nthr))) as ex:
        for p, k, d in ex.map(job, [(p, k) for p in range(16) for k in range(2)]):
            truth[p] += 0.5 * d
    t_or = time.perf_counter() - t0
    res = {name: (_err_metrics(o.astype(np.float64), truth) if o is not None else "scan failed")
           for name, o in forms.items()}
    res["sample"] = (f"4x4 subset of the 64x64 raster (rows/columns 8, 24, 40, 56) scanned within 64-position calls x "
                     f"{npass} configurations (1024-wave launches); the configurations alternate two variant "
                     f"sequences, so the FP64 oracle's 2-configuration average is the exact target; "
                     f"{nobj} slices, {n} planes x {len(dets)} detectors; oracle {t_or:.1f} s on {nthr} threads, "
                     f"GPU legs {t_gpu:.1f} s")
    return res


# strongly scattering variant of the headline cell: atoms 300x stronger and
# half as wide (Gaussian widths 0.05-0.2 A, amplitudes 150-1500 V A), so that
# the 80-200 mrad detector collects 1-3 % of the beam at the exit plane
STRONG = dict(amp_scale=300.0, wid_scale=0.5)


def subset_errors(J, cfg, sp, probe, pro, dets, pos, tc_forms=()):
    """fp64_subset on the headline specimen (plain, chosen and tensor-core
    forms) and on its strongly scattering variant STRONG (plain and chosen)."""
    from jmultislicelib_b200 import synthetic as S

    out = {}
    n_low = coarse_grid(cfg, cfg["dets"][1][1])
    lo = coarse_context(J, cfg, n_low)
    try:
        out["subset_4x4"] = fp64_subset(J, 0, lo, cfg, sp, probe, pro, dets, pos, tc_forms)
    except Exception as ex:
        out["subset_4x4"] = f"not run: {ex}"
    finally:
        J.L.JMS_DestroyContext(lo)
    st = J.L.JMS_CreateContext()
    lo_st = None
    try:
        J.L.JMS_SelectContext(st)
        sp_st = S.make_specimen(cfg["nx"], cfg["ny"], cfg["ncell"], cfg["ncell"], cfg["nslice_types"], cfg["nvar"],
                                cfg["seed"], cfg["kv"], **STRONG)
        _, probe_st, pro_st, dets_st, _ = S.setup_library(J, cfg, specimen=sp_st)
        J.L.JMS_SetScanBatch(1024)
        J.L.JMS_SelectContext(0)
        lo_st = coarse_context(J, cfg, n_low, STRONG)
        r = fp64_subset(J, st, lo_st, cfg, sp_st, probe_st, pro_st, dets_st, pos)
        r["specimen"] = (f"headline cell with atom amplitudes x{STRONG['amp_scale']:g} and widths "
                         f"x{STRONG['wid_scale']:g} (same sites and phonon draws)")
        out["strong_subset_4x4"] = r
    except Exception as ex:
        out["strong_subset_4x4"] = f"not run: {ex}"
    finally:
        J.L.JMS_SelectContext(0)
        if lo_st is not None:
            J.L.JMS_DestroyContext(lo_st)
        J.L.JMS_DestroyContext(st)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=1024,
                    help="waves per launch; above the 64 positions of a row, 16 phonon configurations share a launch")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip timing the reference's own GPU path")
    ap.add_argument("--no-err", action="store_true")
    ap.add_argument("--no-tc", action="store_true", help="skip the tensor-core forms beside the headline")
    ap.add_argument("--no-chosen", action="store_true", help="skip the chosen (multi-fidelity) form of the scan")
    ap.add_argument("--workload", default="scan", choices=["scan", "uneven", "cv", "qep"],
                    help="scan: the headline 512^2 scan; uneven: 12 specimens of uneven grid sizes; "
                         "cv: control-variate frozen-phonon averaging with the learned surrogate; "
                         "qep: the headline scan with fresh QEP gratings generated on the device every pass")
    ap.add_argument("--cv-train-configs", type=int, default=32)
    ap.add_argument("--cv-train-positions", type=int, default=625)
    ap.add_argument("--cv-epochs", type=int, default=30)
    ap.add_argument("--cv-bins", type=int, default=10, help="depth bins (input channels) of the surrogate")
    ap.add_argument("--cv-pool", type=int, default=4, help="pixel blocks averaged in the surrogate's input")
    ap.add_argument("--cv-relu", action="store_true",
                    help="surrogate convolutions with ReLU (default: a linear convolutional network)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.workload == "uneven":
        return run_uneven(args)
    if args.workload == "cv":
        return run_cv(args)
    if args.workload == "qep":
        return run_qep(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
