"""Benchmark: Born forward + adjoint (the FWI gradient kernel pair) of the
elastic engine on the 600x1800 grid, nts=4000, 10 shots, one B200 per rank.

One step = Born forward of every shot followed by the Born adjoint of every
shot (image accumulated over shots) = 4 propagations per shot.
Metric: cell-updates per second over the whole job (Gcell-updates/s).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value : device-resident inputs (single-shot *_reg_dev C entry points)
e2e   : the reference-facing operator API (BornElasticShotsGpu.forward /
        adjoint) with host buffers, host<->device copies inside the region
reference arm (--impl reference): the reference's own CUDA drivers
        (oracle/_ref, compiled from the reference tree for sm_100a), one shot
        of the same workload per step.
Shots are independent, so N > 1 ranks each take their own shots (weak
scaling) and the image is summed with one all-reduce per step, the exchange
the reference does on the host (BornElasticShotsGpu.cpp:313-323).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

BYTES_PER_CELL = 80.0    # read 5 current + 5 old + 5 medium, write 5 new (FP32)
PAIR_BYTES_PER_CELL = 100.0   # two steps per launch: read 5 current + 5 old + 5 medium, write 2 x 5 new


def born_pair_bytes(cells, fine_steps, nts):
    """Algorithmic bytes of one shot's Born forward + adjoint (FP32 source
    history, two fine steps per coarse sample): the four propagations (source
    wavefield in both calls, scattered wavefield, adjoint wavefield) at 80 B
    per cell update, plus per coarse sample and cell the history written twice
    (Vx, Vz: 2 x 8 B), the forward imaging (3 history samples 24 B, the
    perturbation 20 B, the secondary sources written 20 B), the scattered steps
    reading the secondary sources (3 x 20 B: the left sample on both fine
    steps, the right one on the second), and the adjoint imaging (3 history
    samples 24 B, read-modify-write of the five images 40 B)."""
    return cells * (4 * BYTES_PER_CELL * fine_steps + (16 + 64 + 60 + 64) * nts)


def shot_gradient_bytes(cells, fine_steps, nts, propagations=2):
    """Algorithmic bytes of one FWI shot gradient: the propagations at 80 B per
    cell update (2 fused: the nonlinear forward recording the source wavefield
    and the Born adjoint; 3 unfused), plus per coarse sample and cell the 16-bit
    snapshot written and read (4 + 4 B) and the read-modify-write of the five
    FP32 images (40 B)."""
    return cells * (propagations * BYTES_PER_CELL * fine_steps + (4 + 4 + 40) * nts)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="born_600x1800",
                    choices=["born_600x1800", "nl_312x520", "nl_shots", "fwi_1000x3400", "fwi_learned",
                             "cnn_train", "fwi_cfg5"])
    ap.add_argument("--batch", type=int, default=None,
                    help="shots per lockstep launch (1 = one shot at a time on the lanes); nl_shots default 8, "
                         "born_600x1800 default: the library's (1)")
    ap.add_argument("--pairs", type=int, default=48, help="fwi_learned / fwi_cfg5: Born training pairs")
    ap.add_argument("--reduced", action="store_true",
                    help="fwi_cfg5: the 136x520, 8-shot, nts=1200 stand-in instead of 1000x3400 (a quick check)")
    ap.add_argument("--phase", default="both", choices=["both", "plain", "learned"],
                    help="fwi_cfg5: run both methods, or one (a long run split over two calls)")
    ap.add_argument("--record", default=None,
                    help="fwi_cfg5: write the plain method's results to this JSON file as soon as they exist")
    ap.add_argument("--plain-record", default=None,
                    help="fwi_cfg5 --phase learned: the plain method's results (--record of a --phase plain run)")
    ap.add_argument("--conv-path", type=int, default=-1, choices=[-1, 0, 1],
                    help="cnn_train: forward convolutions on mma.sync (0) or tcgen05 (1); "
                         "-1 keeps the library default (mma.sync)")
    ap.add_argument("--epochs", type=int, default=80, help="fwi_learned: training epochs")
    ap.add_argument("--depth", type=int, default=6, help="fwi_learned: convolution layers of the ConvNet")
    ap.add_argument("--tma", type=int, default=None, choices=[0, 1, 2, 3],
                    help="cnn_train (U-Net): 0 copy-loop convolution kernel, 1 TMA kernel with one CTA per SM, "
                         "2 with up to two, 3 with up to four (the library's default)")
    ap.add_argument("--net", default=None, choices=["unet", "convnet"],
                    help="preconditioner network: the four-level U-Net (cnn_train default) or the plain ConvNet "
                         "(fwi_learned default)")
    ap.add_argument("--sigma", type=float, default=3.0,
                    help="fwi_learned: smoothing length (cells) of the training perturbations")
    ap.add_argument("--shots", type=int, default=None,
                    help="shots per GPU (default: 10 for born_600x1800; a bounded sample of 16 of the 120 shots "
                         "for fwi_1000x3400)")
    ap.add_argument("--nts", type=int, default=4000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-fwi", action="store_true",
                    help="born_600x1800: skip the bounded FWI-gradient sample (the 'fwi' keys of the line)")
    ap.add_argument("--graphs", action="store_true", help="run the time loops as CUDA graphs (off by default)")
    ap.add_argument("--fwi-unfused", action="store_true",
                    help="fwi_1000x3400: nonlinear forward + Born adjoint (3 propagations per shot) instead of "
                         "the fused gradient (2)")
    ap.add_argument("--persistent", type=int, default=None,
                    help="Born shot groups: phases run as persistent time loops (bits 1 source, 2 scattered, "
                         "4 adjoint; 0 = one launch per fine step); default: the library's")
    ap.add_argument("--lanes", type=int, default=0,
                    help="shot lanes (concurrent shots on the GPU); 0 keeps the library default")
    ap.add_argument("--kernel", type=int, default=-1, choices=[-1, 0, 1, 2, 3, 4, 5],
                    help="-1: autotune (default); 0: tile kernel k_step; 1: TMA sweep kernel k_sweep; "
                         "2: persistent TMA tile kernel k_tile; 3: k_step at 4 CTAs/SM; 4: split-field k_split; "
                         "5: two steps per launch k_pair")
    return ap.parse_args()


# ----------------------------------------------------------------------------- helpers
class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            cmd = ["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits", "-lms", "200"]
            if self.gpu_id:
                cmd += ["-i", self.gpu_id]
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax.append(float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(bytes_per_cell=BYTES_PER_CELL):
    """DRAM bytes per launch of the dominant step kernel (k_step, or k_pair for
    two steps per launch) from the committed ncu summary, if any."""
    name = "k_pair_traffic.txt" if bytes_per_cell == PAIR_BYTES_PER_CELL else "k_step_traffic.txt"
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_launch_full_size:"):
                return float(line.split(":", 1)[1])
    except Exception:
        pass
    return None


def pin_kernel(L, ctx, args):
    """--kernel k fixes the step kernel (profiling runs); -1 keeps the autotuner.
    --graphs runs the time loops as CUDA graphs."""
    from elastic_isotropic_operators_b200 import _lib
    if args.kernel >= 0:
        _lib.check(L.eio_ctx_set_kernel(ctx, args.kernel, 64, 8, 8))
    if args.graphs:
        _lib.check(L.eio_ctx_set_graphs(ctx, 1))
    if args.lanes > 0:
        _lib.check(L.eio_ctx_set_lanes(ctx, args.lanes))


def kernel_name(L, ctx):
    """Step kernel the context runs (autotuned or pinned)."""
    import ctypes
    v = [ctypes.c_int() for _ in range(4)]
    L.eio_ctx_get_kernel(ctx, *[ctypes.byref(x) for x in v])
    kind, tz, cw, cpr = (x.value for x in v)
    if kind == 0:
        return "k_step (fused 5-field update, 64x16 tiles)"
    if kind == 2:
        return "k_tile (fused 5-field update, persistent, 64x16 tiles staged by TMA)"
    if kind == 3:
        return "k_step (fused 5-field update, 64x16 tiles, 4 CTAs/SM)"
    if kind == 4:
        return "k_split (fused 5-field update, 64x16 tiles, two threads per float4)"
    if kind == 5:
        return "k_pair (two fused 5-field steps per launch, 64x16 tiles widened by the stencil radius)"
    return "k_sweep (fused 5-field update, TMA x-sweep, tz=%d cw=%d cpr=%d)" % (tz, cw, cpr)


def lanes_used(L, ctx):
    """Shot lanes the context ran (concurrent shots on the GPU)."""
    import ctypes
    setting, active = ctypes.c_int(), ctypes.c_int()
    L.eio_ctx_get_lanes(ctx, ctypes.byref(setting), ctypes.byref(active))
    return int(active.value)


def read_stats(L, ctx):
    """Step-kernel counters of the timed region (and reset them): the dominant
    kernel's mean launch time, how many cell updates one of its launches
    makes (several shots per launch with shot batching) and its algorithmic
    bytes per cell update.  With the two-step kernel the dominant launches are
    the two-step ones (100 B per cell for two updates); otherwise the single
    steps (80 B per cell)."""
    import ctypes
    pl, pms = ctypes.c_longlong(), ctypes.c_double()
    L.eio_ctx_pair_stats(ctx, ctypes.byref(pl), ctypes.byref(pms))
    cells = ctypes.c_longlong()
    L.eio_ctx_step_cells(ctx, ctypes.byref(cells))
    launches, sl, sms = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_double()
    L.eio_ctx_stats(ctx, 0, 1, ctypes.byref(launches), ctypes.byref(sl), ctypes.byref(sms))
    singles, single_ms = sl.value - pl.value, sms.value - pms.value
    cells_per_launch = cells.value / max(singles, 1)
    if pl.value > 0 and pms.value >= single_ms:
        avg, bpc, n = pms.value / pl.value, PAIR_BYTES_PER_CELL, pl.value
        cells_per_launch = None
    else:
        avg, bpc, n = single_ms / max(singles, 1), BYTES_PER_CELL, singles
    return {"launches": int(launches.value), "avg_ms": avg, "bytes_per_cell": bpc, "dominant_launches": int(n),
            "step_launches": int(sl.value), "pair_launches": int(pl.value), "step_cells": int(cells.value),
            "cells_per_launch": cells_per_launch}


def dist_init(args):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------------------- our arm
def run_ours(args, ws, rank, local):
    import ctypes
    import torch
    from elastic_isotropic_operators_b200 import _lib, prop, synthetic

    w = synthetic.born_600x1800(nts=args.nts, nshots=args.shots or 10, seed=2024 + rank)
    src, rec = w.geometry()
    sig = [w.source_signal()]
    dev = torch.device("cuda", local)
    w.par.set("iGpu", str(local))
    born = prop.BornElasticShotsGpu(w.elastic, w.par, sig, *src, *rec)
    L = _lib.lib()
    ctx = born.ctx
    pin_kernel(L, ctx, args)
    if args.batch is not None:
        _lib.check(L.eio_ctx_set_born_batch(ctx, args.batch))
    if args.persistent is not None:
        _lib.check(L.eio_ctx_set_persistent(ctx, args.persistent))
    est = torch.cuda.ExternalStream(L.eio_ctx_stream(ctx), device=dev)   # the engine's launch stream
    nsh = w.nExp
    fine_steps, cells = ctypes.c_longlong(), ctypes.c_longlong()
    _lib.check(L.eio_ctx_counts(ctx, ctypes.byref(fine_steps), ctypes.byref(cells)))
    fine_steps, cells = fine_steps.value, cells.value
    updates_per_step = 4.0 * nsh * fine_steps * cells     # fwd: 2 propagations, adj: 2

    # ---- device-resident inputs
    dm5 = [torch.from_numpy(a).to(dev) for a in born.prepareModel(w.extra["dmodel"])]
    grad5 = [torch.zeros_like(a) for a in dm5]
    shots = []
    for e in range(nsh):
        fine, sp, rp = born.prepareShot(e)
        f_dev = [torch.from_numpy(a).to(dev) for a in fine]
        d_dev = [torch.zeros((len(rp[prop._FIELD_GRID[f]]), w.nts), dtype=torch.float32, device=dev)
                 for f in range(5)]
        sp_a = [np.ascontiguousarray(p, np.int32) for p in sp]
        rp_a = [np.ascontiguousarray(p, np.int32) for p in rp]
        shots.append(dict(
            fine=f_dev, data=d_dev, sp=sp_a, rp=rp_a,
            fine_pp=_lib.ptr_array([t.data_ptr() for t in f_dev]),
            data_pp=_lib.ptr_array([t.data_ptr() for t in d_dev]),
            sp_pp=_lib.ptr_array([a.ctypes.data for a in sp_a]), sn=(ctypes.c_int * 4)(*[len(a) for a in sp_a]),
            rp_pp=_lib.ptr_array([a.ctypes.data for a in rp_a]), rn=(ctypes.c_int * 4)(*[len(a) for a in rp_a])))
    dm_pp = _lib.ptr_array([t.data_ptr() for t in dm5])
    grad_pp = _lib.ptr_array([t.data_ptr() for t in grad5])
    # every shot in one call (eio_born_shots_dev), spread over the context's shot lanes
    all_fine = _lib.ptr_array([t.data_ptr() for s in shots for t in s["fine"]])
    all_data = _lib.ptr_array([t.data_ptr() for s in shots for t in s["data"]])
    all_sp = _lib.ptr_array([a.ctypes.data for s in shots for a in s["sp"]])
    all_sn = (ctypes.c_int * (4 * nsh))(*[len(a) for s in shots for a in s["sp"]])
    all_rp = _lib.ptr_array([a.ctypes.data for s in shots for a in s["rp"]])
    all_rn = (ctypes.c_int * (4 * nsh))(*[len(a) for s in shots for a in s["rp"]])
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2
    torch.cuda.synchronize()

    def step():
        _lib.check(L.eio_born_shots_dev(ctx, 0, nsh, all_fine, dm_pp, all_data, all_sp, all_sn, all_rp, all_rn))
        _lib.check(L.eio_born_shots_dev(ctx, 1, nsh, all_fine, grad_pp, all_data, all_sp, all_sn, all_rp, all_rn))
        if ws > 1:
            import torch.distributed as dist
            for g in grad5:
                dist.all_reduce(g)

    for _ in range(args.warmup):
        step()
        flush.zero_()
    torch.cuda.synchronize()

    # ---- timed region (device-resident)
    gpu_uuid = None
    try:
        gpu_uuid = str(torch.cuda.get_device_properties(dev).uuid)
        if not gpu_uuid.startswith("GPU-"):
            gpu_uuid = "GPU-" + gpu_uuid
    except Exception:
        pass
    clocks = ClockSampler(gpu_uuid)
    L.eio_ctx_stats(ctx, 1, 1, None, None, None)
    barrier(ws)
    torch.cuda.synchronize()
    clocks.start()
    t_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(est)
        step()
        ev1.record(est)
        torch.cuda.synchronize()
        t_ms += ev0.elapsed_time(ev1)
    barrier(ws)
    clk = clocks.stop()
    st = read_stats(L, ctx)
    t_ms = max_over_ranks(ws, t_ms)
    value = ws * updates_per_step * args.steps / (t_ms * 1e-3) / 1e9

    # roofline of the dominant kernel (fused step, or two fused steps per launch)
    avg_launch_ms = st["avg_ms"]
    lanes = lanes_used(L, ctx)
    cpl = st["cells_per_launch"] or cells
    batched = cpl > 1.01 * cells             # launches that advance several shots (one stream)
    bytes_per_launch = st["bytes_per_cell"] * cpl
    if lanes == 1 or batched:
        achieved = bytes_per_launch / (avg_launch_ms * 1e-3) / 1e9
        basis = ("algorithmic bytes per launch (%.2f shots x 80 B x interior cells) / mean CUDA-event duration of "
                 "the step launches (engine stream)" % (cpl / cells))
    else:
        # the lanes' step kernels overlap, so a launch's event time includes the other lanes' work:
        # the step launches' algorithmic bytes over the timed region instead
        achieved = st["bytes_per_cell"] * cells * st["dominant_launches"] / (t_ms * 1e-3) / 1e9
        basis = ("%d shot lanes overlap: algorithmic bytes of every step launch of the timed region / its "
                 "duration" % lanes)
    peak, peak_kind = measured_peak()
    roof = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
            "frac": round(achieved / peak, 4), "traffic": profile_traffic(st["bytes_per_cell"]),
            "peak_source": peak_kind, "kernel": kernel_name(L, ctx), "basis": basis,
            "avg_launch_us": round(avg_launch_ms * 1e3, 3),
            "algorithmic_bytes_per_launch": bytes_per_launch,
            "shots_per_launch": round(cpl / cells, 3),
            "launches": {"step_kernel": st["step_launches"], "two_step": st["pair_launches"]},
            # whole job: every cell update of the timed region at 80 B (step kernels, imaging,
            # sparse work and launch gaps included)
            "job_gbs": round(BYTES_PER_CELL * value, 1),
            "job_frac": round(BYTES_PER_CELL * value / peak, 4)}

    # ---- e2e through the reference-facing operator API (host buffers)
    e2e = None
    if not args.no_e2e:
        model = born.modelSpace()
        model.getNdArray()[...] = w.extra["dmodel"]
        data = born.dataSpace()
        gvec = born.modelSpace()
        born.forward(False, model, data)   # warm the host path
        torch.cuda.synchronize()
        barrier(ws)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            born.forward(False, model, data)
            born.adjoint(False, gvec, data)
            if ws > 1:
                import torch.distributed as dist
                g = torch.from_numpy(gvec.getNdArray()).to(dev)
                dist.all_reduce(g)
                gvec.getNdArray()[...] = g.cpu().numpy()
        torch.cuda.synchronize()
        t_e2e = max_over_ranks(ws, time.perf_counter() - t0)
        n = w.nz * w.nx
        # per step: the perturbation grids once (forward) and the gradient grids once
        # (adjoint); per shot and direction the fine source traces and the receiver
        # interpolators; the irregular receiver traces out (forward) and in (adjoint)
        src_bytes = sum(4 * s["fine"][f].numel() for s in shots for f in range(5))
        irr_bytes = 4 * int(np.prod(data.getNdArray().shape))
        interp_bytes = 0
        for k in range(4):
            g = born.rec[k][0]
            interp_bytes += 4 * (3 * g.nDeviceIrreg * g.nFiltTotal + g.nDeviceReg + 1)
        h2d = 4 * 5 * n + src_bytes * 2 + irr_bytes + 2 * nsh * interp_bytes
        d2h = irr_bytes + 4 * 5 * n
        e2e = {"value": round(ws * updates_per_step * args.steps / t_e2e / 1e9, 3), "unit": "Gcell-updates/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": round(1e3 * t_e2e / args.steps, 1)}

    # ---- CPU baseline: the oracle port (OpenMP, FP32) on a bounded sample
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(w, born)

    out = {
        "metric": "Gcells/s", "value": round(value, 3), "unit": "Gcell-updates/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_ms / args.steps, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "born_600x1800: Born forward + adjoint, %d shots per GPU, nts=%d (%d fine steps), "
                               "600x1800 grid, 900 receivers" % (nsh, w.nts, fine_steps),
                   "nz": w.nz, "nx": w.nx, "nts": w.nts, "shots_per_gpu": nsh, "propagations_per_step": 4 * nsh,
                   "cell_updates_per_step": updates_per_step * ws,
                   "shot_lanes": lanes_used(L, ctx),
                   "l2": "inputs larger than L2 (34.6 GB FP32 source-wavefield history per shot) and a 256 MB "
                         "L2 flush between timed steps"},
        # Born forward + adjoint pairs of one shot per second, and their algorithmic bytes
        # (born_pair_bytes) over the measured HBM peak per measured time of a pair
        "born_pairs_per_s": round(ws * nsh * args.steps / (t_ms * 1e-3), 4),
        "born_pair_bytes": born_pair_bytes(cells, fine_steps, w.nts),
        "born_pair_roofline_frac": round(
            (born_pair_bytes(cells, fine_steps, w.nts) / (peak * 1e9)) / ((t_ms * 1e-3) / (ws * nsh * args.steps)),
            4),
        "e2e": e2e, "roofline": roof, "cpu_baseline": cpu, "clocks": clk,
        "gpu_launches": st["launches"],
    }
    return out


def cpu_baseline(w, born):
    """Oracle (FP32 OpenMP port) Born forward of one shot of the same grid on a
    bounded number of time samples."""
    from oracle import oracle as O
    nts_s = 150
    c = O.Case.from_workload(w)
    c.par["nts"] = nts_s
    orc = O.Oracle("f")
    g = c.grid()
    med = orc.medium(c.ep, g["dts"], g["S"])
    src = O._grids(orc, c, *c.src[0])
    rec = O._grids(orc, c, *c.rec)
    sig = w.source_signal()[:, :, :nts_s]
    fine = O.born_sources(orc, c, g, med, src, sig)
    dm = O.born_model_slice(orc, g, med, w.extra["dmodel"])
    data = [np.zeros((len(rec[O.FIELD_GRID[f]]["uniq"]), nts_s), np.float32) for f in range(5)]
    t0 = time.perf_counter()
    orc.born_prop(0, g, med, fine, dm, data, O._reg_pos(src), O._reg_pos(rec))
    dt = time.perf_counter() - t0
    upd = 2.0 * (nts_s - 1) * g["S"] * (g["nz"] - 8) * (g["nx"] - 8)
    return {"value": round(upd / dt / 1e9, 4), "unit": "Gcell-updates/s", "cores": O.num_threads(),
            "kind": "port",
            "sample": "oracle FP32 Born forward (source + scattered propagation), 1 shot, 600x1800 grid, "
                      "nts=%d (%d fine steps), %.1f s" % (nts_s, (nts_s - 1) * g["S"], dt)}


# ----------------------------------------------------------------------------- reference arm
def run_reference(args, ws, rank, local):
    """The reference's own CUDA drivers (oracle/_ref) on one shot of the same workload
    per step: Born forward then Born adjoint, each a full init/alloc/propagate/free
    like BornElasticGpu::forward/adjoint."""
    from oracle import oracle as O
    from elastic_isotropic_operators_b200 import synthetic
    if args.workload == "nl_312x520":
        if not O.RefGpu.available("f"):
            return {"impl": "reference", "unavailable": "oracle/_ref not built (reference tree absent at build time)"}
        return run_reference_nl(args)
    if args.workload == "nl_shots":
        return {"impl": "reference", "unavailable": "the reference arm of the nonlinear path is timed on one shot "
                "(--workload nl_312x520); its drivers propagate the shots of a call one after another"}
    if args.workload in ("fwi_learned", "cnn_train"):
        return {"impl": "reference", "unavailable": "the reference has no learned preconditioner and no FWI driver "
                "(its scripts call pySolver, which is not in the reference tree); the plain L-BFGS arm of this "
                "workload is the method without the learned part"}
    if args.workload == "fwi_1000x3400":
        return {"impl": "reference", "unavailable": "the reference propagates every shot on the whole grid and its "
                "Born drivers index the history with the 32-bit product its*nz*nx (kernelsGpuElastic.cu:1342), "
                "which overflows here (5000*1000*3400 >= 2^31)"}
    w = synthetic.born_600x1800(nts=args.nts, nshots=1, seed=2024)
    if not O.RefGpu.available("f"):
        return run_reference_port(args, w, "oracle/_ref not built (reference tree absent at build time)")
    import torch
    if not torch.cuda.is_available():
        return run_reference_port(args, w, "no CUDA device on this machine")
    sample_note = ""
    if not O.RefGpu.born_supported(O.Case.from_workload(w).grid()):
        # The reference's Born drivers index their Vx/Vz history with the 32-bit product
        # its*nz*nx (kernelsGpuElastic.cu:1342), which overflows for nts*nz*nx >= 2^31 (here
        # 4000*600*1800; on this grid they faulted with an illegal memory access at
        # BornElasticGpuFunctions.cu:763 and are not run at that length again).  The bounded
        # sample is the same grid, shot and perturbation with the record cut to the longest
        # their index admits, nts = 1900 (1900*600*1800 < 2^31); Gcell-updates/s is per cell
        # update, so the record length does not enter the comparison.
        w = synthetic.born_600x1800(nts=1900, nshots=1, seed=2024)
        sample_note = ("; record cut from nts=%d to nts=1900, the longest the reference's 32-bit history "
                       "index admits on this grid (its*nz*nx < 2^31, kernelsGpuElastic.cu:1342)" % args.nts)
    orc = O.Oracle("f")
    c = O.Case.from_workload(w)
    g = c.grid()
    med = orc.medium(c.ep, g["dts"], g["S"])
    src = O._grids(orc, c, *c.src[0])
    rec = O._grids(orc, c, *c.rec)
    fine = O.born_sources(orc, c, g, med, src, w.source_signal())
    dm = O.born_model_slice(orc, g, med, w.extra["dmodel"])
    ref = O.RefGpu("f")
    data = [np.zeros((len(rec[O.FIELD_GRID[f]]["uniq"]), g["nts"]), np.float32) for f in range(5)]
    grad = [np.zeros_like(a) for a in dm]

    def step():
        ref.born_prop(0, g, med, fine, [a.copy() for a in dm], data, O._reg_pos(src), O._reg_pos(rec))
        ref.born_prop(1, g, med, fine, grad, data, O._reg_pos(src), O._reg_pos(rec))

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    cells = (g["nz"] - 8) * (g["nx"] - 8)
    upd = 4.0 * (g["nts"] - 1) * g["S"] * cells * args.steps
    v = upd / dt / 1e9
    return {"impl": "reference", "metric": "Gcells/s", "value": round(v, 3), "unit": "Gcell-updates/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dt / args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "born_600x1800: Born forward + adjoint, 1 shot per step (bounded sample of the "
                                   "10-shot workload), nts=%d%s" % (g["nts"], sample_note), "nz": g["nz"],
                       "nx": g["nx"], "nts": g["nts"]},
            "cpu_baseline": {"value": round(v, 3), "unit": "Gcell-updates/s", "cores": 1, "kind": "reference",
                             "sample": "reference CUDA drivers (elastic_iso_float, built for sm_100a) on the B200, "
                                       "1 shot of the 600x1800 grid, nts=%d, each call a full init/alloc/propagate/"
                                       "free as BornElasticGpu::forward/adjoint; the reference has no CPU "
                                       "implementation of this path" % g["nts"]},
            "e2e": {"value": round(v, 3), "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_reference_port(args, w, why_not_gpu):
    """CPU arm: the oracle (FP32 OpenMP restatement of the reference's algorithm) on
    the box's host cores, all threads.  Each step is a bounded sample of the
    workload: Born forward + Born adjoint of one shot of the 600x1800 grid with
    nts=60 coarse samples."""
    from oracle import oracle as O
    nts_s = 60
    c = O.Case.from_workload(w)
    c.par["nts"] = nts_s
    orc = O.Oracle("f")
    g = c.grid()
    med = orc.medium(c.ep, g["dts"], g["S"])
    src = O._grids(orc, c, *c.src[0])
    rec = O._grids(orc, c, *c.rec)
    fine = O.born_sources(orc, c, g, med, src, w.source_signal()[:, :, :nts_s])
    dm = O.born_model_slice(orc, g, med, w.extra["dmodel"])
    data = [np.zeros((len(rec[O.FIELD_GRID[f]]["uniq"]), nts_s), np.float32) for f in range(5)]
    grad = [np.zeros_like(a) for a in dm]

    def step():
        orc.born_prop(0, g, med, fine, dm, data, O._reg_pos(src), O._reg_pos(rec))
        orc.born_prop(1, g, med, fine, grad, data, O._reg_pos(src), O._reg_pos(rec))

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    upd = 4.0 * (nts_s - 1) * g["S"] * (g["nz"] - 8) * (g["nx"] - 8) * args.steps
    v = upd / dt / 1e9
    sample = ("oracle FP32 Born forward + adjoint (2 propagations each), 1 shot, 600x1800 grid, nts=%d "
              "(%d fine steps) per step, %d threads" % (nts_s, (nts_s - 1) * g["S"], O.num_threads()))
    return {"impl": "reference", "metric": "Gcells/s", "value": round(v, 4), "unit": "Gcell-updates/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dt / args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "born_600x1800: Born forward + adjoint, bounded sample (1 shot, nts=%d) of the "
                                   "10-shot nts=%d workload" % (nts_s, w.nts), "nz": w.nz, "nx": w.nx},
            "cpu_baseline": {"value": round(v, 4), "unit": "Gcell-updates/s", "cores": O.num_threads(),
                             "kind": "port", "sample": sample},
            "reference_gpu": {"unavailable": why_not_gpu},
            "e2e": {"value": round(v, 4), "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_reference_nl(args):
    """Reference CUDA drivers, nonlinear forward of the 312x520 shot (full nts)."""
    from oracle import oracle as O
    from elastic_isotropic_operators_b200 import synthetic
    w = synthetic.nl_312x520()
    orc = O.Oracle("f")
    c = O.Case.from_workload(w)
    g = c.grid()
    med = orc.medium(c.ep, g["dts"], g["S"])
    src = O._grids(orc, c, *c.src[0])
    rec = O._grids(orc, c, *c.rec)
    reg = []
    sig = w.source_signal()
    for f in range(5):
        G = src[O.FIELD_GRID[f]]
        r = np.zeros((len(G["uniq"]), g["nts"]), np.float32)
        orc.sinterp_apply(G, 1, 0, r, np.ascontiguousarray(sig[f]))
        reg.append(r)
    O._scale_sources(orc, g, med, src, reg)
    data = [np.zeros((len(rec[O.FIELD_GRID[f]]["uniq"]), g["nts"]), np.float32) for f in range(5)]
    ref = O.RefGpu("f")

    def step():
        ref.nl_prop(0, g, med, reg, data, O._reg_pos(src), O._reg_pos(rec))

    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    upd = (g["nts"] - 1) * g["S"] * (g["nz"] - 8) * (g["nx"] - 8) * args.steps
    v = upd / dt / 1e9
    return {"impl": "reference", "metric": "Gcells/s", "value": round(v, 3), "unit": "Gcell-updates/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dt / args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "nl_312x520: nonlinear forward, 1 shot, nts=2000 (3998 fine steps)"},
            "cpu_baseline": {"value": round(v, 3), "unit": "Gcell-updates/s", "cores": 1, "kind": "reference",
                             "sample": "reference CUDA drivers (elastic_iso_float, built for sm_100a) on the B200; "
                                       "the reference has no CPU implementation of this path"},
            "e2e": {"value": round(v, 3), "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def run_ours_nl(args, ws, rank, local):
    """Nonlinear forward of the 312x520 shot (one shot per rank)."""
    import ctypes
    import torch
    from elastic_isotropic_operators_b200 import _lib, prop, synthetic
    w = synthetic.nl_312x520()
    dev = torch.device("cuda", local)
    w.par.set("iGpu", str(local))
    src, rec = w.geometry()
    nl = prop.nonlinearPropElasticShotsGpu(w.elastic, w.par, *src, *rec)
    L = _lib.lib()
    ctx = nl.ctx
    pin_kernel(L, ctx, args)
    est = torch.cuda.ExternalStream(L.eio_ctx_stream(ctx), device=dev)   # the engine's launch stream
    fine_steps, cells = ctypes.c_longlong(), ctypes.c_longlong()
    _lib.check(L.eio_ctx_counts(ctx, ctypes.byref(fine_steps), ctypes.byref(cells)))
    fine_steps, cells = fine_steps.value, cells.value
    upd = float(fine_steps * cells)
    # regular-grid sources prepared by the library's own host code
    reg, sp, rp = nl.prepareShot(0, w.source_signal())
    m_dev = [torch.from_numpy(a).to(dev) for a in reg]
    d_dev = [torch.zeros((len(rp[prop._FIELD_GRID[f]]), w.nts), device=dev) for f in range(5)]
    sp = [np.ascontiguousarray(a, np.int32) for a in sp]
    rp = [np.ascontiguousarray(a, np.int32) for a in rp]
    args_c = (_lib.ptr_array([t.data_ptr() for t in m_dev]), _lib.ptr_array([t.data_ptr() for t in d_dev]),
              _lib.ptr_array([a.ctypes.data for a in sp]), (ctypes.c_int * 4)(*[len(a) for a in sp]),
              _lib.ptr_array([a.ctypes.data for a in rp]), (ctypes.c_int * 4)(*[len(a) for a in rp]))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def step():
        _lib.check(L.eio_nl_fwd_reg_dev(ctx, *args_c))

    for _ in range(args.warmup):
        step()
        flush.zero_()
    L.eio_ctx_stats(ctx, 1, 1, None, None, None)
    barrier(ws)
    torch.cuda.synchronize()
    clocks = ClockSampler(None)
    clocks.start()
    t_ms = 0.0
    for _ in range(args.steps):
        flush.zero_()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(est)
        step()
        ev1.record(est)
        torch.cuda.synchronize()
        t_ms += ev0.elapsed_time(ev1)
    clk = clocks.stop()
    st = read_stats(L, ctx)
    t_ms = max_over_ranks(ws, t_ms)
    avg = st["avg_ms"]
    peak, pk = measured_peak()
    ach = st["bytes_per_cell"] * cells / (avg * 1e-3) / 1e9
    model = nl.modelSpace()
    model.getNdArray()[...] = w.source_signal()[None]
    data = nl.dataSpace()
    nl.forward(False, model, data)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        nl.forward(False, model, data)
    t_e2e = max_over_ranks(ws, time.perf_counter() - t0)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        from oracle import oracle as O
        orc, c = O.Oracle("f"), O.Case.from_workload(w)
        t0 = time.perf_counter()
        O.nl_forward(orc, c, model.getNdArray())
        dt = time.perf_counter() - t0
        cpu = {"value": round(upd / dt / 1e9, 4), "unit": "Gcell-updates/s", "cores": O.num_threads(), "kind": "port",
               "sample": "oracle FP32 nonlinear forward of the whole workload (1 shot, 3998 fine steps), %.1f s" % dt}
    return {"metric": "Gcells/s", "value": round(ws * upd * args.steps / (t_ms * 1e-3) / 1e9, 3),
            "unit": "Gcell-updates/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(t_ms / args.steps, 2), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "nl_312x520: nonlinear forward, 1 shot per GPU, 312x520 grid, nts=2000 "
                                   "(3998 fine steps), 400 receivers",
                       "l2": "working set (13 MB) is L2-resident by construction; 256 MB L2 flush between steps"},
            "e2e": {"value": round(ws * upd * args.steps / t_e2e / 1e9, 3), "unit": "Gcell-updates/s",
                    "h2d_bytes_per_step": int(sum(4 * a.size for a in reg)),
                    "d2h_bytes_per_step": int(sum(4 * t.numel() for t in d_dev))},
            "roofline": {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(ach / peak, 4), "traffic": None, "peak_source": pk,
                         "kernel": kernel_name(L, ctx), "avg_launch_us": round(avg * 1e3, 3),
                         "algorithmic_bytes_per_launch": st["bytes_per_cell"] * cells},
            "cpu_baseline": cpu, "clocks": clk, "gpu_launches": st["launches"]}


def run_ours_fwi(args, ws, rank, local):
    """FWI gradients of the batched-FWI case: per step, the misfit and gradient
    of a bounded sample of its shots through the operator API (FwiObjective),
    with cropped shots, BF16 source-wavefield checkpoints and shot lanes.  The
    fused gradient runs 2 propagations of a shot's window (nonlinear forward
    recording the source wavefield, Born adjoint); --fwi-unfused runs the
    reference's 3 (nonlinear forward, Born adjoint with its own source
    propagation).  Cell updates count the propagations actually run."""
    import ctypes
    import torch
    from elastic_isotropic_operators_b200 import _lib, fwi, prop, synthetic
    nsh = args.shots or 16
    # a bounded sample of the 120 shots, spread over the line; each rank its own shots
    pick = np.linspace(0, 119, nsh * ws).round().astype(int)[rank::ws]
    w = synthetic.fwi_1000x3400(nshots=120, select=list(pick))
    w.par.set("iGpu", str(local))
    dev = torch.device("cuda", local)
    src, rec = w.geometry()
    sig = w.source_signal()[None]
    nl = prop.nonlinearFwiPropElasticShotsGpu(w.elastic, w.par, sig, *src, *rec)
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [w.source_signal()], *src, *rec)
    born.setCheckpointPrecision(1)
    for op in (nl, born):
        pin_kernel(op._L, op.ctx, args)
    if args.lanes <= 0:
        # cropped shots are small: four in flight beat two (3.59 -> 3.87 shot gradients/s measured)
        _lib.check(_lib.lib().eio_ctx_set_lanes(born.ctx, 4))
    ix0, nxw = nl.autoShotWindows()
    born.setShotWindows(ix0, nxw)
    d_obs = nl.dataSpace()
    nl.forward(False, w.extra["true_model"], d_obs)          # observed data, untimed
    obj = fwi.FwiObjective(nl, born, d_obs, fused=not args.fwi_unfused)
    props = 2 if obj.fused else 3
    m0 = w.extra["start_model"]
    L = _lib.lib()
    est = torch.cuda.ExternalStream(L.eio_ctx_stream(born.ctx), device=dev)
    fine_steps = (w.nts - 1) * 2
    updates = float(sum(props * fine_steps * (w.nz - 8) * (int(n) - 8) for n in nxw))
    for _ in range(args.warmup):
        obj.value_and_gradient(m0)
    torch.cuda.synchronize()
    for op in (nl, born):
        L.eio_ctx_stats(op.ctx, 1, 1, None, None, None)
    barrier(ws)
    clocks = ClockSampler(None)
    clocks.start()
    t_ms = 0.0
    for _ in range(args.steps):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(est)
        obj.value_and_gradient(m0)
        ev1.record(est)
        torch.cuda.synchronize()
        t_ms += ev0.elapsed_time(ev1)
    clk = clocks.stop()
    launches = 0
    for op in (nl, born):
        launches += read_stats(L, op.ctx)["launches"]
    t_ms = max_over_ranks(ws, t_ms)
    value = ws * updates * args.steps / (t_ms * 1e-3) / 1e9
    peak, pk = measured_peak()
    sg_per_s = ws * nsh * args.steps / (t_ms * 1e-3)
    # algorithmic bytes of the mean shot gradient (each shot on its own window)
    sg_bytes = float(np.mean([shot_gradient_bytes((w.nz - 8) * (int(n) - 8), fine_steps, w.nts, props)
                              for n in nxw]))
    n_data = int(np.prod(d_obs.getNdArray().shape))
    # model (forward and Born background, or the one fused background), residual
    h2d = 4 * (3 * w.nz * w.nx) * (1 if obj.fused else 2) + 4 * n_data
    d2h = 4 * n_data + 4 * 3 * w.nz * w.nx               # modelled data, gradient
    return {"metric": "Gcells/s", "value": round(value, 3), "unit": "Gcell-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_ms / args.steps, 1),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "fwi_1000x3400: FWI misfit + gradient (%s), "
                                   "%d of the 120 shots per GPU (bounded sample), 1000x3400 grid, nts=5000, "
                                   "cropped shots (uneven 2-8 km windows, mean %d columns), BF16 checkpoints"
                                   % ("fused: nonlinear forward recording the source wavefield + Born adjoint"
                                      if obj.fused else "nonlinear forward + Born adjoint", nsh, int(np.mean(nxw))),
                       "propagations_per_shot": props,
                       "shots_per_gpu": nsh, "shot_lanes": lanes_used(L, born.ctx),
                       "cell_updates_per_step": updates * ws,
                       "l2": "inputs larger than L2 (BF16 history of a window: several GB per shot)"},
            "shot_gradients_per_s": round(sg_per_s, 4),
            "shot_gradient_bytes": sg_bytes,
            "shot_gradient_roofline_frac": round(sg_bytes / (peak * 1e9) * sg_per_s, 4),
            "e2e": {"value": round(value, 3), "unit": "Gcell-updates/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "note": "the operator API with host buffers is the only path"},
            "roofline": {"bound": "hbm", "achieved": round(BYTES_PER_CELL * value, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(BYTES_PER_CELL * value / peak, 4), "traffic": None, "peak_source": pk,
                         "basis": "80 B per cell update over the timed region (job level)",
                         "kernel": kernel_name(L, born.ctx)},
            "cpu_baseline": None, "clocks": clk, "gpu_launches": int(launches)}


class _CountedObjective:
    """Counts the shot propagations an FWI objective runs (misfit: 1 per shot;
    gradient: 2 fused, 3 unfused)."""

    def __init__(self, obj, nshots):
        self.obj, self.n, self.props = obj, nshots, 0

    def value(self, m):
        self.props += self.n
        return self.obj.value(m)

    def value_and_gradient(self, m):
        self.props += (2 if self.obj.fused else 3) * self.n
        return self.obj.value_and_gradient(m)


class _Reached(Exception):
    pass


def _interior_error(m, true, pad):
    """Relative L2 error of each elastic parameter against the true model over
    the interior (the absorbing pads excluded)."""
    sl = (slice(None), slice(pad, -pad), slice(pad, -pad))
    d = (np.asarray(m, np.float64) - true)[sl]
    t = np.asarray(true, np.float64)[sl]
    return [round(float(np.linalg.norm(d[c]) / np.linalg.norm(t[c])), 6) for c in range(3)]


CFG5_BANDS = ((0.5, 1.0, 3.0, 4.5), (0.5, 1.0, 5.0, 6.5), (0.5, 1.0, 10.0, 12.0))   # 3 -> 5 -> 10 Hz


def run_ours_cfg5(args, ws, rank, local):
    """End-to-end elastic FWI on the batched-FWI model (1000x3400, 120 shots,
    nts=5000 at 1 ms): L-BFGS over the 3 -> 5 -> 10 Hz bands (fwi.multiscale,
    --steps iterations per band, 10 by default: 30 in all), once with the plain
    gradient and once with learned steps (precond.LearnedPreconditioner, U-Net
    by default: --pairs Born normal-operator images J^T J dm of seeded smooth
    perturbations at the start model, --epochs of training; each learned step
    is kept only when the exact misfit accepts it, else the plain step runs).
    Reports the wall-clock to a 1e-2 reduction of the final band's misfit,
    the learned method's wall-clock (with and without training) to the plain
    method's final misfit, iterations and the model error against the true
    model.  --reduced: the 136x520, 8-shot stand-in (a quick check)."""
    import torch
    from elastic_isotropic_operators_b200 import _lib, fwi, precond, prop, synthetic
    if args.reduced:
        nsh = args.shots or 8
        w = synthetic.fwi_1000x3400(nz=136, nx=520, nts=1200, nshots=nsh, nrec=60, pad=20, window_km=(2.0, 4.0))
        pad = 20
    else:
        nsh = args.shots or 120
        # fewer shots: an evenly spaced subset of the 120-shot acquisition (the same shots, windows and receivers)
        sel = None if nsh >= 120 else [int(i) for i in np.linspace(0, 119, nsh).round()]
        w = synthetic.fwi_1000x3400(nshots=120, select=sel)
        nsh = w.nExp
        pad = 50
    w.par.set("iGpu", str(local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    src, rec = w.geometry()
    sig = w.source_signal()
    nl = prop.nonlinearFwiPropElasticShotsGpu(w.elastic, w.par, sig[None], *src, *rec)
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [sig], *src, *rec)
    for op in (nl, born):
        pin_kernel(op._L, op.ctx, args)
    true = np.asarray(w.extra["true_model"], np.float64)
    pad += synthetic.FAT                                       # the interior starts past the pads and the stencil halo
    d_obs = nl.dataSpace()
    nl.forward(False, w.extra["true_model"], d_obs)          # observed data from the true model, untimed
    d_obs = np.array(d_obs.getNdArray(), copy=True)
    m0 = w.extra["start_model"]
    niter = args.steps
    final_band = CFG5_BANDS[-1]

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / 1e3

    # the final band's misfit at the start model (untimed): the reference of the 1e-2 reduction
    f0 = fwi.band_objective(nl, born, d_obs, None, w.dts, final_band).value(m0)

    def run_traced(precond_obj):
        """multiscale L-BFGS; trace: per iteration (band, iteration, misfit, seconds since the start)"""
        trace, stats = [], {}
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev0.record()

        def objective_for_band(band):
            return fwi.band_objective(nl, born, d_obs, None, w.dts, band)

        def cb(k, it, m, f, g):
            ev = torch.cuda.Event(enable_timing=True)
            ev.record()
            torch.cuda.synchronize()
            trace.append((k, it + 1, float(f), ev0.elapsed_time(ev) / 1e3))
            print("fwi_cfg5 %s band %d iteration %d: misfit %.6g at %.1f s" % (
                "learned" if precond_obj is not None else "plain", k, it + 1, f, trace[-1][3]),
                file=sys.stderr, flush=True)

        m, hists = fwi.multiscale(objective_for_band, m0, CFG5_BANDS, niter=niter, iter_callback=cb, scale=m0,
                                  precond=precond_obj, stats=stats)
        return m, hists, trace, stats

    def first(trace, level):
        """seconds at the first final-band iteration whose misfit is at or below level (None: never)"""
        for b, it, f, t in trace:
            if b == len(CFG5_BANDS) - 1 and f <= level:
                return round(t, 3)
        return None

    barrier(ws)
    clocks = ClockSampler(None)
    clocks.start()
    if args.phase in ("both", "plain"):
        (m_plain, h_plain, tr_plain, _), t_plain = timed(lambda: run_traced(None))
        f_plain_end = fwi.band_objective(nl, born, d_obs, None, w.dts, final_band).value(m_plain)
        plain = {"seconds": round(t_plain, 3), "iterations": len(tr_plain),
                 "seconds_per_iteration": round(t_plain / max(len(tr_plain), 1), 3),
                 "final_band_misfit_reduction": round(f_plain_end / f0, 6),
                 "seconds_to_1e-2_reduction": first(tr_plain, 1e-2 * f0),
                 "band_histories": [[float(v) for v in h] for h in h_plain],
                 "model_rel_error_rho_lambda_mu": _interior_error(m_plain, true, pad),
                 "trace": [list(t) for t in tr_plain]}
        if args.record and rank == 0:
            with open(args.record, "w") as f:
                json.dump(plain, f)
        print("fwi_cfg5 plain: %.1f s, final-band misfit reduction %.4g" % (t_plain, f_plain_end / f0),
              file=sys.stderr, flush=True)
    else:
        if not args.plain_record:
            raise SystemExit("fwi_cfg5 --phase learned needs --plain-record (the JSON of a --phase plain run)")
        with open(args.plain_record) as f:
            plain = json.load(f)
        t_plain = plain["seconds"]
    tr_plain = [tuple(t) for t in plain["trace"]]
    learned, t_train, t_to_plain = None, 0.0, None
    if args.phase in ("both", "learned"):
        # training pairs + training at the start model (broadband sources), then the same multiscale run
        P = [None]

        def train():
            born.setSourceSignals([sig])
            net = (precond.ConvNet(depth=args.depth, device=local, seed=0) if args.net == "convnet" else
                   precond.UNet(device=local, seed=0))
            P[0] = precond.LearnedPreconditioner(born, m0, sigma=args.sigma, seed=0, net=net)
            X, T, _, _ = P[0].make_pairs(args.pairs, seed=1)
            P[0].train(X, T, epochs=args.epochs, batch=min(4, args.pairs), lr=1e-3)

        _, t_train = timed(train)
        (m_learn, h_learn, tr_learn, st_learn), t_learn = timed(lambda: run_traced(P[0]))
        f_learn_end = fwi.band_objective(nl, born, d_obs, None, w.dts, final_band).value(m_learn)
        plain_final = tr_plain[-1][2] if tr_plain else None
        t_to_plain = first(tr_learn, plain_final) if plain_final is not None else None
        learned = {"seconds": round(t_learn, 3), "training_seconds": round(t_train, 3),
                   "iterations": len(tr_learn), "seconds_per_iteration": round(t_learn / max(len(tr_learn), 1), 3),
                   "final_band_misfit_reduction": round(f_learn_end / f0, 6),
                   "seconds_to_1e-2_reduction": first(tr_learn, 1e-2 * f0),
                   "seconds_to_plain_final_misfit": t_to_plain,
                   "learned_steps_accepted": st_learn.get("learned", 0),
                   "learned_steps_rejected": st_learn.get("rejected", 0),
                   "band_histories": [[float(v) for v in h] for h in h_learn],
                   "model_rel_error_rho_lambda_mu": _interior_error(m_learn, true, pad)}
    clk = clocks.stop()
    err0 = _interior_error(m0, true, pad)
    plain.pop("trace", None)
    speed = (round(t_plain / (t_to_plain + t_train), 3) if t_to_plain is not None else 0.0)
    speed_nt = (round(t_plain / t_to_plain, 3) if t_to_plain else 0.0)
    grid = "136x520 stand-in" if args.reduced else "1000x3400"
    return {"metric": "FWI wall-clock speed-up to the plain method's final misfit (learned vs plain, training "
                      "included)", "value": speed if learned is not None else None, "unit": "x", "n_gpus": ws,
            "steps": 3 * niter,
            "warmup": 0, "ms_per_step": round(1e3 * t_plain / (3 * niter), 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 propagation, bf16 network", "data": "synthetic",
            "config": {"workload": "fwi_cfg5: %s batched-FWI model (12.5 m, nts=%d at 1 ms, %d shots with 2-8 km "
                                   "windows), L-BFGS over the 3/5/10 Hz bands, %d iterations each, plain vs "
                                   "learned (%s, %d Born normal-operator images, %d epochs)"
                                   % (grid, w.nts, nsh, niter, "ConvNet" if args.net == "convnet" else "U-Net",
                                      args.pairs, args.epochs),
                       "l2": "each gradient streams the source history of every shot through HBM"},
            "speedup_without_training": speed_nt, "target": ">= 3x", "target_met": bool(speed >= 3.0),
            "final_band_misfit_at_start": f0, "phase": args.phase, "plain": plain, "learned": learned,
            "start_model_rel_error_rho_lambda_mu": err0,
            "cpu_baseline": None, "clocks": clk,
            "gpu_launches": int(sum(read_stats(_lib.lib(), op.ctx)["launches"] for op in (nl, born)))}


def run_ours_learned(args, ws, rank, local):
    """Learned vs plain FWI: wall-clock to the misfit that plain L-BFGS reaches in
    --steps iterations, plain against learned (Born training pairs + training +
    L-BFGS with learned steps the exact misfit accepts or rejects), on a reduced
    grid of the batched-FWI model (layered background, 4500 m/s inclusion,
    smoothed start model).  Each GPU runs the same comparison (replicas)."""
    import torch
    from elastic_isotropic_operators_b200 import _lib, fwi, precond, prop, synthetic
    nsh = args.shots or 8
    w = synthetic.fwi_1000x3400(nz=136, nx=520, nts=1200, nshots=nsh, nrec=60, pad=20, window_km=(2.0, 4.0))
    w.par.set("iGpu", str(local))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    src, rec = w.geometry()
    sig = w.source_signal()
    nl = prop.nonlinearFwiPropElasticShotsGpu(w.elastic, w.par, sig[None], *src, *rec)
    born = prop.BornElasticShotsGpu(w.elastic, w.par, [sig], *src, *rec)
    for op in (nl, born):
        pin_kernel(op._L, op.ctx, args)
    d_obs = nl.dataSpace()
    nl.forward(False, w.extra["true_model"], d_obs)          # observed data, untimed
    m0 = w.extra["start_model"]
    obj = _CountedObjective(fwi.FwiObjective(nl, born, d_obs), nsh)
    for _ in range(args.warmup):
        obj.value_and_gradient(m0)
    obj.props = 0
    L = _lib.lib()
    for op in (nl, born):
        L.eio_ctx_stats(op.ctx, 1, 1, None, None, None)
    cells = (w.nz - 8) * (w.nx - 8) * (w.nts - 1) * 2

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / 1e3

    barrier(ws)
    clocks = ClockSampler(None)
    clocks.start()
    (_, plain), t_plain = timed(lambda: fwi.lbfgs(obj, m0, niter=args.steps, scale=m0))
    props_plain = obj.props
    target = plain[-1]
    obj.props = 0
    P = None

    def train():
        nonlocal P
        net = (precond.UNet(device=local, seed=0) if args.net == "unet" else
               precond.ConvNet(depth=args.depth, device=local, seed=0))
        P = precond.LearnedPreconditioner(born, m0, sigma=args.sigma, seed=0, net=net)
        X, T, _, _ = P.make_pairs(args.pairs, seed=1)
        P.train(X, T, epochs=args.epochs, batch=8, lr=3e-3)

    _, t_train = timed(train)
    pair_props = (args.pairs + 1) * 4 * nsh                   # Born forward + adjoint (+ the illumination pair)
    trace = []
    t_start = [0.0]
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev0.record()

    def cb(it, m, f, g):
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        torch.cuda.synchronize()
        trace.append((it + 1, f, ev0.elapsed_time(ev) / 1e3))
        if f <= target:
            raise _Reached()

    stats = {}
    try:
        fwi.lbfgs(obj, m0, niter=2 * args.steps, scale=m0, precond=P, stats=stats, callback=cb)
    except _Reached:
        pass
    torch.cuda.synchronize()
    clk = clocks.stop()
    launches = sum(read_stats(L, op.ctx)["launches"] for op in (nl, born))
    reached = bool(trace) and trace[-1][1] <= target
    t_iter = trace[-1][2] if trace else float("nan")
    t_learned = t_train + t_iter
    t_plain = max_over_ranks(ws, t_plain)
    t_learned = max_over_ranks(ws, t_learned)
    speedup = t_plain / t_learned if reached else 0.0
    props_learned = obj.props + pair_props
    gcells_plain = props_plain * cells / t_plain / 1e9
    peak, pk = measured_peak()
    return {"metric": "FWI wall-clock speed-up to the plain method's final misfit (learned vs plain)",
            "value": round(speedup, 3), "unit": "x", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * t_plain / args.steps, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 propagation, bf16 network", "data": "synthetic",
            "config": {"workload": "fwi_learned: 136x520 grid of the batched-FWI model (12.5 m, nts=1200, %d shots, "
                                   "60 receivers each), plain L-BFGS for %d iterations vs learned steps "
                                   "(%d Born pairs, %d epochs, %d layers, perturbation smoothing %.1f cells)"
                                   % (nsh, args.steps, args.pairs, args.epochs, args.depth, args.sigma),
                       "l2": "each gradient streams the FP32 source history of a shot (about 1.1 GB) through HBM"},
            "plain": {"iterations": args.steps, "seconds": round(t_plain, 3), "final_misfit": target,
                      "misfit_history": [float(v) for v in plain], "propagations": props_plain},
            "learned": {"reached": reached, "iterations": trace[-1][0] if trace else 0,
                        "seconds_total": round(t_learned, 3), "seconds_training": round(t_train, 3),
                        "seconds_iterations": round(t_iter, 3),
                        "misfit_history": [float(x[1]) for x in trace], "accepted": stats.get("learned", 0),
                        "rejected": stats.get("rejected", 0), "propagations": props_learned},
            "iterations_ratio": round(args.steps / trace[-1][0], 3) if reached else None,
            "speedup_excluding_training": round(t_plain / t_iter, 3) if reached else None,
            "e2e": {"value": round(speedup, 3), "unit": "x", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                    "note": "the FWI API with host buffers is the only path"},
            "roofline": {"bound": "hbm", "achieved": round(BYTES_PER_CELL * gcells_plain, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(BYTES_PER_CELL * gcells_plain / peak, 4), "traffic": None,
                         "peak_source": pk, "basis": "80 B per cell update of the plain run over its wall-clock",
                         "kernel": kernel_name(L, born.ctx)},
            "cpu_baseline": None, "clocks": clk, "gpu_launches": int(launches)}


def cnn_step_flops(chans, npix):
    """Tensor-core FLOPs of one training step of the preconditioner network:
    forward convolutions of every layer, data gradients of all but the first,
    weight gradients of every layer (2 * 9 * cin * cout per pixel each)."""
    per = [2 * 9 * ci * co for ci, co in zip(chans[:-1], chans[1:])]
    return float(npix) * (2 * sum(per) + sum(per[1:]))


def unet_step_cost(chans, levels, batch, h, w):
    """(tensor-core FLOPs, algorithmic HBM bytes) of one U-Net training step.
    FLOPs: forward, data gradient (all but the first layer) and weight
    gradient of each 3x3 convolution, 2 * 9 * cin * cout per pixel of its
    level.  Bytes: each BF16 activation read or written once per pass it
    enters -- forward input + output; backward output gradient + ReLU mask +
    input (weight gradient) and input gradient (data gradient) -- and the
    pooling, upsampling and concatenation copies with their adjoints."""
    fl, by = 0.0, 0.0
    for k, ((ci, co), lv) in enumerate(zip(chans, levels)):
        npx = batch * (h >> lv) * (w >> lv)
        fl += 2.0 * 9 * ci * co * npx * (2 if k == 0 else 3)
        by += 2.0 * npx * ((ci + co) + (2 * co + ci) + (0 if k == 0 else ci + co))
    b = chans[0][1]
    for lv, c in ((0, b), (1, 2 * b), (2, 4 * b)):
        npx = batch * (h >> lv) * (w >> lv)
        by += 2.0 * npx * c * (1.25 + 1.25)           # pooling (read 4, write 1 per 4) and its adjoint
        by += 2.0 * npx * (3 * c) * 2 * 2             # upsampling + concatenation, their adjoints
    return fl, by


def run_ours_cnn(args, ws, rank, local):
    """Training throughput of the learned preconditioner's network: per step,
    forward, loss, data and weight gradients and the Adam update of a batch of
    --shots 256 x 256 patches (4 features in 16 channels) through the
    library's kernels -- the four-level U-Net (32 / 64 / 128 / 256 channels,
    1.17 M parameters; every convolution an implicit GEMM on tcgen05) or, with
    --net convnet, the 6-layer 32-channel ConvNet.  Inputs are resident on the
    device; each step reads them fresh from a pool larger than L2."""
    import ctypes
    import torch
    from elastic_isotropic_operators_b200 import _lib, precond
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if args.conv_path >= 0:
        _lib.check(_lib.lib().eio_cnn_set_conv_path(args.conv_path))
    path = ctypes.c_int()
    _lib.check(_lib.lib().eio_cnn_get_conv_path(ctypes.byref(path)))
    batch = args.shots or 16
    h = w = 256
    unet = (args.net or "unet") == "unet"
    if args.tma is not None:
        _lib.check(_lib.lib().eio_unet_set_tma(args.tma))
    net = precond.UNet(device=local, seed=0) if unet else precond.ConvNet(depth=6, hidden=32, device=local, seed=0)
    g = torch.Generator(device=dev)
    g.manual_seed(1)
    pool = 4                                                  # 4 batches: 4 x 64 MB of BF16 inputs
    X = torch.zeros((pool * batch, h, w, 16), dtype=torch.bfloat16, device=dev)
    X[..., :4] = torch.randn((pool * batch, h, w, 4), generator=g, device=dev).to(torch.bfloat16)
    T = torch.randn((pool * batch, h, w, 3), generator=g, device=dev)
    for i in range(args.warmup):
        k = i % pool
        net.forward(X[k * batch:(k + 1) * batch])
        net.backward(T[k * batch:(k + 1) * batch])
        net.adam()
    torch.cuda.synchronize()
    barrier(ws)
    clocks = ClockSampler(None)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for i in range(args.steps):
        k = i % pool
        net.forward(X[k * batch:(k + 1) * batch])
        loss = net.backward(T[k * batch:(k + 1) * batch])
        net.adam()
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    t_ms = max_over_ranks(ws, e0.elapsed_time(e1))
    if unet:
        nl = len(net.chans)
        # per conv: the forward GEMM; the ReLU adjoint (not the head), the weight-gradient GEMM and its split
        # sum, the weight flip and the data-gradient GEMM (not the first layer); 3 poolings, 3 x (upsampling +
        # concatenation), 3 x (concatenation adjoint + upsampling adjoint), 3 pooling adjoints; the loss and its
        # sum; Adam per layer
        launches_per_step = nl + (nl - 1) + 2 * nl + 2 * (nl - 1) + 3 + 6 + 6 + 3 + 2 + nl
        flops, alg_bytes = unet_step_cost(net.chans, net._lvl(), batch, h, w)
    else:
        depth = len(net.chans) - 1
        launches_per_step = depth + 2 * depth + 2 * (depth - 1) + 2 + depth   # conv, wgrad+sum, flip+conv, mse+sum, adam
        flops, alg_bytes = cnn_step_flops(net.chans, batch * h * w), None
    tflops = flops * args.steps / (t_ms * 1e-3) / 1e12
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            mp = json.load(f)
            peak, pk, hbm = float(mp["bf16_tflops"]), "measured", float(mp["hbm_gbs"])
    except Exception:
        peak, pk, hbm = 1590.0, "fallback", 6650.0
    samples = ws * batch * args.steps / (t_ms * 1e-3)
    gbs = alg_bytes * args.steps / (t_ms * 1e-3) / 1e9 if alg_bytes else None
    if gbs is not None and gbs / hbm > tflops / peak:
        roof = {"bound": "hbm", "achieved": round(gbs, 1), "peak": hbm, "unit": "GB/s", "frac": round(gbs / hbm, 4)}
    else:
        roof = {"bound": "tensor", "achieved": round(tflops, 2), "peak": peak, "unit": "TFLOP/s",
                "frac": round(tflops / peak, 4)}
    if unet:
        desc = ("cnn_train: %d patches of 256x256 per step, U-Net 32/64/128/256 channels (%d parameters), "
                "2x2 average pooling, nearest upsampling, concatenated skips" % (batch, net.n_params()))
        kern = ("k_conv_tma (tcgen05, TMA-fed implicit GEMM, up to 4 CTAs per SM) for forward, data and weight "
                "gradients")
    else:
        desc = "cnn_train: %d patches of 256x256 per step, 6 conv layers 16-32-32-32-32-32-16" % batch
        kern = (("k_conv3_tc (tcgen05, TMEM accumulator)" if path.value == 1 else
                 "k_conv3 (mma.sync m16n8k16)") + " + k_conv3_wgrad (mma.sync m16n8k16)")
    return {"metric": "preconditioner training throughput", "value": round(samples, 2), "unit": "patches/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_ms / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16 (FP32 accumulate)",
            "data": "synthetic", "loss": float(loss.item()),
            "config": {"workload": desc, "l2": "inputs read from a pool of 4 batches (256 MB) larger than L2"},
            "e2e": {"value": round(samples, 2), "unit": "patches/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                    "note": "training consumes device-resident pairs that the Born operators produce"},
            "roofline": dict(roof, traffic=None, peak_source=pk, tensor_tflops=round(tflops, 2),
                             tensor_frac=round(tflops / peak, 4), hbm_gbs=round(gbs, 1) if gbs else None,
                             basis="tensor-core FLOPs of a training step (forward, data and weight gradients) and, "
                                   "for the U-Net, its algorithmic activation bytes, over the timed region; the "
                                   "bound is the larger fraction", kernel=kern),
            "cpu_baseline": None, "clocks": clk, "gpu_launches": int(launches_per_step * args.steps)}


def run_ours_nl_shots(args, ws, rank, local):
    """Nonlinear forward of --shots (default 8) shots of the 312x520 case per
    step through nonlinearPropElasticShotsGpu.forward with host buffers, the
    shots batched --batch per lockstep launch (1: one at a time on the lanes)."""
    import torch
    from elastic_isotropic_operators_b200 import _lib, prop, synthetic
    nsh = args.shots or 8
    if args.batch is None:
        args.batch = 8
    w = synthetic.nl_312x520(nshots=nsh)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    w.par.set("iGpu", str(local))
    src, rec = w.geometry()
    nl = prop.nonlinearPropElasticShotsGpu(w.elastic, w.par, *src, *rec)
    L = _lib.lib()
    pin_kernel(L, nl.ctx, args)
    nl.setShotBatch(max(1, min(args.batch, 8)))   # the library default is 8
    model = nl.modelSpace()
    model.getNdArray()[...] = w.source_signal()[None]
    data = nl.dataSpace()
    upd = float(nsh * (w.nts - 1) * 2 * (w.nz - 8) * (w.nx - 8))
    est = torch.cuda.ExternalStream(L.eio_ctx_stream(nl.ctx), device=dev)
    for _ in range(args.warmup):
        nl.forward(False, model, data)
    L.eio_ctx_stats(nl.ctx, 1, 1, None, None, None)
    barrier(ws)
    torch.cuda.synchronize()
    clocks = ClockSampler(None)
    clocks.start()
    t_ms = 0.0
    for _ in range(args.steps):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record(est)
        nl.forward(False, model, data)
        ev1.record(est)
        torch.cuda.synchronize()
        t_ms += ev0.elapsed_time(ev1)
    clk = clocks.stop()
    t_ms = max_over_ranks(ws, t_ms)
    value = ws * upd * args.steps / (t_ms * 1e-3) / 1e9
    peak, pk = measured_peak()
    n_model = int(np.prod(model.getNdArray().shape))
    n_data = int(np.prod(data.getNdArray().shape))
    return {"metric": "Gcells/s", "value": round(value, 3), "unit": "Gcell-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(t_ms / args.steps, 2),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "nl_shots: nonlinear forward of %d shots of the 312x520 case (nts=2000) per step, "
                                   "%s" % (nsh, "%d shots per lockstep launch" % args.batch if args.batch > 1
                                           else "one shot at a time on the lanes"),
                       "shots_per_gpu": nsh, "l2": "host buffers in and out every step (operator API)"},
            "e2e": {"value": round(value, 3), "unit": "Gcell-updates/s", "h2d_bytes_per_step": 4 * n_model,
                    "d2h_bytes_per_step": 4 * n_data, "note": "the operator API with host buffers"},
            "roofline": {"bound": "hbm", "achieved": round(BYTES_PER_CELL * value, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(BYTES_PER_CELL * value / peak, 4), "traffic": None, "peak_source": pk,
                         "basis": "80 B per cell update over the timed region (job level)"},
            "cpu_baseline": None, "clocks": clk, "gpu_launches": int(read_stats(L, nl.ctx)["launches"])}


def fwi_sample(args, ws, rank, local):
    """A bounded FWI-gradient measurement beside the default Born line: the
    batched-FWI case (1000x3400, nts = 5000, cropped shots of uneven 2-8 km
    windows, BF16 source-wavefield checkpoints, fused gradient), 8 of its 120
    shots per GPU, 1 warm-up and 2 timed steps whatever --steps says."""
    import copy
    import gc
    import torch
    gc.collect()
    torch.cuda.empty_cache()
    a = copy.copy(args)
    a.shots, a.steps, a.warmup, a.fwi_unfused = 8, 2, 1, False
    r = run_ours_fwi(a, ws, rank, local)
    return {"metric": "shot-gradients/s", "value": r["shot_gradients_per_s"], "unit": "shot-gradients/s",
            "roofline_frac": r["shot_gradient_roofline_frac"], "bytes_per_shot_gradient": r["shot_gradient_bytes"],
            "gcell_updates_per_s": r["value"], "ms_per_step": r["ms_per_step"], "steps": a.steps, "warmup": a.warmup,
            "workload": r["config"]["workload"], "shot_lanes": r["config"]["shot_lanes"],
            "peak": r["roofline"]["peak"], "clocks": r["clocks"],
            "basis": "per shot gradient: 2 propagations x 80 B x window cells x fine steps + window cells x nts x "
                     "(4 B BF16 snapshot write + 4 B read + 40 B image read-modify-write)"}


def main():
    args = parse()
    if args.impl == "reference":
        # rank 0 alone times the reference; the other ranks exit without work
        if int(os.environ.get("RANK", "0")) != 0:
            return 0
        print(json.dumps(run_reference(args, 1, 0, int(os.environ.get("LOCAL_RANK", "0")))))
        return 0
    ws, rank, local = dist_init(args)
    if args.workload == "nl_312x520":
        out = run_ours_nl(args, ws, rank, local)
    elif args.workload == "fwi_1000x3400":
        out = run_ours_fwi(args, ws, rank, local)
    elif args.workload == "nl_shots":
        out = run_ours_nl_shots(args, ws, rank, local)
    elif args.workload == "fwi_learned":
        out = run_ours_learned(args, ws, rank, local)
    elif args.workload == "fwi_cfg5":
        out = run_ours_cfg5(args, ws, rank, local)
    elif args.workload == "cnn_train":
        out = run_ours_cnn(args, ws, rank, local)
    else:
        out = run_ours(args, ws, rank, local)
        if not args.no_fwi:
            out["fwi"] = fwi_sample(args, ws, rank, local)
    if rank == 0:
        print(json.dumps(out))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
