"""Benchmark: pixels/s of Stokes synthesis + chi2 gradient w.r.t. 10 nodes on one B200.

Workload (the responses-and-adjoint configuration): 64 x 64 pixels, 80 depths (log tau500 -6..1),
201 wavelengths (Fe I 6301.5 / 6302.5, 12 mA), mu = 1, ten-node model (T x4, v_turb, v_los x2, B,
inclination, azimuth).  One step = one snapi_adjoint_nodes call over all pixels, from node vectors
to outputs: the node -> record build on the device (node interpolation, hydrostatic equilibrium with
the chemistry at every step, the record set-up; the node tangents by the reference's central
differences: 9 builds per pixel), then forward synthesis, chi2 against a noisy target and the
adjoint (reverse) sweep giving d chi2 / d node -- the work of the reference's build_from_nodes +
obs_stokes_responses_to_nodes, which its reference arm times.

Inputs: seeded config-3 node vectors (seed 3: the reference arm's pixels are the first ones of the
same generator); target = device synthesis of the truth + N(0, 1e-3 Ic); evaluated model = truth
+ fixed node offsets.  A step's working set (the adjoint's state, 8 GB, and the build scratch)
exceeds the 126 MB L2, so no flush is needed between steps.  Secondary keys: the adjoint alone on
device-resident records and packed node tangents (the record boundary), the plain FD gradient at
that boundary (2 npar + 1 solves) and from node vectors (2 npar + 1 builds + syntheses), the
measured FP32 / FP64 peaks and the rooflines of both phases.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl snapi|reference]

Prints one JSON line (rank 0).  --impl reference times the reference's own CPU implementation
(oracle/_ref/snapi_ref_bench, the reference sources compiled with their -O3 -ffast-math flags)
on the host cores for the same metric.
"""
import argparse
import json
import shutil
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
POOL = os.path.join(ROOT, "tests", "golden", "bench_pool.npz")
TASK = os.path.join(ROOT, "tests", "golden", "c3.tsk")
REF_BENCH = os.path.join(ROOT, "oracle", "_ref", "snapi_ref_bench")
METRIC = "pixels/s Stokes synth+grad on 1 B200, adjoint vs plain FD, at 1e-5 Ic"
NPIX = 64 * 64
FD_STEPS = np.array([5.0, 5.0, 5.0, 5.0, 2e3, 2e3, 2e3, 5.0, 5e-3, 5e-3])
# ncu (--set full) of the four adjoint kernels on 2048 pixels of this workload, per pixel:
# dram__bytes_read.sum + dram__bytes_write.sum
NCU_DRAM_BYTES_PER_PIXEL = 4.90e6
# Algorithmic work, frozen from `python oracle/opcount/count_flops.py --pixels 8` (op-count builds of
# the kernels' CPU emulator and of the FP64 node -> record restatement; profiles/flops_per_cell.md):
# flop per pixel of the adjoint call (forward + reverse, 3915 per wavelength x depth cell) and FP64
# flop per column of the node build with tangents (9 builds, continued chemistry start).
FLOPS = {"adjoint_flops_per_pixel": 6.296e7, "build_flops_per_column_with_tangents": 1.081e8}
# the evaluated model = truth + these offsets (T x4, v_turb, v_los x2, B, inclination, azimuth)
MODEL_OFFSET = np.array([0.0, 0.0, 0.0, 0.0, 0.3e5, 0.3e5, -0.3e5, 200.0, 0.1, 0.1])


def make_workload(pool, npix=NPIX, seed=3, return_nodes=False):
    """Per-pixel records / tangents / truth for the benchmark (see the module docstring); with
    return_nodes also the truth node vectors (T x4, v_turb, v_los x2, B, inclination, azimuth)."""
    rng = np.random.default_rng(seed)
    ncol = pool["record"].shape[0]
    col = rng.integers(0, ncol, npix)
    rec = pool["record"][col].astype(np.float32)
    tan = pool["tangent"][col].astype(np.float32)
    w1 = pool["tangent"][0, 5, :, 3].astype(np.float64)  # d v_los(depth) / d v_los node 1
    w2 = pool["tangent"][0, 6, :, 3].astype(np.float64)
    truth = {
        "vt": rng.uniform(0.5e5, 2.0e5, npix),
        "v1": rng.normal(0.0, 1.0e5, npix),
        "v2": rng.normal(0.0, 1.0e5, npix),
        "B": 10.0 ** rng.uniform(2.0, np.log10(2500.0), npix),
        "th": rng.uniform(np.deg2rad(20.0), np.deg2rad(160.0), npix),
        "ph": rng.uniform(np.deg2rad(10.0), np.deg2rad(170.0), npix),
    }

    def apply(r, p):
        r = r.copy()
        r[:, :, 1] = p["vt"][:, None]
        r[:, :, 3] = p["v1"][:, None] * w1[None, :] + p["v2"][:, None] * w2[None, :]
        r[:, :, 4] = p["B"][:, None]
        r[:, :, 5] = np.rad2deg(p["th"])[:, None]
        az = np.rad2deg(p["ph"])
        r[:, :, 6] = np.where(az > 90.0, az - 180.0, az)[:, None]  # atan quirk, atmos_rad.cc:45
        return r

    model = dict(truth)
    model["vt"] = truth["vt"] + 0.3e5
    model["v1"] = truth["v1"] + 0.3e5
    model["v2"] = truth["v2"] - 0.3e5
    model["B"] = truth["B"] + 200.0
    model["th"] = truth["th"] + 0.1
    model["ph"] = truth["ph"] + 0.1
    if return_nodes:
        nodes = np.concatenate([pool["nodes"][col, :4], np.stack([truth[k] for k in ("vt", "v1", "v2", "B", "th", "ph")],
                                                                 axis=1)], axis=1)
        return apply(rec, truth), apply(rec, model), tan, nodes
    return apply(rec, truth), apply(rec, model), tan


class ClockSampler:
    """nvidia-smi samples during the timed region (clocks and throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(prefix="clocks_", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.out.close()
        rows = [ln.split(",") for ln in open(self.out.name).read().strip().splitlines() if ln.strip()]
        os.unlink(self.out.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for n, v in zip(names, r[5:9]):
                if v.strip().lower() in ("active", "1"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def dist_setup(args=None, backend="nccl"):
    """One process per GPU (torchrun's RANK / WORLD_SIZE / LOCAL_RANK).  Pixels are independent, so
    the ranks only meet for barriers around the timed region and the max-over-ranks time."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def job_throughput(pixels_per_rank, ms_per_step, world, device):
    """Whole-job pixels/s: every rank's pixels over the slowest rank's step time."""
    ms = reduce_max(ms_per_step, world, device)
    return pixels_per_rank * world / (ms / 1e3), ms


def reduce_max(x, world, device):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def node_workload(npix, seed):
    """The headline workload's node vectors: seeded config-3 truth nodes (T x4 around 4600 / 4900 /
    5500 / 7400 K with N(0, 150 K), v_turb U(0.5, 2) km/s, v_los N(0, 1 km/s) x2, B log-uniform
    100-2500 G, inclination U(20, 160) deg, azimuth U(10, 170) deg; the reference arm's pixels are
    the first ones of the same generator) and the evaluated model = truth + fixed offsets."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import config3_nodes
    truth = config3_nodes(npix, seed=seed)
    return truth, truth + MODEL_OFFSET


def run_snapi(args):
    import torch

    sys.path.insert(0, ROOT)
    import snapi_b200 as sb
    from snapi_b200 import build as b

    world, rank, local = dist_setup(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    b.build_cuda()
    pool = dict(np.load(POOL))
    NPIX = args.pixels
    ic = float(pool["stokes"][:, :, 0].max())
    nl = pool["lambda_air"].shape[0]
    ctx = sb.Context.from_fixture(pool, stokes_scale=ic, max_batch=NPIX, device=local)
    ctx.eos_set(_eos_tables())
    # launch shapes timed on the first (warm-up) calls: the timed steps use the tuned ones; with
    # --tune-cache an earlier run's choices are read (and new ones appended)
    ctx.autotune(True, args.tune_cache)
    npar = ctx._eos_npar
    truth, model = node_workload(NPIX, seed=3 + 1000 * rank)
    # target: the device synthesis of the truth + N(0, 1e-3 Ic) (set-up, not timed)
    rec_t, _, _, _ = ctx.build_records(truth, tangents=False)
    obs = ctx.synth(rec_t)
    obs += np.random.default_rng(77 + rank).normal(0.0, 1e-3 * ic, obs.shape).astype(np.float32)
    del rec_t
    d_nodes = torch.from_numpy(np.ascontiguousarray(model)).to(dev)
    d_obs = torch.from_numpy(obs).to(dev)
    d_chi2 = torch.zeros(NPIX, dtype=torch.float64, device=dev)
    d_grad = torch.zeros(NPIX, npar, dtype=torch.float64, device=dev)
    d_st = torch.zeros(NPIX, nl, 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    torch.cuda.synchronize()

    def step():
        ctx.adjoint_nodes_device(NPIX, d_nodes.data_ptr(), d_obs.data_ptr(), d_chi2.data_ptr(), d_grad.data_ptr(),
                                 stokes_ptr=d_st.data_ptr())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(local)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    phase = np.zeros(2)
    launches = 0
    torch.cuda.synchronize()
    ev0.record(stream)
    torch.cuda.nvtx.range_push("timed_steps")  # ncu --nvtx --nvtx-include timed_steps/ selects these launches
    for _ in range(args.steps):
        step()
        phase += np.array(ctx.last_phase_ms)
        launches += ctx.last_launches
    torch.cuda.nvtx.range_pop()
    ev1.record(stream)
    torch.cuda.synchronize()
    total_ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()
    barrier(world)
    value, ms_step = job_throughput(NPIX, total_ms / args.steps, world, dev)
    build_ms, adj_ms = phase / args.steps

    # end to end through the host API: page-locked node vectors and targets in, Stokes / chi2 /
    # gradient out, every step (snapi_adjoint_nodes with host arrays)
    h_nodes = np.frombuffer(ctypes_buffer(ctx, model.nbytes), dtype=np.float64).reshape(model.shape)
    h_nodes[...] = model
    h_obs = np.frombuffer(ctypes_buffer(ctx, obs.nbytes), dtype=np.float32).reshape(obs.shape)
    h_obs[...] = obs
    h_out = {"stokes": np.frombuffer(ctypes_buffer(ctx, 4 * NPIX * nl * 4), dtype=np.float32).reshape(NPIX, nl, 4),
             "chi2": np.frombuffer(ctypes_buffer(ctx, 8 * NPIX), dtype=np.float64),
             "grad": np.frombuffer(ctypes_buffer(ctx, 8 * NPIX * npar), dtype=np.float64).reshape(NPIX, npar),
             "status": np.frombuffer(ctypes_buffer(ctx, 4 * NPIX), dtype=np.int32)}
    ctx.adjoint_nodes(h_nodes, h_obs, out=h_out)
    torch.cuda.synchronize()
    barrier(world)
    ne = max(1, args.steps // 2)
    ev0.record(stream)
    for _ in range(ne):
        out = ctx.adjoint_nodes(h_nodes, h_obs, out=h_out)
    ev1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = reduce_max(ev0.elapsed_time(ev1) / ne, world, dev)
    h2d = model.nbytes + obs.nbytes
    d2h = out["stokes"].nbytes + out["chi2"].nbytes + out["grad"].nbytes + out["status"].nbytes
    flagged = int((out["status"] != 0).sum())

    # the record boundary (snapi_adjoint_packed on device-resident records and packed node tangents,
    # built once from the same nodes): the adjoint alone, and the plain FD gradient it replaces
    rec_m, tan_m, _, _ = ctx.build_records(model, tangents=True)
    fmask = sb.tangent_field_mask(tan_m)
    ptan = sb.pack_tangents(tan_m, fmask)
    d_rec = torch.from_numpy(rec_m).to(dev)
    d_tan = torch.from_numpy(tan_m).to(dev)
    d_ptan = torch.from_numpy(ptan).to(dev)
    del tan_m

    def rec_step():
        ctx.adjoint_packed_device(NPIX, d_rec.data_ptr(), d_obs.data_ptr(), fmask, d_ptan.data_ptr(),
                                  d_chi2.data_ptr(), d_grad.data_ptr(), stokes_ptr=d_st.data_ptr())

    def fd_step():
        ctx.fd_grad_device(NPIX, d_rec.data_ptr(), d_obs.data_ptr(), npar, d_tan.data_ptr(), FD_STEPS,
                           d_chi2.data_ptr(), d_grad.data_ptr())

    def timed(fn, n):
        fn()
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(n):
            fn()
        ev1.record(stream)
        torch.cuda.synchronize()
        return reduce_max(ev0.elapsed_time(ev1) / n, world, dev)

    rec_ms = timed(rec_step, args.steps)
    fd_ms = timed(fd_step, max(1, args.steps // 5))

    # plain FD from the node vectors: 2 npar + 1 builds (records only) and syntheses, chi2 each
    d_nfd = torch.empty_like(d_nodes)
    d_rfd = torch.empty_like(d_rec)

    def fd_nodes_step():
        g = []
        for q in range(-1, npar):
            for sgn in ((0.0,) if q < 0 else (0.5, -0.5)):
                with torch.cuda.stream(stream):
                    d_nfd.copy_(d_nodes)
                    if q >= 0:
                        d_nfd[:, q] += sgn * FD_STEPS[q]
                ctx.build_records_device(NPIX, d_nfd.data_ptr(), d_rfd.data_ptr())
                ctx.synth_device(NPIX, d_rfd.data_ptr(), d_st.data_ptr())
                with torch.cuda.stream(stream):
                    g.append(((d_obs - d_st) ** 2).sum(dim=(1, 2)))
        return g

    fdn_ms = timed(fd_nodes_step, 1)
    del d_rec, d_tan, d_ptan, d_rfd

    line = None
    if rank == 0:
        peaks = load_peaks()
        fp32 = sb.api.fma_peak(local, fp64=False)
        fp64 = sb.api.fma_peak(local, fp64=True)
        adj_tf = FLOPS["adjoint_flops_per_pixel"] * NPIX / (adj_ms / 1e3) / 1e12
        bld_tf = FLOPS["build_flops_per_column_with_tangents"] * NPIX / (build_ms / 1e3) / 1e12
        r_adj = {"bound": "fp32", "achieved": adj_tf, "peak": fp32, "unit": "TFLOP/s", "frac": adj_tf / fp32,
                 "traffic": NCU_DRAM_BYTES_PER_PIXEL * NPIX,
                 "kernel": "adjoint (k_adj_forward + k_adj_rt + k_adj_opacity + k_adjoint_finish)",
                 "ms_per_launch": adj_ms, "peak_source": "measured on this GPU (snapi_fma_peak, FP32 FMA chains)",
                 "flops": "algorithmic: %.4g flop per pixel from the op-count build of the kernels' CPU emulator "
                          "(oracle/opcount; 3915 per wavelength x depth cell)" % FLOPS["adjoint_flops_per_pixel"],
                 "traffic_note": "ncu DRAM bytes of the four adjoint kernels per pixel (2048-pixel capture) x pixels"}
        r_bld = {"bound": "fp64", "achieved": bld_tf, "peak": fp64, "unit": "TFLOP/s", "frac": bld_tf / fp64,
                 "traffic": None, "kernel": "node build (k_eos_he + k_eos_var + k_eos_rec)", "ms_per_launch": build_ms,
                 "peak_source": "measured on this GPU (snapi_fma_peak, FP64 FMA chains)",
                 "flops": "algorithmic upper bound: %.4g FP64 flop per column with tangents (9 builds) from the "
                          "op-count build of the FP64 restatement, continued chemistry start (oracle/opcount)"
                          % FLOPS["build_flops_per_column_with_tangents"],
                 "bound_note": "a serial chemistry chain per column (latency-bound)"}
        dominant = r_bld if build_ms >= adj_ms else r_adj
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "pixels/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 (profiles, formal solver, adjoint); f64 (chemistry, hydrostatic equilibrium, optical depth)",
            "data": "synthetic: seeded config-3 node vectors (seed 3); target = device synthesis of the truth + "
                    "N(0, 1e-3 Ic); evaluated at truth + fixed offsets",
            "config": {"workload": workload_name(NPIX), "pixels_per_gpu": NPIX, "nd": int(ctx.nd),
                       "nlambda": int(nl), "npar": int(npar),
                       "step": "snapi_adjoint_nodes: node vectors -> records + node tangents (hydrostatic "
                               "equilibrium + chemistry, 9 builds per pixel) -> synthesis + chi2 + adjoint "
                               "d chi2 / d nodes, all on the device",
                       "chem_start": "continued in the hydrostatic march (SNAPI_CHEM_START_CONTINUE)",
                       "launch_shapes": "autotuned in the warm-up steps (snapi_autotune)",
                       "l2_flush": "a step's working set (adjoint state 8 GB, build scratch) exceeds the 126 MB L2",
                       "parallelism": "replicas (pixels independent)"},
            "gpu_launches": launches,
            "clocks": clk,
            "e2e": {"value": NPIX * world / (e2e_ms / 1e3), "unit": "pixels/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
            "phases_ms": {"node_build": build_ms, "adjoint": adj_ms},
            "roofline": dominant,
            "rooflines": {"adjoint": r_adj, "node_build": r_bld},
            "record_boundary": {"value": NPIX * world / (rec_ms / 1e3), "unit": "pixels/s", "ms_per_step": rec_ms,
                                "what": "snapi_adjoint_packed on device-resident records + packed node tangents "
                                        "(the adjoint alone)"},
            "fd_baseline": {"record_boundary": {"value": NPIX * world / (fd_ms / 1e3), "unit": "pixels/s",
                                                "ms_per_step": fd_ms, "solves_per_gradient": 2 * npar + 1,
                                                "adjoint_speedup": fd_ms / rec_ms},
                            "from_nodes": {"value": NPIX * world / (fdn_ms / 1e3), "unit": "pixels/s",
                                           "ms_per_step": fdn_ms,
                                           "what": "2 npar + 1 node-vector builds (records only) + syntheses",
                                           "adjoint_speedup": fdn_ms / ms_step}},
            "measured_peaks": {"fp32_fma_tflops": fp32, "fp64_fma_tflops": fp64, "hbm_gbs": peaks["hbm_gbs"],
                               "hbm_source": peaks["source"]},
            "flagged_columns": flagged,
            "tuned_shapes": ctx.tuned_config(NPIX)[0],
        }
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = reference_cpu_rate(samples_per_core=1, mode=1)
    if rank == 0 and not args.no_extras:
        line["lm"] = bench_lm(sb, pool, ic, local)
        line["node_build"] = bench_build(sb, pool, local)
        line["lm_device_build"] = bench_lm_device(sb, pool, ic, local)
        line["ali"] = bench_ali(sb, local, cpu=not args.no_cpu_baseline)
        line["cube_invert"] = bench_cube(sb, pool, ic, local, n=64)
        line["cube_synth"] = bench_cube_synth(sb, pool, local, n=256)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return line


def bench_lm(sb, pool, ic, device, npix=4096, iters=10):
    """Device time of the batched LM (snapi_lm_step): 10-node fits of npix pixels from offset
    starting nodes, with the Jacobian by central differences and by the forward-mode sweeps.  The
    node -> record map between steps is the caller's; here it is the records' linearisation along
    the node tangents (numpy, not timed on the device)."""
    out = {}
    for mode, key in ((sb.api.JACOBIAN_FD, "fd_jacobian"), (sb.api.JACOBIAN_TANGENT, "tangent_jacobian")):
        out[key] = _bench_lm_mode(sb, pool, ic, device, npix, iters, mode)
    out["tangent_speedup"] = out["fd_jacobian"]["device_ms_per_step"] / out["tangent_jacobian"]["device_ms_per_step"]
    return out


def _bench_lm_mode(sb, pool, ic, device, npix, iters, mode):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from ref_builder import LinearBuilder
    truth, _, tan, nodes_t = make_workload(pool, npix, seed=11, return_nodes=True)
    build = LinearBuilder(truth, tan, nodes_t)
    ctx = sb.Context.from_fixture(pool, stokes_scale=ic, max_batch=npix, device=device)
    ctx.jacobian_mode(mode)
    obs = ctx.synth(truth)
    obs += np.random.default_rng(12).normal(0.0, 1e-3 * ic, obs.shape).astype(np.float32)
    kinds = pool["node_kind"].astype(int)
    scale = np.array([{1: 5000.0, 2: 1e5, 3: 1e5, 4: 1000.0}.get(k, 1.0) for k in kinds])
    n0 = nodes_t + np.array([200.0, 200.0, 200.0, 200.0, 3e4, 3e4, 3e4, 200.0, 0.1, 0.1])
    req = ctx.lm_begin(n0, obs, kinds, 1e-2 * scale, lm_start=1e3, max_iter=iters, delta=1e-4)
    dev_ms, steps, active = 0.0, 0, np.ones(npix, bool)
    t0 = time.perf_counter()
    while True:
        rec, tn = build(req, active)
        req, active, n = ctx.lm_step(rec, tn)
        dev_ms += ctx.last_kernel_ms
        steps += 1
        if n == 0:
            break
    wall = time.perf_counter() - t0
    res = ctx.lm_result()
    ctx.close()
    return {"pixels": npix, "npar": int(tan.shape[1]), "steps": steps, "device_ms_per_step": dev_ms / steps,
            "device_pixel_steps_per_s": npix * steps / (dev_ms / 1e3), "wall_s_with_host_linear_builder": wall,
            "median_iterations": float(np.median(res["iters"])),
            "note": "device work per step: synthesis at the trial nodes, Jacobian at accepted nodes (2 npar "
                    "solves, or one state pass + the forward-mode sweeps), J^T J / J^T r on the tcgen05 tensor "
                    "cores (3xTF32 split, FP32 accumulation), FP64 damped eigen-solve; node -> record map on the "
                    "host"}


def _eos_tables():
    from snapi_b200.eos_tables import EosTables
    return EosTables(dict(np.load(os.path.join(ROOT, "tests", "golden", "eos_c3.npz"))))


def bench_build(sb, pool, device, ncol=4096):
    """Node model -> column records on the GPU (snapi_build_records): hydrostatic equilibrium with
    the chemistry per depth, the record set-up, and the node tangents (two builds per temperature
    node, 9 builds per column for 4 temperature nodes), for the 32 seeded config-3 node vectors
    tiled to ncol columns.  The reference's build_from_nodes time per column (compiled reference,
    strict FP64, one core) is the fixture's."""
    nodes = np.tile(pool["nodes"], (ncol // pool["nodes"].shape[0] + 1, 1))[:ncol]
    ctx = sb.Context.from_fixture(pool, max_batch=4096, device=device)
    ctx.eos_set(_eos_tables())
    ctx.build_records(nodes, tangents=True)  # warm-up (allocates the work buffers)
    out = {}
    for start, tag in ((sb.api.CHEM_START_CONTINUE, ""), (sb.api.CHEM_START_COLD, "_cold_start")):
        ctx.eos_chem_start(start)
        for tang in (False, True):
            t0 = time.perf_counter()
            _, _, _, status = ctx.build_records(nodes, tangents=tang)
            wall = time.perf_counter() - t0
            key = ("with_tangents" if tang else "records_only") + tag
            out[key] = {"device_ms": ctx.last_kernel_ms, "wall_ms": wall * 1e3,
                        "columns_per_s": ncol / (ctx.last_kernel_ms / 1e3), "flagged": int((status != 0).sum())}
    ctx.close()
    ref_build = float(pool["ref_seconds_per_pixel"][0])
    out["columns"] = ncol
    out["reference_build_s_per_column_one_core"] = ref_build
    out["reference_columns_per_s_one_core_with_tangents"] = 1.0 / (ref_build * 9)
    out["note"] = ("flagged: columns where a hydrostatic step reached the reference's own 20-pass cap "
                   "(status 2, the reference continues the same way); *_cold_start: every chemistry solve "
                   "started as the reference starts it (SNAPI_CHEM_START_COLD)")
    return out


def bench_lm_device(sb, pool, ic, device, npix=1024, iters=10):
    """The whole stokes_lm_fit on the GPU (snapi_lm_fit): every step builds records and tangents of
    the requested nodes on the device and takes one LM iteration; npix pixels, 10 nodes, iters
    iterations from offset starting nodes against noisy targets synthesised from the pool's nodes;
    with the Jacobian by central differences and by the forward-mode sweeps."""
    out = {}
    for mode, key in ((sb.api.JACOBIAN_FD, "fd_jacobian"), (sb.api.JACOBIAN_TANGENT, "tangent_jacobian")):
        out[key] = _bench_lm_device_mode(sb, pool, ic, device, npix, iters, mode)
    return out


def _bench_lm_device_mode(sb, pool, ic, device, npix, iters, mode):
    nodes = np.tile(pool["nodes"], (npix // pool["nodes"].shape[0] + 1, 1))[:npix]
    ctx = sb.Context.from_fixture(pool, stokes_scale=ic, max_batch=4096, device=device)
    ctx.eos_set(_eos_tables())
    ctx.jacobian_mode(mode)
    rec, _, _, _ = ctx.build_records(nodes, tangents=False)
    obs = ctx.synth(rec)
    obs += np.random.default_rng(13).normal(0.0, 1e-3 * ic, obs.shape).astype(np.float32)
    kinds = pool["node_kind"].astype(int)
    scale = np.array([{1: 5000.0, 2: 1e5, 3: 1e5, 4: 1000.0}.get(k, 1.0) for k in kinds])
    n0 = nodes + np.array([200.0, 200.0, 200.0, 200.0, 3e4, 3e4, 3e4, 200.0, 0.1, 0.1])
    t0 = time.perf_counter()
    res = ctx.lm_fit_device(n0, obs, kinds, 1e-2 * scale, lm_start=1e3, max_iter=iters, delta=1e-4)
    wall = time.perf_counter() - t0
    dev = ctx.last_kernel_ms
    ctx.close()
    return {"pixels": npix, "iterations": iters, "steps": res["steps"], "device_s": dev / 1e3, "wall_s": wall,
            "device_ms_per_step": dev / res["steps"], "pixel_steps_per_s": npix * res["steps"] / (dev / 1e3),
            "median_iterations": float(np.median(res["iters"]))}


def bench_cube(sb, pool, ic, device, n=64, iters=30, chunk=0):
    """The master's invert job (snapi_cube_invert) over an n x n float32 .f0 cube: noisy Stokes
    synthesised on the GPU from the pool's node vectors tiled over the cube, every pixel started from
    the same node vector (the job's model) and fitted for up to iters iterations, the cube streamed
    from the file in chunks while the GPU fits, the node cube and float64 spectra written back."""
    npix = n * n
    nodes = np.tile(pool["nodes"], (npix // pool["nodes"].shape[0] + 1, 1))[:npix]
    ctx = sb.Context.from_fixture(pool, stokes_scale=ic, max_batch=4096, device=device)
    ctx.eos_set(_eos_tables())
    rec, _, _, _ = ctx.build_records(nodes, tangents=False)
    obs = ctx.synth(rec)
    del rec
    obs += np.random.default_rng(14).normal(0.0, 1e-3 * ic, obs.shape).astype(np.float32)
    nl = obs.shape[1]
    kinds = pool["node_kind"].astype(int)
    scale = np.array([{1: 5000.0, 2: 1e5, 3: 1e5, 4: 1000.0}.get(k, 1.0) for k in kinds])
    start = pool["nodes"].mean(axis=0) + np.array([200.0, 200.0, 200.0, 200.0, 3e4, 3e4, 3e4, 200.0, 0.1, 0.1])
    tmp = tempfile.mkdtemp(prefix="snapi_cube_")
    try:
        path = os.path.join(tmp, "obs.f0")
        sb.api.f0_write(path, np.ascontiguousarray(obs.reshape(n, n, nl, 4).transpose(0, 1, 3, 2)))
        del obs
        out = ctx.cube_invert(path, kinds, 1e-2 * scale, nodes0=start, out_nodes=os.path.join(tmp, "nodes.f0"),
                              out_spectra=os.path.join(tmp, "spectra.f0"), chunk=chunk, lm_start=1e3,
                              max_iter=iters, delta=1e-4)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    ctx.close()
    st = out["stats"]
    return {"cube": [n, n], "pixels": npix, "chunks": st["chunks"], "iterations": iters, "lm_steps": st["lm_steps"],
            "wall_s": st["wall_s"], "fit_s": st["fit_s"], "read_wait_s": st["read_wait_s"],
            "write_wait_s": st["write_wait_s"], "device_s": st["kernel_ms"] / 1e3,
            "pixels_per_s": npix / st["wall_s"], "bytes_read": st["bytes_read"], "bytes_written": st["bytes_written"],
            "median_iterations": float(np.median(out["iters"])),
            "note": "wall_s covers the whole job: reads, fits and writes; read / write waits are the I/O "
                    "not hidden behind the fits"}


def bench_cube_synth(sb, pool, device, n=256, chunk=0):
    """The synthesis branch of the master's job (snapi_cube_synth) over an n x n float64 atmosphere
    cube in the 12-row layout (the columns of the pool's node vectors tiled over the cube, built on
    the GPU by snapi_build_atmos), streamed from the file through records and synthesis to the
    float64 spectra file."""
    npix = n * n
    ctx = sb.Context.from_fixture(pool, max_batch=4096, device=device)
    ctx.eos_set(_eos_tables())
    cols, _ = ctx.build_atmos(pool["nodes"])
    cols = cols[np.arange(npix) % cols.shape[0]]
    tmp = tempfile.mkdtemp(prefix="snapi_synth_")
    try:
        path = os.path.join(tmp, "atmos.f0")
        sb.api.f0_write(path, np.ascontiguousarray(cols.reshape(n, n, 12, -1).transpose(2, 0, 1, 3)))
        del cols
        out = ctx.cube_synth(path, out_spectra=os.path.join(tmp, "spectra.f0"), chunk=chunk, want_stokes=False)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    ctx.close()
    st = out["stats"]
    return {"cube": [n, n], "pixels": npix, "chunks": st["chunks"], "wall_s": st["wall_s"], "gpu_s": st["fit_s"],
            "device_s": st["kernel_ms"] / 1e3, "read_wait_s": st["read_wait_s"], "write_wait_s": st["write_wait_s"],
            "pixels_per_s": npix / st["wall_s"], "bytes_read": st["bytes_read"], "bytes_written": st["bytes_written"],
            "flagged": st["flagged"],
            "note": "wall_s covers reading the atmosphere cube, records, synthesis and writing the spectra; "
                    "read / write waits are the I/O not hidden behind the GPU work"}


def bench_ali(sb, device, ncol=1024, cpu=True):
    """NLTE Ca II populations (snapi_ali_iter) for ncol columns to the reference's convergence
    criterion (max relative change < 1e-2): the three reference-built columns of
    tests/golden/config5.npz tiled to ncol (80 depths, 444 NLTE wavelengths, 2 rays)."""
    fx = dict(np.load(os.path.join(ROOT, "tests", "golden", "config5.npz")))
    ctx = sb.api.AliContext.from_fixture(fx, device=device)
    cols = ctx.columns_from_fixture(fx)
    idx = np.arange(ncol) % fx["ali_T"].shape[0]
    cols = {k: np.ascontiguousarray(v[idx]) for k, v in cols.items()}
    pops0 = np.ascontiguousarray(fx["ali_pop0"][idx])
    ctx.iterate({k: v[:8] for k, v in cols.items()}, pops0[:8], max_iter=2, tol=1e-2)  # warm-up
    t0 = time.perf_counter()
    pops, rel, iters, st = ctx.iterate(cols, pops0, max_iter=100, tol=1e-2)
    wall = time.perf_counter() - t0
    dev_ms = ctx.last_kernel_ms
    ctx.close()
    out = {"columns": ncol, "nd": int(fx["ali_T"].shape[1]), "nlambda": int(fx["ali_lambda"].shape[0]),
           "rays": int(fx["ali_th"].shape[0]), "levels": int(fx["ali_A"].shape[0]),
           "iterations_max": int(iters.max()), "device_ms": dev_ms, "columns_per_s_device": ncol / (dev_ms / 1e3),
           "columns_per_s_e2e": ncol / wall, "max_rel_to_reference_converged":
               float(np.abs(pops[:3] / fx["ali_pop_conv"] - 1.0).max()), "negative_columns": int((st < 0).sum())}
    out["from_columns"] = bench_ali_from_columns(sb, device, fx, ncol)
    if cpu:
        out["reference_cpu"] = reference_ali_rate()
    # config 5 at its stated settings: 10 ray directions (5-point Gauss set), 100 depths, the 1e-4
    # population stop (the patched reference build); the six columns of tests/golden/config5_spec.npz
    # tiled, from columns with the set-up on the device
    fs = dict(np.load(os.path.join(ROOT, "tests", "golden", "config5_spec.npz")))
    spec = bench_ali_from_columns(sb, device, fs, ncol, tol=1e-4)
    spec.update({"columns": ncol, "nd": int(fs["ali_T"].shape[1]), "rays": int(fs["ali_th"].shape[0]),
                 "tol": 1e-4})
    if cpu:
        spec["reference_cpu"] = reference_ali_rate(spec=True)
    out["spec"] = spec
    return out


def bench_ali_from_columns(sb, device, fx, ncol, tol=1e-2):
    """The same populations from atmosphere columns alone, everything on the device: the columns
    (12 return_as_array rows, float64) from pinned host memory, the population-independent set-up
    (snapi_ali_setup: chemistry, LTE background per ray and wavelength, rates), the iteration, the
    populations back to the host."""
    import torch
    from snapi_b200.eos_tables import EosTables
    dev = torch.device("cuda", device)
    ctx = sb.Context.from_fixture(fx, device=device)
    ctx.eos_set(EosTables({k[4:]: v for k, v in fx.items() if k.startswith("eos_")}))
    ali = sb.api.AliContext.from_fixture(fx, device=device)
    tabs = sb.api.AliSetupTables.from_fixture(fx)
    idx = np.arange(ncol) % fx["alis_atm"].shape[0]
    h_cols = torch.from_numpy(np.ascontiguousarray(fx["alis_atm"][idx])).pin_memory()
    sh = ali.column_shapes(ncol)
    out = {n: torch.empty(sh[n], dtype=torch.float64, device=dev) for n in sh}
    ptrs = {n: out[n].data_ptr() for n in sh if n != "pops"}
    d_cols = torch.empty(h_cols.shape, dtype=torch.float64, device=dev)
    h_pops = torch.empty(sh["pops"], dtype=torch.float64).pin_memory()
    st = torch.zeros(ncol, dtype=torch.int32, device=dev)

    def run(n, max_iter=100):
        d_cols[:n].copy_(h_cols[:n], non_blocking=True)
        torch.cuda.synchronize(dev)
        ali.setup_device(ctx, tabs, n, d_cols.data_ptr(), ptrs, out["pops"].data_ptr())
        setup_ms = ctx.last_kernel_ms
        ali.iterate_device(n, ptrs, out["pops"].data_ptr(), max_iter=max_iter, tol=tol, status_ptr=st.data_ptr())
        h_pops[:n].copy_(out["pops"][:n])
        torch.cuda.synchronize(dev)
        return setup_ms, ali.last_kernel_ms

    run(ncol, max_iter=1)  # warm-up: the contexts' work buffers sized for ncol columns
    t0 = time.perf_counter()
    setup_ms, iter_ms = run(ncol)
    wall = time.perf_counter() - t0
    pops = h_pops.numpy()
    res = {"setup_device_ms": setup_ms, "iterate_device_ms": iter_ms,
           "columns_per_s_device": ncol / ((setup_ms + iter_ms) / 1e3), "columns_per_s_e2e": ncol / wall,
           "h2d_bytes": int(h_cols.numel() * 8), "d2h_bytes": int(pops.size * 8),
           "max_rel_to_reference_converged":
               float(np.abs(pops[:fx["ali_pop_conv"].shape[0]] / fx["ali_pop_conv"] - 1.0).max()),
           "negative_columns": int((st < 0).sum())}
    ctx.close()
    ali.close()
    return res


def reference_ali_rate(cores=None, spec=False):
    """The reference's nltepops on config-5 columns, one process per host core (one column each);
    spec: the patched build at the configuration's stated settings (10 rays, 100 depths, 1e-4)."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import config3_nodes
    from sbin import read_sbin
    dump = os.path.join(ROOT, "oracle", "_ref", "snapi_ref_dump_spec" if spec else "snapi_ref_dump")
    task = os.path.join(ROOT, "tests", "golden", "c5_spec.tsk" if spec else "c5.tsk")
    if not os.path.exists(dump):
        return None
    ncores = cores or os.cpu_count() or 1
    nodes = config3_nodes(ncores, seed=5)
    tmp = tempfile.mkdtemp(prefix="snapi_ali_ref_")
    procs = []
    for i in range(ncores):
        nf = os.path.join(tmp, "n%d.f64" % i)
        nodes[i:i + 1].astype("<f8").tofile(nf)
        procs.append(subprocess.Popen([dump, "ali", task, nf, "1", "0", os.path.join(tmp, "o%d.sbin" % i)],
                                      stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL))
    ok = all(p.wait() == 0 for p in procs)
    secs = [float(read_sbin(os.path.join(tmp, "o%d.sbin" % i))["ali_ref_seconds"][0]) for i in range(ncores)] if ok \
        else []
    for f in os.listdir(tmp):
        os.unlink(os.path.join(tmp, f))
    os.rmdir(tmp)
    if not ok:
        return None
    return {"columns_per_s": ncores / max(secs), "cores": ncores, "seconds_per_column_mean": float(np.mean(secs)),
            "kind": "reference", "sample": "%d seeded config-5 columns, atmosphere::nltepops (strict FP64 build%s), "
                                          "one process per core" % (ncores, ", patched to 10 rays and the 1e-4 stop"
                                                                    if spec else "")}


def ctypes_buffer(ctx, nbytes):
    import ctypes

    import snapi_b200 as sb
    p = sb.lib().snapi_host_alloc(nbytes)
    if not p:
        raise MemoryError("snapi_host_alloc")
    return (ctypes.c_char * nbytes).from_address(p)


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return {"hbm_gbs": float(d["hbm_gbs"]), "bf16_tflops": float(d["bf16_tflops"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


def reference_cpu_rate(samples_per_core=1, mode=1, cores=None):
    """Run the reference's own CPU code (oracle/_ref/snapi_ref_bench) as one process per host
    core, the reference's islave model, on seeded config-3 pixels."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from make_golden import config3_nodes
    ncores = cores or os.cpu_count() or 1
    npix = ncores * samples_per_core
    nodes = config3_nodes(npix, seed=3)
    nf = tempfile.NamedTemporaryFile(suffix=".f64", delete=False)
    nodes.astype("<f8").tofile(nf.name)
    t0 = time.perf_counter()
    procs = [subprocess.Popen([REF_BENCH, TASK, nf.name, str(i * samples_per_core), str(samples_per_core), str(mode)],
                              stdout=subprocess.PIPE, stderr=subprocess.DEVNULL) for i in range(ncores)]
    outs = [p.communicate()[0].decode() for p in procs]
    wall = time.perf_counter() - t0
    os.unlink(nf.name)
    ok = all(p.returncode == 0 for p in procs) and all(o.startswith("pixels") for o in outs)
    what = {0: "obs_stokes", 1: "obs_stokes_responses_to_nodes", 2: "obs_stokes_num_responses_to_nodes"}[mode]
    return {"value": npix / wall if ok else None, "unit": "pixels/s", "cores": ncores, "kind": "reference",
            "sample": "%d seeded config-3 pixels (%d per core), build_from_nodes + %s, reference sources "
                      "compiled -O3 -ffast-math, one process per core" % (npix, samples_per_core, what),
            "wall_s": wall}


def workload_name(npix):
    return (("64x64" if npix == 64 * 64 else str(npix)) + " pixels x 80 depths x 201 wavelengths, Fe I 6301.5/6302.5, "
            "mu=1, 10 nodes (T x4, vturb, vlos x2, B, incl, azi): synthesis + chi2 + adjoint d chi2/d nodes")


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    ncores = os.cpu_count() or 1
    for _ in range(args.warmup):
        reference_cpu_rate(samples_per_core=1, mode=1, cores=ncores)
    t0 = time.perf_counter()
    tot = 0
    last = None
    for _ in range(args.steps):
        last = reference_cpu_rate(samples_per_core=1, mode=1, cores=ncores)
        tot += ncores
    wall = time.perf_counter() - t0
    value = tot / wall
    cpu = dict(last)
    cpu["value"] = value
    return {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": "pixels/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": wall / args.steps * 1e3,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: seeded node models of the workload's distribution (seed 3); the reference builds "
                "the columns itself",
        "config": {"workload": workload_name(NPIX),
                   "sample": "each step a bounded sample of that workload: %d of its pixels (one per host core), "
                             "each through the reference's build_from_nodes + obs_stokes_responses_to_nodes "
                             "(synthesis + node responses, the quantities the gradient needs)" % ncores,
                   "pixels_per_step": ncores, "parallelism": "one process per host core"},
        "cpu_baseline": cpu,
        "e2e": {"value": value, "unit": "pixels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="snapi", choices=["snapi", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--tune-cache", default=None, help="autotuner cache file (snapi_autotune)")
    ap.add_argument("--pixels", type=int, default=NPIX, help="pixels per GPU (smaller cases for profiling)")
    ap.add_argument("--no-extras", action="store_true", help="skip the LM and NLTE measurements")
    ap.add_argument("--node-build-only", type=int, default=0, metavar="N",
                    help="only measure the node -> record build of N columns (profiling)")
    ap.add_argument("--lm-fit-only", type=int, default=0, metavar="N",
                    help="only measure the whole LM on the device (snapi_lm_fit) for N pixels, 30 iterations")
    ap.add_argument("--cube-only", type=int, default=0, metavar="N",
                    help="only measure the invert job (snapi_cube_invert) over an N x N .f0 cube")
    ap.add_argument("--cube-chunk", type=int, default=0, help="pixels per GPU batch of the invert job")
    ap.add_argument("--cube-synth-only", type=int, default=0, metavar="N",
                    help="only measure the synthesis job (snapi_cube_synth) over an N x N atmosphere cube")
    ap.add_argument("--ali-only", type=int, default=0, metavar="N",
                    help="only measure the NLTE populations of N columns (snapi_ali_iter; from columns with "
                         "snapi_ali_setup)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.node_build_only:
        sys.path.insert(0, ROOT)
        import snapi_b200 as sb
        from snapi_b200 import build as b
        b.build_cuda()
        print(json.dumps({"node_build": bench_build(sb, dict(np.load(POOL)), 0, ncol=args.node_build_only)}), flush=True)
        return
    if args.lm_fit_only:
        sys.path.insert(0, ROOT)
        import snapi_b200 as sb
        from snapi_b200 import build as b
        b.build_cuda()
        pool = dict(np.load(POOL))
        ic = float(pool["stokes"][:, :, 0].max())
        print(json.dumps({"lm_device_build": bench_lm_device(sb, pool, ic, 0, npix=args.lm_fit_only, iters=30)}),
              flush=True)
        return
    if args.cube_synth_only:
        sys.path.insert(0, ROOT)
        import snapi_b200 as sb
        from snapi_b200 import build as b
        b.build_cuda()
        pool = dict(np.load(POOL))
        print(json.dumps({"cube_synth": bench_cube_synth(sb, pool, 0, n=args.cube_synth_only,
                                                         chunk=args.cube_chunk)}), flush=True)
        return
    if args.ali_only:
        sys.path.insert(0, ROOT)
        import snapi_b200 as sb
        from snapi_b200 import build as b
        b.build_cuda()
        print(json.dumps({"ali": bench_ali(sb, 0, ncol=args.ali_only, cpu=not args.no_cpu_baseline)}), flush=True)
        return
    if args.cube_only:
        sys.path.insert(0, ROOT)
        import snapi_b200 as sb
        from snapi_b200 import build as b
        b.build_cuda()
        pool = dict(np.load(POOL))
        ic = float(pool["stokes"][:, :, 0].max())
        print(json.dumps({"cube_invert": bench_cube(sb, pool, ic, 0, n=args.cube_only, chunk=args.cube_chunk)}),
              flush=True)
        return
    line = run_reference(args) if args.impl == "reference" else run_snapi(args)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
