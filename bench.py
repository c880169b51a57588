"""Benchmark of the B200 direction-iterative gain solver.

Workload (one "step" = one solution interval solved to tolerance 1e-5 or the
iteration cap, from unit initial solutions, as DDECal does without solution
propagation): 62 stations in a 2 km disk (1891 baselines), 10 directions of 20
point sources, 240 channels at 120-160 MHz in 24 channel blocks, 8 time steps
of 10 s, XX/YY complex64 visibilities, step size 0.2, at most 50 iterations,
seeded synthetic data (no public dataset exists for this benchmark).

Output: one JSON line (rank 0). `value` is seconds per solution interval with
the inputs resident in HBM (CUDA events on the solver's stream, max over
ranks, all ranks' intervals counted); `e2e` is the same metric through the
public API with host (pinned) buffers, i.e. including the host-to-device
upload of the interval and the device-to-host read of the solutions.
`roofline` covers the streaming kernel, `cpu_baseline` the reference's own
solver (DP3's solver sources compiled here, oracle/_ref) on the host cores;
where those are absent or the interval has uneven channel blocks, the
restated reference algorithm with its FP32 arithmetic (oracle/).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
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

METRIC = ("s per solution interval to tol 1e-5, GPU learned warm-start vs "
          "plain; HBM GB/s")
WORKLOAD = ("lofar-scale interval: 62 stations (1891 baselines), 10 directions"
            " x 20 sources, 240 channels / 24 blocks, 8 timesteps, XX/YY "
            "complex64, diagonal gains, unit start, tol 1e-5, max 50 iterations")
CONFIG_INDEX = 1


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples the SM clock and the clock-event (throttle) reasons of one GPU
    every 20 ms during a region, through NVML (read-only queries), or through
    nvidia-smi where NVML cannot be loaded."""

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40,
               "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, device, period_s=0.02):
        self.device = device
        self.period = period_s
        self.samples = []  # (sm_mhz, sm_max_mhz, reasons bitmask)
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None

    def _sample_nvml(self):
        n = self._nvml
        h = self._handle
        sm = n.nvmlDeviceGetClockInfo(h, n.NVML_CLOCK_SM)
        reasons = n.nvmlDeviceGetCurrentClocksEventReasons(h)
        return (float(sm), self._max, int(reasons))

    def _sample_smi(self):
        out = subprocess.run(
            ["nvidia-smi", "-i", str(self.device),
             "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active",
             "--format=csv,noheader,nounits"],
            capture_output=True, text=True, timeout=5).stdout.strip()
        sm, smax, act = [x.strip() for x in out.split(",")]
        return (float(sm), float(smax), int(act, 16))

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self._sample_nvml() if self._nvml
                                    else self._sample_smi())
            except Exception:
                pass
            self._stop.wait(self.period)

    def __enter__(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            self._handle = pynvml.nvmlDeviceGetHandleByIndex(self.device)
            self._max = float(pynvml.nvmlDeviceGetMaxClockInfo(
                self._handle, pynvml.NVML_CLOCK_SM))
            self._nvml = pynvml
        except Exception:
            self._nvml = None
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._thread.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"],
                    "samples": 0}
        reasons = sorted({name for _, _, m in self.samples
                          for name, bit in self.REASONS.items() if m & bit})
        return {"sm_mhz": statistics.median(s[0] for s in self.samples),
                "sm_max_mhz": max(s[1] for s in self.samples),
                "reasons": reasons, "samples": len(self.samples),
                "source": "nvml" if self._nvml else "nvidia-smi"}


def _dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def _max_over_ranks(x, world, device):
    """Max of a per-rank timing over all ranks (device None: a CPU tensor,
    for the gloo backend)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64,
                     device="cpu" if device is None else f"cuda:{device}")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def weak_scaling_value(t_local, steps, world, device):
    """Seconds per interval of the whole job: every rank solves `steps`
    intervals of its own, the job takes the slowest rank's time, so the
    job's throughput is steps * world intervals in max-over-ranks seconds."""
    t_max = _max_over_ranks(t_local, world, device)
    return t_max, t_max / (steps * world)


def _barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def workload_name(cfg, config_index, npol):
    if config_index == CONFIG_INDEX and npol == 2:
        return WORKLOAD
    gains = "diagonal" if npol == 2 else "scalar"
    return (f"{cfg.name}, XX/YY complex64, {gains} gains, unit start, tol 1e-5, "
            f"max {cfg.max_iterations} iterations")


class ReferenceCpu:
    """The reference's own solver (DP3's IterativeDiagonalSolver /
    IterativeScalarSolver compiled from its sources, oracle/_ref) on the
    benchmark interval, packed once through its SolveData constructor
    (timed separately), with all host threads."""

    def __init__(self, cfg, obs, npol):
        from oracle import ref_ffi as rf
        self.rf, self.cfg, self.npol = rf, cfg, npol
        self.threads = os.cpu_count() or 1
        self.prep = rf.Prepared(cfg, obs.antenna1, obs.antenna2, obs.data, obs.model, 2, npol)
        self.packing_s = self.prep.seconds_packing
        self._per_it = None

    def _solve(self, n_it):
        cfg = self.cfg
        sol = np.ones((cfg.n_channel_blocks, cfg.n_stations, sum(cfg.nspd), self.npol),
                      np.complex128)
        st = self.rf.settings(max_iterations=n_it, accuracy=cfg.tolerance,
                              step_size=cfg.step_size)
        return self.prep.solve(sol, st, self.threads).seconds_solve

    def sample(self, iterations_per_interval, budget_s):
        """Solve time per interval, from a solve of as many iterations as fit
        in budget_s (at most the interval's own count), scaled to the
        interval's iteration count."""
        if self._per_it is None:
            self._per_it = self._solve(1)
        n_it = int(max(1, min(iterations_per_interval, budget_s // max(self._per_it, 1e-6))))
        per_it = self._solve(n_it) / n_it
        return {"value": per_it * iterations_per_interval, "unit": "s/interval",
                "cores": self.threads, "kind": "reference",
                "packing_s": self.packing_s,
                "sample": f"DP3's own solver (reference sources compiled here, all host "
                          f"threads): {n_it} iterations of the benchmark interval "
                          f"({per_it * 1e3:.1f} ms/iteration) scaled to "
                          f"{iterations_per_interval} iterations; SolveData packing "
                          f"{self.packing_s:.2f} s, not included"}

    def close(self):
        self.prep.close()


def cpu_baseline(cfg, obs, iterations_per_interval, budget_s=20.0, npol=2):
    """The reference's own solver when its compiled sources are present
    (kind "reference"), else the restated oracle (kind "port")."""
    from oracle import ref_ffi as rf
    if rf.available() and cfg.n_channel_blocks and all(
            nc == (cb + 1) * cfg.n_channels // cfg.n_channel_blocks
            - cb * cfg.n_channels // cfg.n_channel_blocks
            for cb, nc in enumerate(cfg.cb_channels)):
        ref = ReferenceCpu(cfg, obs, npol)
        try:
            return ref.sample(iterations_per_interval, budget_s)
        finally:
            ref.close()
    return cpu_baseline_port(cfg, obs, iterations_per_interval, budget_s, npol)


def cpu_baseline_port(cfg, obs, iterations_per_interval, budget_s=20.0, npol=2):
    """Times the oracle (restated reference solver, FP32 arithmetic, all host
    threads) on a bounded sample: a few iterations of the same interval,
    scaled to the GPU interval's iteration count. Used where the reference's
    regular SolveData cannot express the interval (uneven channel blocks)."""
    from oracle import oracle_ffi as of
    ap, sm = obs.generic_arrays()
    prob = dict(n_antennas=cfg.n_stations, n_correlations=2, n_pol=npol,
                n_solutions_per_direction=cfg.nspd, data=obs.data,
                model=obs.model, antenna_pairs=ap, solution_map=sm)
    n_threads = os.cpu_count() or 1
    sol = np.ones((cfg.n_channel_blocks, cfg.n_stations, sum(cfg.nspd), npol),
                  np.complex128)
    t0 = time.perf_counter()
    of.perform_iteration(prob, sol, precision=32, n_threads=n_threads)
    t_one = time.perf_counter() - t0
    n_it = int(max(1, min(iterations_per_interval, budget_s // max(t_one, 1e-6))))
    st = of.settings(max_iterations=n_it, accuracy=cfg.tolerance,
                     step_size=cfg.step_size)
    t0 = time.perf_counter()
    res, _ = of.solve(prob, sol, st, precision=32, n_threads=n_threads)
    t = time.perf_counter() - t0
    per_it = t / n_it
    return {"value": per_it * iterations_per_interval, "unit": "s/interval",
            "cores": n_threads, "kind": "port",
            "sample": f"{n_it} iterations of the benchmark interval "
                      f"({per_it * 1e3:.1f} ms/iteration) scaled to "
                      f"{iterations_per_interval} iterations"}


def _max_rel_diff(a, b):
    """max |a - b| / |b| over finite elements after referencing both to
    antenna 0's phase (per channel block, sub-solution, polarization)."""
    def ref(s):
        r = s[:, :1]
        ph = np.where(np.abs(r) > 0, r / np.abs(r), 1.0)
        return s * np.conj(ph)
    ar, br = ref(a), ref(b)
    with np.errstate(all="ignore"):
        return float(np.nanmax(np.abs(ar - br) / np.maximum(np.abs(br), 1e-30)))


def run_warm_start(args, device):
    """Learned warm start vs previous-solution start on the random-walk
    sequence: 62 stations, 10 directions, 120 channels / 12 blocks, 2
    timesteps per interval, `args.warm_intervals` intervals; the networks are
    trained on the plain solver's solutions of the first half and evaluated on
    the second half. Per evaluated interval (data resident on the GPU, wall
    clock around the whole start + solve, each path from its own previous
    solutions, both with their solutions on the GPU): plain = solve from the
    previous solutions; warm = two-stage network start (including its
    undamped feature passes) + solve. The host read-back of the final
    solutions is timed separately for both and reported as a second figure
    (`*_with_readback`)."""
    import torch
    from dp3_b200 import ddsolve, synth, warmstart
    cfg = synth.benchmark_configs()[4]
    n_int = args.warm_intervals
    n_train = n_int // 2
    seq = synth.gain_sequence(cfg, n_int)
    n_sub = sum(cfg.nspd)
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 2, 2, device=device)
    st = ddsolve.default_settings()
    st.max_iterations = 100
    st.accuracy = cfg.tolerance
    st.step_size = cfg.step_size
    ctx.set_settings(st)
    tight = ddsolve.default_settings()
    tight.max_iterations, tight.accuracy, tight.step_size = 400, 1e-8, cfg.step_size
    tight.detect_stalling = 0
    tight_plain = tight_warm = 0.0
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=f"cuda:{device}")
    ws = warmstart.LearnedWarmStart(cfg.n_channel_blocks, cfg.n_stations, n_sub, 2,
                                    passes=(3, 3), provisional_after=max(8, n_train * 3 // 8),
                                    device=device)
    unit = np.ones((cfg.n_channel_blocks, cfg.n_stations, n_sub, 2), np.complex128)
    dev = torch.device(f"cuda:{device}")
    plain_hist = [unit] * 4
    plain_prev = torch.from_numpy(unit).to(dev)  # both paths keep solutions on the GPU
    warm_hist = [torch.from_numpy(unit).to(dev)] * 4
    t_plain, t_warm, it_plain, it_warm, worst = [], [], [], [], 0.0
    rb_plain, rb_warm = [], []
    t_train = 0.0
    warm_tuning = None
    for i in range(n_int):
        obs = synth.observe(cfg, true_gains=seq[i], start_time_s=i * cfg.n_times * cfg.time_step_s,
                            noise_seed=cfg.seed * 31 + i)
        for cb, nc in enumerate(cfg.cb_channels):
            ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc, obs.data[cb],
                                          obs.model[cb], obs.antenna1, obs.antenna2)
        if i == 0 and not args.no_autotune:
            warm_tuning, _ = ctx.autotune(5)  # the same plan for both starts
        stream.synchronize()  # upload and repack done before the clock starts
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        s_dev = plain_prev.clone()
        r = ctx.solve(s_dev)
        t1 = time.perf_counter()
        s = s_dev.cpu().numpy()
        rb_plain_s = time.perf_counter() - t1
        plain_prev = s_dev
        if i < n_train:
            if i >= 4:
                t2 = time.perf_counter()
                ws.add_interval(ctx, plain_hist, s)
                t_train += time.perf_counter() - t2
            if i == n_train - 1:
                t2 = time.perf_counter()
                ws.fit()
                t_train += time.perf_counter() - t2
            warm_hist = [torch.from_numpy(s).to(dev)] + warm_hist[:3]
        else:
            t_plain.append(t1 - t0)
            rb_plain.append(t1 - t0 + rb_plain_s)
            it_plain.append(r.iterations)
            torch.cuda.synchronize(dev)
            t2 = time.perf_counter()
            g_dev = ws.start(ctx, warm_hist)
            rw = ctx.solve(g_dev)
            t3 = time.perf_counter()
            g = g_dev.cpu().numpy()
            t_warm.append(t3 - t2)
            rb_warm.append(time.perf_counter() - t2)
            it_warm.append(rw.iterations)
            worst = max(worst, _max_rel_diff(g, s))
            if len(t_warm) <= args.warm_tight:
                # distance of both answers to a tight-tolerance solve
                ref = s.copy()
                ctx.set_settings(tight)
                ctx.solve(ref)
                ctx.set_settings(st)
                tight_plain = max(tight_plain, _max_rel_diff(s, ref))
                tight_warm = max(tight_warm, _max_rel_diff(g, ref))
            warm_hist = [g_dev] + warm_hist[:3]
        plain_hist = [s] + plain_hist[:3]
    passes = ws.passes
    ws.close()
    ctx.close()
    plain_s, warm_s = float(np.mean(t_plain)), float(np.mean(t_warm))
    return {
        "workload": ("62 stations, 10 directions, 120 channels / 12 blocks, 2 timesteps per "
                     f"interval, {n_int} random-walk intervals (trained on the first "
                     f"{n_train}, evaluated on the last {n_int - n_train})"),
        "plain_s_per_interval": plain_s, "warm_s_per_interval": warm_s,
        "speedup": plain_s / warm_s,
        "timing": "both starts with solutions on the GPU, wall clock of start + solve",
        "plain_s_with_readback": float(np.mean(rb_plain)),
        "warm_s_with_readback": float(np.mean(rb_warm)),
        "speedup_with_readback": float(np.mean(rb_plain) / np.mean(rb_warm)),
        "plain_iterations": float(np.mean(it_plain)),
        "warm_iterations": float(np.mean(it_warm)),
        "warm_feature_passes": passes,
        "max_rel_diff_vs_plain": worst,
        "max_rel_diff_vs_tight_solve": {"plain": tight_plain, "warm": tight_warm,
                                        "intervals": min(args.warm_tight, len(t_warm)),
                                        "tight_accuracy": 1e-8},
        # tolerance 1e-5 bounds the step, not the distance to the fixed point:
        # the test's criterion is the warm answer's distance to a tight solve
        # against the plain answer's own (tests/test_warmstart.py)
        "accuracy_criterion": {
            "rule": "warm within max(1e-4, 1.5 x plain) of a tolerance-1e-8 solve",
            "warm_over_plain": tight_warm / tight_plain if tight_plain > 0 else None,
            "holds": bool(tight_warm < max(1e-4, 1.5 * tight_plain))},
        "train_s": t_train, "tuning": warm_tuning,
        "network": "2 stages x (n_in -> 256 -> 256 -> 48), BF16 on tcgen05, FP32 accumulation",
    }


def run_mlp_only(args):
    """Training throughput of the warm-start network alone (the shape of the
    first stage on the 62-station, 12-block workload: 336 inputs, two hidden
    layers of 256, 48 outputs) on seeded random data; the command the
    tensor-core profile uses."""
    import torch
    from dp3_b200 import warmstart
    rng = np.random.default_rng(5)
    n, n_in, n_out = args.mlp_rows, 336, 48
    x = rng.normal(size=(n, n_in)).astype(np.float32)
    t = rng.normal(size=(n, n_out)).astype(np.float32) * 0.1
    mlp = warmstart.MLP(n_in, n_out, hidden=256, seed=1)
    mlp.train(x[:4096], t[:4096], epochs=1, batch=1024)  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mlp.train(x, t, epochs=args.mlp_epochs, batch=1024)
    dt = time.perf_counter() - t0
    flops_row = 2 * (n_in * 256 + 256 * 256 + 256 * n_out) * 3  # forward + 2x backward
    print(json.dumps({"mlp_train_s": dt, "rows": n, "epochs": args.mlp_epochs,
                      "tflops": flops_row * n * args.mlp_epochs / dt / 1e12}), flush=True)
    mlp.close()
    return 0


def run_mlp_infer(args):
    """The warm start's inference product alone: forward passes of the
    first-stage network (336 inputs, two hidden layers of 256, 48 outputs) on
    the 620 samples of one 62-station, 10-direction interval, through
    ddwarm_predict (one fused mlp_forward_kernel launch per call after the
    input rows are gathered and tiled); the command the inference profile
    uses. Prints the wall time per call."""
    import torch
    from dp3_b200 import warmstart
    rng = np.random.default_rng(7)
    n, n_in, n_out = 620, 336, 48
    x = rng.normal(size=(n, n_in)).astype(np.float32)
    mlp = warmstart.MLP(n_in, n_out, hidden=256, seed=1)
    for _ in range(args.warmup):
        mlp.predict(x)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        mlp.predict(x)
    dt = (time.perf_counter() - t0) / max(args.steps, 1)
    flops = 2 * n * (n_in * 256 + 256 * 256 + 256 * n_out)
    print(json.dumps({"mlp_predict_us_per_call": dt * 1e6, "rows": n,
                      "note": "host x in, host y out: includes the H2D / D2H copies",
                      "forward_mflop": flops / 1e6}), flush=True)
    mlp.close()
    return 0


def run_predict_only(args):
    """The GPU point-source predict alone on configuration `args.config`
    (default the 62-station interval: 10 directions x 20 sources, 24 blocks
    of 10 channels, 8 timesteps): every channel block's model visibilities
    predicted into device memory (ddsolve_predict_regular, one predict_kernel
    launch per block), timed with CUDA events on the context's stream; the
    command the predict profile uses. Prints the device time per interval,
    the source-visibility terms per second and the model bytes written."""
    import torch
    from dp3_b200 import build as native_build
    from dp3_b200 import ddsolve, synth
    native_build.build_all()
    torch.cuda.set_device(0)
    cfg = synth.benchmark_configs()[args.config]
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 2, 2)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device="cuda:0")
    sky = synth.sky(cfg)
    uvw = synth.station_uvw(cfg)
    # cross baselines in the generator's order: (0, 1), (0, 2), ..., (1, 2), ...
    a1, a2 = (np.ascontiguousarray(x, np.uint32) for x in np.triu_indices(cfg.n_stations, 1))
    freqs = synth.frequencies(cfg)
    edges = np.cumsum([0] + list(cfg.cb_channels))
    cb_freqs = [np.ascontiguousarray(freqs[edges[i]:edges[i + 1]])
                for i in range(cfg.n_channel_blocks)]
    outs = [torch.empty((cfg.n_directions, cfg.n_times * cfg.n_baselines * len(f), 2, 2),
                        dtype=torch.float32, device="cuda:0") for f in cb_freqs]

    def predict():
        for cb, f in enumerate(cb_freqs):
            ctx.predict_regular(cfg.n_times, cfg.n_baselines, f, uvw, a1, a2, sky, out=outs[cb])

    for _ in range(args.warmup):
        predict()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        predict()
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    terms = cfg.n_vis * sum(len(l) for l, _ in sky)  # sources x visibilities
    out_bytes = sum(o.numel() * 4 for o in outs)
    print(json.dumps({"config": cfg.name, "predict_ms_per_interval": ms,
                      "source_visibility_terms_per_s": terms / (ms / 1e3),
                      "model_bytes": out_bytes,
                      "model_write_gbs": out_bytes / (ms / 1e3) / 1e9}), flush=True)
    ctx.close()
    return 0


def run_correct_subtract(args):
    """DDECal's CorrectAndSubtractModels (the step after the solve) on the GPU
    through ddsolve_correct_and_subtract, on configuration `args.config`: the
    interval in DP3's buffer layout with four correlations ([t][bl][ch][4]
    data, [dir][t][bl][ch][4] models; XX / YY from the synthetic
    observation, XY = YX = 0), the true gains of each channel block as the
    solutions, every direction's model corrected and the sum subtracted from
    the data in place. Device-resident: buffers and solutions in device
    memory, each call timed with CUDA events on the context's stream (the
    call also copies the two antenna arrays to the device). End to end:
    pinned host buffers, the copies to and from the device inside the timed
    call. Algorithmic bytes per visibility: 32 x (2 + n_dir) (data read and
    written, every model read once). The CPU figure is the numpy oracle on
    one time step of the interval, scaled to the interval."""
    import ctypes
    import torch
    from dp3_b200 import build as native_build
    from dp3_b200 import ddsolve, synth
    from oracle import subtract_oracle
    native_build.build_all()
    torch.cuda.set_device(0)
    cfg = synth.benchmark_configs()[args.config]
    obs = synth.observe(cfg)
    n_t, n_bl, n_dir = cfg.n_times, cfg.n_baselines, cfg.n_directions
    n_ch, n_cb = sum(cfg.cb_channels), cfg.n_channel_blocks
    data = np.zeros((n_t, n_bl, n_ch, 4), np.complex64)
    model = np.zeros((n_dir, n_t, n_bl, n_ch, 4), np.complex64)
    c0 = 0
    for cb, nc in enumerate(cfg.cb_channels):
        d = obs.data[cb].reshape(n_t, n_bl, nc, 2, 2)
        m = obs.model[cb].reshape(n_dir, n_t, n_bl, nc, 2, 2)
        data[:, :, c0:c0 + nc, 0] = d[..., 0, 0] + 1j * d[..., 0, 1]
        data[:, :, c0:c0 + nc, 3] = d[..., 1, 0] + 1j * d[..., 1, 1]
        model[..., c0:c0 + nc, 0] = m[..., 0, 0] + 1j * m[..., 0, 1]
        model[..., c0:c0 + nc, 3] = m[..., 1, 0] + 1j * m[..., 1, 1]
        c0 += nc
    starts = np.cumsum([0] + list(cfg.cb_channels))[:-1]
    sol = np.ascontiguousarray(obs.true_gains[starts], np.complex128)  # [cb][st][dir][2]
    a1 = np.ascontiguousarray(obs.antenna1, np.uint32)
    a2 = np.ascontiguousarray(obs.antenna2, np.uint32)
    ctx = ddsolve.Context(cfg.n_stations, [1] * n_dir, n_cb, 2, 2)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device="cuda:0")
    n_vis = n_t * n_bl * n_ch
    algo = n_vis * 32 * (2 + n_dir)

    def call(d_in, m_in, s, d_out):
        # one model buffer per direction, as DDECal keeps them
        ptrs = (ctypes.c_void_p * n_dir)(*[m_in + d * (n_vis * 32) for d in range(n_dir)])
        ib = ddsolve.SubtractBuffers()
        ib.n_times, ib.n_baselines, ib.n_channels = n_t, n_bl, n_ch
        ib.antenna1, ib.antenna2 = a1.ctypes.data, a2.ctypes.data
        ib.data, ib.models = d_in, ctypes.cast(ptrs, ctypes.c_void_p).value
        rc = ddsolve.lib().ddsolve_correct_and_subtract(ctx._h, ctypes.byref(ib), s, d_out, None)
        if rc != 0:
            raise RuntimeError(ddsolve.lib().ddsolve_last_error(ctx._h).decode())

    def timed(d_in, m_in, s, d_out, steps):
        ms = []
        for _ in range(steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            call(d_in, m_in, s, d_out)
            e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        return float(np.median(ms))

    dev = torch.device("cuda", 0)
    t_data = torch.from_numpy(data.view(np.float32)).to(dev)
    t_model = torch.from_numpy(model.view(np.float32)).to(dev)
    t_sol = torch.from_numpy(sol.view(np.float64)).to(dev)
    torch.cuda.synchronize()
    args_dev = (t_data.data_ptr(), t_model.data_ptr(), t_sol.data_ptr(), t_data.data_ptr())
    timed(*args_dev, args.warmup)
    dev_ms = timed(*args_dev, args.steps)
    h_data = torch.from_numpy(data.view(np.float32)).pin_memory()
    h_model = torch.from_numpy(model.view(np.float32)).pin_memory()
    h_out = torch.empty_like(h_data).pin_memory()
    args_host = (h_data.data_ptr(), h_model.data_ptr(), sol.ctypes.data, h_out.data_ptr())
    timed(*args_host, args.warmup)
    e2e_ms = timed(*args_host, max(3, args.steps // 4))
    ctx.close()
    peak, peak_kind = _peaks()
    achieved = algo / (dev_ms / 1e3) / 1e9
    # CPU: the numpy oracle on the first time step, scaled to the interval
    t0 = time.perf_counter()
    subtract_oracle.correct_and_subtract(data[:1], model[:, :1], sol, a1, a2, True, False)
    cpu_s = (time.perf_counter() - t0) * n_t
    print(json.dumps({
        "config": cfg.name, "step": "DDECal::CorrectAndSubtractModels",
        "n_vis": n_vis, "ms_per_interval": dev_ms, "algorithmic_bytes": algo,
        "achieved_gbs": achieved, "peak_gbs": peak, "peak_kind": peak_kind,
        "frac": achieved / peak,
        "e2e_ms_per_interval": e2e_ms,
        "e2e_bytes": {"h2d": data.nbytes + model.nbytes + sol.nbytes, "d2h": data.nbytes},
        "cpu_oracle_s_per_interval": cpu_s,
        "cpu_oracle_sample": "numpy restatement, 1 thread, first time step scaled to the interval",
    }), flush=True)
    return 0


def run_full_jones(args):
    """The full-Jones pass (IterativeFullJonesSolver's PerformIteration on
    the GPU: fj_pass_kernel, or fj_chunk_kernel above four directions, and
    fj_finalize_kernel) on the layout of configuration `args.config` with
    four correlations and `args.fj_directions` directions (one solution
    each), seeded random visibilities and unit gains; mean device time of
    one pass over `args.kernel_launches` launches (CUDA events on the
    context's stream, ddsolve_time_stream_kernel) and the algorithmic bytes
    (32 B per visibility for the data and every direction's model)."""
    from dp3_b200 import build as native_build
    from dp3_b200 import ddsolve, synth
    native_build.build_all()
    cfg = synth.benchmark_configs()[args.config]
    n_dir = args.fj_directions
    rng = np.random.default_rng(0)
    ctx = ddsolve.Context(cfg.n_stations, [1] * n_dir, cfg.n_channel_blocks, 4, 4)
    a1, a2 = (np.ascontiguousarray(x, np.uint32) for x in np.triu_indices(cfg.n_stations, 1))
    n_vis = 0
    data, model = [], []
    for cb, nc in enumerate(cfg.cb_channels):
        nv = cfg.n_times * cfg.n_baselines * nc
        data.append(rng.standard_normal((nv, 4, 2)).astype(np.float32))
        model.append(rng.standard_normal((n_dir, nv, 4, 2)).astype(np.float32))
        ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc, data[-1], model[-1],
                                      a1, a2)
        n_vis += nv
    sol = np.zeros((cfg.n_channel_blocks, cfg.n_stations, n_dir, 4), np.complex128)
    sol[..., 0] = sol[..., 3] = 1.0
    ctx.perform_iteration(sol)
    launches = ctx.last_launch_count()
    ms = ctx.time_stream_kernel(args.kernel_launches)
    ctx.close()
    algo = n_vis * 32 * (1 + n_dir)
    peak, peak_kind = _peaks()
    out = {"config": cfg.name, "solver": "full-Jones (4 correlations, 2x2 gains)",
           "n_directions": n_dir, "n_vis": n_vis, "pass_ms": ms,
           "launches_per_pass": launches, "algorithmic_bytes": algo,
           "achieved_gbs": algo / (ms / 1e3) / 1e9, "peak_gbs": peak,
           "peak_kind": peak_kind, "frac": algo / (ms / 1e3) / 1e9 / peak}
    if not args.no_cpu_baseline:
        # the reference's own IterativeFullJonesSolver (oracle/_ref) on the
        # same interval with all host threads: seconds per iteration from a
        # 3-iteration solve, SolveData packing excluded
        try:
            from types import SimpleNamespace
            from oracle import ref_ffi as rf
            rcfg = SimpleNamespace(n_stations=cfg.n_stations, n_times=cfg.n_times,
                                   n_baselines=cfg.n_baselines, cb_channels=cfg.cb_channels,
                                   nspd=[1] * n_dir)
            prep = rf.Prepared(rcfg, a1, a2, data, model, 4, 4)
            threads = os.cpu_count() or 1
            st = rf.settings(max_iterations=3, accuracy=1e-12, step_size=0.2)
            s0 = sol.copy()
            sec = prep.solve(s0, st, threads).seconds_solve
            prep.close()
            out["cpu_baseline"] = {"value": sec / 3 * 1e3, "unit": "ms per iteration",
                                   "cores": threads, "kind": "reference",
                                   "sample": "DP3's IterativeFullJonesSolver (reference sources "
                                             "compiled here), 3 iterations of the same interval"}
        except Exception as e:  # the reference oracle is test infrastructure
            out["cpu_baseline"] = {"unavailable": str(e)[:200]}
    print(json.dumps(out), flush=True)
    return 0


def run_fp64_check(args):
    """Solution error of the GPU solver against the FP64 oracle on
    configuration `args.config` (a numerical statement, not a timing): one
    pass from a perturbed start (max relative error per element) and the full
    solve from unit solutions (iteration counts; max relative difference after
    antenna-0 phase referencing), plus the same for the oracle with the
    reference's FP32 arithmetic."""
    from dp3_b200 import build as native_build
    from dp3_b200 import ddsolve, synth
    from oracle import oracle_ffi as of
    native_build.build_all()
    of.build()
    cfg = synth.benchmark_configs()[args.config]
    obs = synth.observe(cfg)
    ap, sm = obs.generic_arrays()
    npol = args.npol
    prob = dict(n_antennas=cfg.n_stations, n_correlations=2, n_pol=npol,
                n_solutions_per_direction=list(cfg.nspd), data=obs.data, model=obs.model,
                antenna_pairs=ap, solution_map=sm)
    n_sub = sum(cfg.nspd)
    shape = (cfg.n_channel_blocks, cfg.n_stations, n_sub, npol)
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 2, npol)
    for cb, nc in enumerate(cfg.cb_channels):
        ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc, obs.data[cb],
                                      obs.model[cb], obs.antenna1, obs.antenna2)
    st = ddsolve.default_settings()
    st.max_iterations, st.accuracy, st.step_size = (cfg.max_iterations, cfg.tolerance,
                                                    cfg.step_size)
    ctx.set_settings(st)
    rng = np.random.default_rng(3)
    start = np.exp(0.1 * (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)))
    got = ctx.perform_iteration(start)
    ref = of.perform_iteration(prob, start, precision=64)
    ref32 = of.perform_iteration(prob, start, precision=32)
    with np.errstate(all="ignore"):
        pass_err = float(np.nanmax(np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)))
        pass_err32 = float(np.nanmax(np.abs(ref32 - ref) / np.maximum(np.abs(ref), 1e-300)))
        # relative to the block's typical gain magnitude instead of each element
        scale = np.nanmedian(np.abs(ref), axis=(1, 2, 3), keepdims=True)
        pass_err_scaled = float(np.nanmax(np.abs(got - ref) / scale))
        pass_err32_scaled = float(np.nanmax(np.abs(ref32 - ref) / scale))
    g = np.ones(shape, np.complex128)
    r = ctx.solve(g)
    ost = of.settings(max_iterations=cfg.max_iterations, accuracy=cfg.tolerance,
                      step_size=cfg.step_size)
    out = {"config": workload_name(cfg, args.config, npol), "pass_max_rel_err_vs_fp64": pass_err,
           "pass_max_rel_err_oracle32_vs_fp64": pass_err32,
           "pass_max_err_per_median_gain": pass_err_scaled,
           "pass_max_err_per_median_gain_oracle32": pass_err32_scaled,
           "gpu_iterations": int(r.iterations)}
    for prec in (64, 32):
        o = np.ones(shape, np.complex128)
        ro, _ = of.solve(prob, o, ost, precision=prec)
        out[f"oracle{prec}_iterations"] = int(ro.iterations)
        out[f"solve_max_rel_diff_vs_oracle{prec}"] = _max_rel_diff(g, o)
    print(json.dumps(out), flush=True)
    ctx.close()
    return 0


def run_reference_arm(args):
    world, rank, local = _dist_setup()
    if rank != 0:
        return 0
    from dp3_b200 import synth
    cfg = synth.benchmark_configs()[args.config]
    obs = synth.observe(cfg)
    from oracle import oracle_ffi as of
    from oracle import ref_ffi as rf
    of.build()
    iters = cfg.max_iterations + 1  # the interval does not converge in 50
    times = []
    base = None
    # the whole run within about three minutes of CPU work
    budget = min(args.ref_budget, 180.0 / (args.warmup + args.steps))
    ref = ReferenceCpu(cfg, obs, args.npol) if rf.available() else None
    for i in range(args.warmup + args.steps):
        if ref is not None:
            b = ref.sample(iters, budget)
        else:
            b = cpu_baseline_port(cfg, obs, iters, budget_s=budget, npol=args.npol)
        if i >= args.warmup:
            times.append(b["value"])
            base = b
    if ref is not None:
        ref.close()
    value = statistics.mean(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": value,
        "unit": "s/interval", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(cfg, args.config, args.npol),
                   "threads": base["cores"]},
        "cpu_baseline": base,
        "e2e": {"value": value, "unit": "s/interval", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_batch(args):
    """`args.batch` independent intervals of configuration `args.config` (own
    gains, noise and hour angles each) in one context: one streaming pass per
    iteration over every interval still iterating, each interval with its
    own stopping. value = device seconds per interval (batch time / batch)."""
    import torch
    from dp3_b200 import ddsolve, synth
    from dp3_b200 import build as native_build
    native_build.build_all()
    device = 0
    torch.cuda.set_device(device)
    cfg = synth.benchmark_configs()[args.config]
    nb = args.batch
    n_cb = cfg.n_channel_blocks
    obs = [synth.observe(cfg, true_gains=synth.gains(cfg, seed=cfg.seed + 1 + g),
                         start_time_s=g * cfg.n_times * cfg.time_step_s,
                         noise_seed=cfg.seed * 7919 + 17 + g) for g in range(nb)]
    n_sub = sum(cfg.nspd)
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, nb * n_cb, 2, args.npol, device=device)
    st = ddsolve.default_settings()
    st.max_iterations = cfg.max_iterations
    st.accuracy = cfg.tolerance
    st.step_size = cfg.step_size
    ctx.set_settings(st)
    ctx.set_intervals([g * n_cb for g in range(nb + 1)])

    def upload():
        for g, o in enumerate(obs):
            for cb, nc in enumerate(cfg.cb_channels):
                ctx.set_channel_block_regular(g * n_cb + cb, cfg.n_times, cfg.n_baselines, nc,
                                              o.data[cb], o.model[cb], o.antenna1, o.antenna2)

    upload()
    tuning, tuned_ms = ctx.autotune(3)
    tuning["iteration_ms"] = tuned_ms
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=f"cuda:{device}")
    sols = np.ones((nb * n_cb, cfg.n_stations, n_sub, args.npol), np.complex128)
    for _ in range(args.warmup):
        sols[...] = 1.0
        res = ctx.solve_batch(sols)
    torch.cuda.synchronize()
    launches = 0
    with ClockSampler(device) as clocks:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            sols[...] = 1.0
            res = ctx.solve_batch(sols)
            launches += ctx.last_launch_count()
        ev1.record(stream)
        ev1.synchronize()
    t_dev = ev0.elapsed_time(ev1) / 1e3
    value = t_dev / (args.steps * nb)
    # end to end: upload of every interval + batch solve + solutions back
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e_steps = max(1, args.steps // 10)
    e0.record(stream)
    for _ in range(e_steps):
        upload()
        sols[...] = 1.0
        ctx.solve_batch(sols)
    e1.record(stream)
    e1.synchronize()
    e2e_value = e0.elapsed_time(e1) / 1e3 / (e_steps * nb)
    h2d = sum(d.nbytes for o in obs for d in o.data) + sum(m.nbytes for o in obs for m in o.model)
    kernel_ms = ctx.time_stream_kernel(3)
    alg_bytes = nb * cfg.n_vis * 16 * (1 + cfg.n_directions)
    peak, peak_kind = _peaks()
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    result = {
        "metric": METRIC, "value": value, "unit": "s/interval", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_dev / args.steps * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"{nb} independent intervals batched: " +
                               workload_name(cfg, args.config, args.npol),
                   "n_vis": nb * cfg.n_vis, "tuning": tuning,
                   "iterations_per_interval": [int(r.iterations) for r in res],
                   "l2": f"inputs larger than L2 ({alg_bytes / 1e6:.0f} MB per iteration)",
                   "parallelism": "1 GPU, one context, one pass per iteration for the batch"},
        "e2e": {"value": e2e_value, "unit": "s/interval", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(sols.nbytes)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                     "kernel": "stream_kernel" if tuning.get("use_pipe") == 0 else "pipe_kernel",
                     "kernel_ms": kernel_ms,
                     "algorithmic_bytes_per_launch": alg_bytes},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    print(json.dumps(result), flush=True)
    ctx.close()
    return 0


def run_gpu_arm(args):
    import torch
    world, rank, local = _dist_setup()
    device = local
    torch.cuda.set_device(device)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device(f"cuda:{device}"))
    from dp3_b200 import ddsolve, synth
    from dp3_b200 import build as native_build
    native_build.build_all()
    cfg = synth.benchmark_configs()[args.config]
    # every rank solves its own interval (independent intervals: weak scaling)
    obs = synth.observe(cfg, pinned=True, noise_seed=cfg.seed * 7919 + 17 + rank)
    n_sub = sum(cfg.nspd)
    ctx = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 2, args.npol,
                          device=device)
    st = ddsolve.default_settings()
    st.max_iterations = cfg.max_iterations
    st.accuracy = cfg.tolerance
    st.step_size = cfg.step_size
    ctx.set_settings(st)
    if args.direction_groups or args.max_slab_times:
        ctx.set_tuning(args.direction_groups, args.max_slab_times)

    def upload():
        for cb, nc in enumerate(cfg.cb_channels):
            ctx.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc,
                                          obs.data[cb], obs.model[cb],
                                          obs.antenna1, obs.antenna2)

    sols = np.ones((cfg.n_channel_blocks, cfg.n_stations, n_sub, args.npol), np.complex128)
    mags = np.zeros(cfg.max_iterations + 1, np.float64)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=f"cuda:{device}")

    upload()
    tuning = None
    if not args.no_autotune and not (args.direction_groups or args.max_slab_times):
        # one-off per problem shape (cached per process), outside the timing
        tuning, tuned_ms = ctx.autotune(5)
        tuning["iteration_ms"] = tuned_ms
    if args.pass_only:
        # One streaming pass, timed alone (the command profiles use).
        kernel_ms = ctx.time_stream_kernel(args.kernel_launches)
        alg_bytes = cfg.n_vis * 16 * (1 + cfg.n_directions)
        print(json.dumps({"config": cfg.name, "pass_ms": kernel_ms,
                          "achieved_gbs": alg_bytes / (kernel_ms / 1e3) / 1e9}),
              flush=True)
        ctx.close()
        return 0
    # ---- device-resident timing: K solves of the resident interval --------
    iters = []
    for _ in range(args.warmup):
        sols[...] = 1.0
        r = ctx.solve(sols, mags)
    launches = 0
    _barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(device) as clocks:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            sols[...] = 1.0
            r = ctx.solve(sols, mags)
            iters.append(r.iterations)
            launches += ctx.last_launch_count()
        ev1.record(stream)
        ev1.synchronize()
    torch.cuda.synchronize()
    _barrier(world)
    t_dev = ev0.elapsed_time(ev1) / 1e3
    t_dev, value = weak_scaling_value(t_dev, args.steps, world, device)
    n_iter_run = r.iterations if not r.has_converged else r.iterations
    device_iters = min(r.iterations, cfg.max_iterations)

    # ---- end to end through the public API with host buffers --------------
    h2d = sum(d.numel() * 4 for d in obs.data) + sum(m.numel() * 4 for m in obs.model)
    h2d += sols.nbytes
    d2h = sols.nbytes
    for _ in range(max(1, args.warmup // 2)):
        upload()
        sols[...] = 1.0
        ctx.solve(sols, mags)
    _barrier(world)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    w0 = time.perf_counter()
    e0.record(stream)
    for _ in range(args.steps):
        upload()
        sols[...] = 1.0
        ctx.solve(sols, mags)
    e1.record(stream)
    e1.synchronize()
    w_e2e = time.perf_counter() - w0
    t_serial, e2e_serial = weak_scaling_value(e0.elapsed_time(e1) / 1e3, args.steps, world,
                                              device)

    # Pipelined end to end (how a stream of intervals runs): two contexts
    # alternate, the next interval's upload (pinned host memory, on the idle
    # context's stream) overlapping the current interval's solve. Every step
    # still uploads its inputs and reads its solutions back; timed by wall
    # clock between device synchronisations.
    ctx2 = ddsolve.Context(cfg.n_stations, cfg.nspd, cfg.n_channel_blocks, 2, args.npol,
                           device=device)
    ctx2.set_settings(st)
    if args.direction_groups or args.max_slab_times:
        ctx2.set_tuning(args.direction_groups, args.max_slab_times)

    def upload_to(c):
        for cb, nc in enumerate(cfg.cb_channels):
            c.set_channel_block_regular(cb, cfg.n_times, cfg.n_baselines, nc,
                                        obs.data[cb], obs.model[cb],
                                        obs.antenna1, obs.antenna2)

    # The same interval with the model predicted on the GPU from the sky
    # (ddsolve_set_channel_block_regular_sky): only the data, the station
    # UVW and the point sources cross PCIe.
    sky = synth.sky(cfg)
    uvw = synth.station_uvw(cfg)
    freqs = synth.frequencies(cfg)
    edges = np.cumsum([0] + list(cfg.cb_channels))
    cb_freqs = [np.ascontiguousarray(freqs[edges[i]:edges[i + 1]])
                for i in range(cfg.n_channel_blocks)]

    def upload_sky_to(c):
        for cb in range(cfg.n_channel_blocks):
            c.set_channel_block_regular_sky(cb, cfg.n_times, cfg.n_baselines, obs.data[cb],
                                            cb_freqs[cb], uvw, obs.antenna1, obs.antenna2, sky)

    upload_to(ctx2)
    if tuning is not None:
        ctx2.autotune(5)  # the cached choice of `ctx` (same shape)
    ctxs = [ctx, ctx2]

    def pipelined(up):
        # The next interval's upload runs on a second host thread (the C ABI
        # calls release the GIL), so that its host-side work and its copies
        # and kernels on the other context's stream overlap the synchronous
        # solve of the current interval.
        from concurrent.futures import ThreadPoolExecutor
        for _ in range(2):  # warm-up of the pipeline
            up(ctx)
            sols[...] = 1.0
            ctx.solve(sols, mags)
        _barrier(world)
        torch.cuda.synchronize()
        with ThreadPoolExecutor(max_workers=1) as pool:
            w0 = time.perf_counter()
            up(ctxs[0])
            for k in range(args.steps):
                nxt = pool.submit(up, ctxs[(k + 1) % 2]) if k + 1 < args.steps else None
                sols[...] = 1.0
                ctxs[k % 2].solve(sols, mags)
                if nxt is not None:
                    nxt.result()
            torch.cuda.synchronize()
            wall = time.perf_counter() - w0
        return weak_scaling_value(wall, args.steps, world, device)[1]

    e2e_model_upload = pipelined(upload_to)
    e2e_value = pipelined(upload_sky_to)
    h2d_model_upload = h2d
    h2d = (sum(d.numel() * 4 for d in obs.data) + sols.nbytes + uvw.nbytes
           + cfg.n_channels * 8 + 2 * cfg.n_channel_blocks * cfg.n_baselines * 4
           + cfg.n_channel_blocks * sum(l.nbytes + s.nbytes for l, s in sky))
    ctx2.close()

    # ---- roofline of the streaming kernel ----------------------------------
    kernel_ms = ctx.time_stream_kernel(args.kernel_launches)
    alg_bytes = cfg.n_vis * 16 * (1 + cfg.n_directions)
    peak, peak_kind = _peaks()
    achieved = alg_bytes / (kernel_ms / 1e3) / 1e9
    # the kernel of the autotuned plan (the default plan prefers pipe_kernel)
    use_pipe = (tuning or {}).get("use_pipe", -1)
    kernel_name = ("stream_kernel" if use_pipe == 0 else
                   "pipe_kernel" if use_pipe == 1 else "default plan (pipe_kernel where it applies)")
    traffic = None
    prof = os.path.join(ROOT, "profiles", f"pipe_kernel_c{args.config}_traffic.json")
    if os.path.exists(prof):
        try:
            with open(prof) as f:
                traffic = json.load(f).get("dram_bytes_per_launch")
        except Exception:
            traffic = None

    result = {
        "metric": METRIC, "value": value, "unit": "s/interval",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_dev / args.steps * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": workload_name(cfg, args.config, args.npol), "n_vis": cfg.n_vis,
                   "iterations_per_interval": int(r.iterations),
                   "tuning": tuning,
                   "l2": (f"inputs larger than L2 ({alg_bytes / 1e6:.0f} MB streamed per "
                          "iteration)" if alg_bytes > 126e6 else
                          f"inputs ({alg_bytes / 1e6:.2f} MB) fit in L2: not a bench line"),
                   "parallelism": f"{world} independent interval(s), one per GPU"},
        "vis_iterations_per_s": cfg.n_vis * device_iters * args.steps * world / t_dev,
        "e2e": {"value": e2e_value, "unit": "s/interval",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "path": "data, station UVW and point-source sky uploaded; model "
                        "visibilities predicted on the GPU "
                        "(ddsolve_set_channel_block_regular_sky), then ddsolve_solve",
                "pipelined": "two contexts: next interval's upload and predict, issued "
                             "from a second host thread, overlap the solve",
                "model_upload": {"value": e2e_model_upload,
                                 "h2d_bytes_per_step": int(h2d_model_upload),
                                 "path": "data and model visibilities uploaded "
                                         "(ddsolve_set_channel_block_regular)"},
                "serial_value": e2e_serial, "serial_wall_s": w_e2e},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": kernel_name,
                     "kernel_ms": kernel_ms,
                     "algorithmic_bytes_per_launch": alg_bytes},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and args.warm_intervals > 0:
        result["warm_start"] = run_warm_start(args, device)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle_ffi as of
        of.build()
        obs_np = synth.observe(cfg)
        result["cpu_baseline"] = cpu_baseline(cfg, obs_np, int(r.iterations),
                                              budget_s=args.ref_budget, npol=args.npol)
    if rank == 0:
        print(json.dumps(result), flush=True)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=60)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--kernel-launches", type=int, default=20)
    ap.add_argument("--direction-groups", type=int, default=0)
    ap.add_argument("--max-slab-times", type=int, default=0)
    ap.add_argument("--ref-budget", type=float, default=8.0,
                    help="seconds of CPU work per reference sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config", type=int, default=CONFIG_INDEX,
                    help="benchmark configuration index (synth.benchmark_configs)")
    ap.add_argument("--npol", type=int, default=2, choices=[1, 2],
                    help="2: IterativeDiagonalSolver, 1: IterativeScalarSolver")
    ap.add_argument("--warm-intervals", type=int, default=200,
                    help="intervals of the learned-warm-start sequence (0: skip)")
    ap.add_argument("--warm-tight", type=int, default=20,
                    help="evaluated intervals also solved to tolerance 1e-8 for accuracy")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--fp64-check", action="store_true",
                    help="solution error against the FP64 oracle (no timing)")
    ap.add_argument("--batch", type=int, default=1,
                    help="independent intervals of --config solved in one context")
    ap.add_argument("--mlp-infer", action="store_true",
                    help="time only the warm-start network's forward pass (for profiling)")
    ap.add_argument("--predict-only", action="store_true",
                    help="time only the GPU point-source predict of --config (for profiling)")
    ap.add_argument("--full-jones", action="store_true",
                    help="time only the full-Jones pass on the layout of --config")
    ap.add_argument("--fj-directions", type=int, default=4)
    ap.add_argument("--correct-subtract", action="store_true",
                    help="time only the GPU CorrectAndSubtractModels step of --config")
    ap.add_argument("--mlp-only", action="store_true",
                    help="time only the warm-start network's training (for profiling)")
    ap.add_argument("--mlp-rows", type=int, default=60000)
    ap.add_argument("--mlp-epochs", type=int, default=5)
    ap.add_argument("--pass-only", action="store_true",
                    help="time only the streaming pass (for profiling)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference_arm(args)
    if args.mlp_only:
        return run_mlp_only(args)
    if args.mlp_infer:
        return run_mlp_infer(args)
    if args.predict_only:
        return run_predict_only(args)
    if args.correct_subtract:
        return run_correct_subtract(args)
    if args.full_jones:
        return run_full_jones(args)
    if args.fp64_check:
        return run_fp64_check(args)
    if args.batch > 1:
        return run_batch(args)
    return run_gpu_arm(args)


if __name__ == "__main__":
    sys.exit(main())
