"""The BDA SolveData packing restated in numpy (test infrastructure only).

DDECal solves baseline-dependently averaged (BDA) data through a second
SolveData constructor (ddecal/gain_solvers/SolveData.cc:190-300): every BDA
row (one baseline, one averaged time, its own channel count) is split into
the solver's channel blocks by its own channel count (channel block cb takes
channels [cb n / n_cb, (cb + 1) n / n_cb) of a row with n channels,
:205-208, :240-244), autocorrelations are dropped (:202, :237), and each
direction's solution index is the nearest-neighbour bin of the row's mid time
in the solution interval, truncated to the last solution
(min(n_sol - 1, floor(t_mid n_sol / duration)), :270-282), with the
per-direction counts limited as for regular data (LimitNSolutionsPerDirection,
by the number of rows, :214). The product solves such data through the
generic per-visibility entry point (ddsolve_set_channel_block), which is what
DP3's SolverBase adapter uploads for any SolveData. Like the regular
constructor's output, the packed data must meet the solvers' precondition that
SolutionIndex(d, 0) is direction d's lowest solution index
(ddecal/gain_solvers/SolveData.h:72-80; the CPU solvers index their
accumulators relative to it). The reference's BDA
constructor needs DP3's BdaSolverBuffer and casacore-backed BdaBuffer, which
do not build here, hence this restatement.
"""
import numpy as np

TIME_STEP_S = 10.0  # duration of one unaveraged time step of the rows


def bda_rows(obs, time_factor, freq_factor, rng=None):
    """BDA rows of a regular observation: baseline b averages time_factor[b]
    time steps and freq_factor[b] channels (both dividing the interval's).
    Returns a list of dicts (baseline, time, n_channels, data [n_ch, 2, 2],
    model [n_dir, n_ch, 2, 2], complex64 XX/YY) and the interval duration."""
    cfg = obs.cfg
    n_ch = sum(cfg.cb_channels)
    rows = []
    # the regular data per (time, baseline, channel) over the whole band
    data = np.concatenate([d.reshape(cfg.n_times, cfg.n_baselines, nc, 2, 2)
                           for d, nc in zip(obs.data, cfg.cb_channels)], axis=2)
    model = np.concatenate([m.reshape(cfg.n_directions, cfg.n_times, cfg.n_baselines, nc, 2, 2)
                            for m, nc in zip(obs.model, cfg.cb_channels)], axis=3)
    dt = TIME_STEP_S
    for t0 in range(0, cfg.n_times):
        for b in range(cfg.n_baselines):
            ft, ff = time_factor[b], freq_factor[b]
            if t0 % ft:
                continue
            d = data[t0:t0 + ft, b].reshape(ft, n_ch // ff, ff, 2, 2).mean(axis=(0, 2))
            m = model[:, t0:t0 + ft, b].reshape(cfg.n_directions, ft, n_ch // ff, ff, 2, 2)
            m = m.mean(axis=(1, 3))
            rows.append(dict(baseline=b, time=(t0 + 0.5 * ft) * dt, n_channels=n_ch // ff,
                             data=d.astype(np.float32), model=m.astype(np.float32)))
    if rng is not None:
        rng.shuffle(rows)
    return rows, cfg.n_times * dt


def limit_n_solutions(nspd, n_rows):
    # SolveData.cc LimitNSolutionsPerDirection: at most one solution per row
    return [min(n, n_rows) for n in nspd]


def bda_solve_data(rows, duration, antenna1, antenna2, n_cb, nspd, n_corr=2):
    """The BDA constructor's channel blocks: per cb data float32 [n_vis, 2, 2],
    model [n_dir, n_vis, 2, 2], antenna_pairs uint32 [n_vis, 2] and
    solution_map uint32 [n_dir, n_vis] (generic-layout problem arrays)."""
    n_dir = len(nspd)
    n_sol = limit_n_solutions(nspd, len(rows))
    start = np.concatenate([[0], np.cumsum(n_sol)[:-1]]).astype(np.int64)
    out = [dict(data=[], model=[], ap=[], sm=[]) for _ in range(n_cb)]
    for row in rows:
        a1, a2 = int(antenna1[row["baseline"]]), int(antenna2[row["baseline"]])
        if a1 == a2:
            continue
        n = row["n_channels"]
        for cb in range(n_cb):
            c0, c1 = cb * n // n_cb, (cb + 1) * n // n_cb
            if c1 == c0:
                continue
            o = out[cb]
            o["data"].append(row["data"][c0:c1])
            o["model"].append(row["model"][:, c0:c1])
            o["ap"].append(np.tile([a1, a2], (c1 - c0, 1)))
            sol = [min(n_sol[d] - 1, int(np.floor(row["time"] * n_sol[d] / duration))) + start[d]
                   for d in range(n_dir)]
            o["sm"].append(np.repeat(np.asarray(sol)[:, None], c1 - c0, axis=1))
    res = []
    for o in out:
        res.append(dict(
            data=np.ascontiguousarray(np.concatenate(o["data"]), np.float32),
            model=np.ascontiguousarray(np.concatenate(o["model"], axis=1), np.float32),
            antenna_pairs=np.ascontiguousarray(np.concatenate(o["ap"]), np.uint32),
            solution_map=np.ascontiguousarray(np.concatenate(o["sm"], axis=1), np.uint32)))
    return res, n_sol
