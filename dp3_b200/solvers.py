"""Python mirror of the reference's solver plugin interface.

Same class and method names, argument meaning and error behaviour as
dp3::ddecal::SolverBase (ddecal/gain_solvers/SolverBase.h:24-361) and its
direction-iterative subclasses IterativeDiagonalSolver
(IterativeDiagonalSolver.h:13-35) and IterativeScalarSolver
(IterativeScalarSolver.h:16-44), so that tests read like the reference's
ddecal/test/unit/tSolvers.cc. All computation happens in the CUDA library
through the C ABI (dp3_b200.ddsolve); these classes only hold settings.
"""
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import ddsolve


@dataclass
class SolveResult:
    """SolverBase::SolveResult (SolverBase.h:61-65)."""
    iterations: int = 0
    constraint_iterations: int = 0
    results: list = field(default_factory=list)
    has_converged: bool = False
    has_stalled: bool = False
    step_magnitudes: Optional[np.ndarray] = None


class ChannelBlockData:
    """One channel block of a SolveData (SolveData.h:31-133), reference
    layout: data [n_vis, n_corr, 2] float32, model [n_dir, n_vis, n_corr, 2],
    antenna_pairs [n_vis, 2] uint32, solution_map [n_dir, n_vis] uint32.
    A regular block (SolveData.cc:77-188) may instead carry
    (n_times, n_baselines, n_channels, antenna1, antenna2) and no
    per-visibility index arrays."""

    def __init__(self, data, model, antenna_pairs=None, solution_map=None,
                 regular=None):
        self.data = data
        self.model = model
        self.antenna_pairs = antenna_pairs
        self.solution_map = solution_map
        self.regular = regular

    def NVisibilities(self):
        return int(self.data.shape[0])

    def NDirections(self):
        return int(self.model.shape[0])

    def Antenna1Index(self, vis):
        if self.antenna_pairs is not None:
            return int(self.antenna_pairs[vis, 0])
        t, bl, ch, a1, a2 = self._regular_index(vis)
        return int(a1[bl])

    def Antenna2Index(self, vis):
        if self.antenna_pairs is not None:
            return int(self.antenna_pairs[vis, 1])
        t, bl, ch, a1, a2 = self._regular_index(vis)
        return int(a2[bl])

    def _regular_index(self, vis):
        n_times, n_bl, n_ch, a1, a2 = self.regular
        return vis // (n_bl * n_ch), (vis // n_ch) % n_bl, vis % n_ch, a1, a2


class SolveData:
    """SolveData<VisMatrix> (SolveData.h:28-194): list of ChannelBlockData.
    n_correlations: 1 (UniSolveData), 2 (DuoSolveData), 4 (FullSolveData)."""

    def __init__(self, channel_blocks: Sequence[ChannelBlockData],
                 n_correlations: int):
        self.channel_blocks = list(channel_blocks)
        self.n_correlations = int(n_correlations)

    def NChannelBlocks(self):
        return len(self.channel_blocks)

    def ChannelBlock(self, i):
        return self.channel_blocks[i]

    @classmethod
    def from_arrays(cls, data, model, antenna_pairs, solution_map,
                    n_correlations):
        return cls([ChannelBlockData(d, m, a, s) for d, m, a, s in
                    zip(data, model, antenna_pairs, solution_map)],
                   n_correlations)

    @classmethod
    def regular(cls, data, model, n_times, n_baselines, cb_channels, antenna1,
                antenna2, n_correlations=2):
        blocks = [ChannelBlockData(d, m, regular=(n_times, n_baselines, nc,
                                                  antenna1, antenna2))
                  for d, m, nc in zip(data, model, cb_channels)]
        return cls(blocks, n_correlations)


class Constraint:
    """dp3::ddecal::Constraint (ddecal/constraints/Constraint.h:28-90): the
    hooks SolverBase::ApplyConstraints calls on the host between iterations.
    Apply() receives next_solutions as an ndarray [n_cb, n_ant, n_sub, n_pol]
    (complex128) and modifies it in place."""

    def Satisfied(self):
        return True

    def PrepareIteration(self, has_reached_precision, iteration, final_iter):
        pass

    def Apply(self, solutions, time):
        raise NotImplementedError

    def GetResult(self):
        return None


class AntennaConstraint(Constraint):
    """AntennaConstraint (ddecal/constraints/AntennaConstraint.h:29-82): the
    antennas of each set get the mean of their finite solutions, per channel
    block, sub-solution and polarization."""

    def __init__(self, antenna_sets):
        self.antenna_sets = [sorted(set(a)) for a in antenna_sets]

    def Apply(self, solutions, time):
        for ants in self.antenna_sets:
            sel = solutions[:, ants]  # [cb, |set|, sub, pol]
            finite = np.isfinite(sel)
            total = np.where(finite, sel, 0).sum(axis=1)
            with np.errstate(all="ignore"):
                mean = total / finite.sum(axis=1)
            solutions[:, ants] = mean[:, None]


def make_solutions_finite(arr, n_pol):
    """SolverBase::MakeSolutionsFinite1Pol / 2Pol (SolverBase.cc:316-371) on
    [n_cb, per_cb] complex128, in place; the 2-pol version averages |pol 0|
    for both polarizations, as the reference does (SolverBase.cc:354)."""
    for cb in range(arr.shape[0]):
        v = arr[cb].reshape(-1, n_pol)
        ok = np.all(np.isfinite(v), axis=1)
        avg = np.abs(v[ok, 0]).mean() if ok.any() else 1.0
        v[~ok] = avg


def step(solutions, nxt, step_size, phase_only):
    """SolverBase::Step (SolverBase.cc:88-158): returns the moved solutions."""
    if not phase_only:
        return solutions * (1.0 - step_size) + nxt * step_size
    frm = np.angle(solutions)
    dist = np.angle(nxt) - frm
    dist = np.where(dist > np.pi, dist - 2 * np.pi, np.where(dist < -np.pi, dist + 2 * np.pi, dist))
    return np.exp(1j * (frm + step_size * dist))


def assign_solutions(solutions, nxt, n_pol, step_size, accuracy):
    """SolverBase::AssignSolutions (SolverBase.cc:215-306) for 1 or 2
    polarizations: appends nothing, returns (step magnitude, converged) and
    copies nxt into solutions."""
    total, n = 0.0, 0
    with np.errstate(all="ignore"):
        if n_pol == 1:
            s = solutions.reshape(-1)
            ns = nxt.reshape(-1)
            nz = s != 0
            a = np.abs((ns[nz] - s[nz]) / s[nz])
            fin = np.isfinite(a)
            total, n = a[fin].sum(), int(fin.sum())
        else:
            s = solutions.reshape(-1, 2)
            ns = nxt.reshape(-1, 2)
            inv = 1.0 / s
            ok = np.all(np.isfinite(inv), axis=1)
            d = np.abs((ns[ok] - s[ok]) * inv[ok]).sum(axis=1)
            fin = np.isfinite(d)
            total, n = d[fin].sum(), 2 * int(fin.sum())
    solutions[...] = nxt
    mag = 0.0 if n == 0 else total / step_size / n
    return mag, mag <= accuracy


class SolverBase:
    """Settings and dimensions of dp3::ddecal::SolverBase, with its defaults
    (SolverBase.cc:27-39)."""

    def __init__(self, device=0):
        self._settings = ddsolve.Settings(100, 0, 1.0e-5, 1.0e-4, 0.2, 1, 0.1, 0)
        self._device = device
        self._ctx = None
        self._ctx_key = None
        self._tuning = (0, 0)
        self.n_antennas = 0
        self.n_solutions_per_direction: List[int] = []
        self.n_channel_blocks = 0
        self.constraints = []

    # SolverBase::Initialize (SolverBase.cc:41-61)
    def Initialize(self, n_antennas, n_solutions_per_direction,
                   n_channel_blocks):
        nspd = [int(x) for x in n_solutions_per_direction]
        if not self.SupportsDdSolutionIntervals() and sum(nspd) != len(nspd):
            raise RuntimeError(
                "DD interval solutions not supported for the selected solver "
                "algorithm")
        if len(nspd) == 0 or sum(nspd) == 0:
            raise ValueError("no directions")
        self.n_antennas = int(n_antennas)
        self.n_solutions_per_direction = nspd
        self.n_channel_blocks = int(n_channel_blocks)

    def NDirections(self):
        return len(self.n_solutions_per_direction)

    def NSubSolutions(self):
        return sum(self.n_solutions_per_direction)

    def NAntennas(self):
        return self.n_antennas

    def NChannelBlocks(self):
        return self.n_channel_blocks

    def SupportsDdSolutionIntervals(self):
        return False

    def NSolutionPolarizations(self):
        raise NotImplementedError

    def ConstraintSolvers(self):
        return [self]

    def AddConstraint(self, constraint):
        assert constraint is not None
        self.constraints.append(constraint)

    def GetConstraints(self):
        return self.constraints

    # setters / getters (SolverBase.h:89-177)
    def SetMaxIterations(self, n):
        self._settings.max_iterations = int(n)

    def GetMaxIterations(self):
        return self._settings.max_iterations

    def SetMinIterations(self, n):
        self._settings.min_iterations = int(n)

    def GetMinIterations(self):
        return self._settings.min_iterations

    def SetAccuracy(self, a):
        self._settings.accuracy = float(a)

    def GetAccuracy(self):
        return self._settings.accuracy

    def SetConstraintAccuracy(self, a):
        self._settings.constraint_accuracy = float(a)

    def GetConstraintAccuracy(self):
        return self._settings.constraint_accuracy

    def SetStepSize(self, s):
        self._settings.step_size = float(s)

    def GetStepSize(self):
        return self._settings.step_size

    def SetDetectStalling(self, detect, step_diff_sigma):
        self._settings.detect_stalling = int(bool(detect))
        self._settings.step_diff_sigma = float(step_diff_sigma)

    def GetDetectStalling(self):
        return bool(self._settings.detect_stalling)

    def SetPhaseOnly(self, phase_only):
        self._settings.phase_only = int(bool(phase_only))

    def GetPhaseOnly(self):
        return bool(self._settings.phase_only)

    def SetTuning(self, direction_groups=0, max_slab_times=0):
        """Kernel tuning (no reference counterpart)."""
        self._tuning = (int(direction_groups), int(max_slab_times))
        if self._ctx is not None:
            self._ctx.set_tuning(*self._tuning)

    # ------------------------------------------------------------------
    def _context(self, n_correlations):
        key = (self.n_antennas, tuple(self.n_solutions_per_direction),
               self.n_channel_blocks, n_correlations,
               self.NSolutionPolarizations(), self._device)
        if self._ctx is None or self._ctx_key != key:
            if self._ctx is not None:
                self._ctx.close()
            self._ctx = ddsolve.Context(self.n_antennas,
                                        self.n_solutions_per_direction,
                                        self.n_channel_blocks, n_correlations,
                                        self.NSolutionPolarizations(),
                                        device=self._device)
            self._ctx_key = key
            self._ctx.set_tuning(*self._tuning)
        return self._ctx

    def _upload(self, data: SolveData):
        if data.NChannelBlocks() != self.n_channel_blocks:
            raise ValueError("SolveData has a different number of channel blocks")
        ctx = self._context(data.n_correlations)
        for cb, block in enumerate(data.channel_blocks):
            if block.regular is not None:
                n_times, n_bl, n_ch, a1, a2 = block.regular
                ctx.set_channel_block_regular(cb, n_times, n_bl, n_ch,
                                              block.data, block.model, a1, a2)
            else:
                ctx.set_channel_block(cb, block.data, block.model,
                                      block.antenna_pairs, block.solution_map)
        return ctx

    def _solutions_array(self, solutions):
        per_cb = self.n_antennas * self.NSubSolutions() * \
            self.NSolutionPolarizations()
        if isinstance(solutions, np.ndarray):
            arr = solutions.reshape(self.n_channel_blocks, per_cb)
            return np.ascontiguousarray(arr, dtype=np.complex128)
        if len(solutions) != self.n_channel_blocks:
            raise ValueError("solutions must have one vector per channel block")
        for s in solutions:
            if len(s) != per_cb:
                raise ValueError("solution vector has the wrong size")
        return np.ascontiguousarray(np.stack([np.asarray(s) for s in solutions]),
                                    dtype=np.complex128)

    def _store(self, solutions, arr):
        if isinstance(solutions, np.ndarray):
            solutions.reshape(arr.shape)[...] = arr
        else:
            for cb in range(self.n_channel_blocks):
                solutions[cb][...] = arr[cb]

    def Solve(self, data: SolveData, solutions, time=0.0, stat_stream=None):
        """SolverBase::Solve(data, solutions, time) (SolverBase.h:205-227):
        iterates to convergence on the GPU. `solutions` (list of per-channel-
        block complex128 vectors, or one ndarray) holds the initial values and
        receives the result. stat_stream, when given, receives one line per
        iteration with the step magnitude."""
        if self.constraints:
            ctx = self._upload(data)
            return self._solve_with_constraints(
                lambda sol: ctx.perform_iteration(sol), solutions, time, stat_stream)
        ctx = self._upload(data)
        ctx.set_settings(self._settings)
        arr = self._solutions_array(solutions)
        mags = np.zeros(max(self._settings.max_iterations,
                            self._settings.min_iterations, 1), np.float64)
        res = ctx.solve(arr, mags)
        self._store(solutions, arr)
        n_it = min(res.iterations, len(mags))
        if stat_stream is not None:
            for i in range(n_it):
                stat_stream.write(f"{i + 1} {mags[i]!r}\n")
        return SolveResult(res.iterations, res.constraint_iterations, [],
                           bool(res.has_converged), bool(res.has_stalled),
                           mags[:n_it].copy())

    def _solve_with_constraints(self, perform, solutions, time, stat_stream):
        """IterativeDiagonalSolver::Solve / IterativeScalarSolver::Solve with
        constraints (IterativeDiagonalSolver.cc:38-97, SolverBase.cc:160-306):
        the pass runs on the GPU (`perform`: [n_cb, n_ant, n_sub, n_pol] ->
        next_solutions), MakeSolutionsFinite, Step, the constraints,
        AssignSolutions and the stopping criterion on the host, as in the
        reference."""
        st = self._settings
        n_pol = self.NSolutionPolarizations()
        shape4 = (self.n_channel_blocks, self.n_antennas, self.NSubSolutions(), n_pol)
        arr = self._solutions_array(solutions).reshape(self.n_channel_blocks, -1)
        for c in self.constraints:  # PrepareConstraints (SolverBase.cc:160-164)
            c.PrepareIteration(False, 0, False)
        iteration, has_converged, has_prev, satisfied = 0, False, False, False
        mags = []
        n_var, mean, var = 0, 0.0, 0.0
        while True:
            make_solutions_finite(arr, n_pol)
            nxt = np.asarray(perform(arr.reshape(shape4)), np.complex128).reshape(shape4)
            nxt = step(arr.reshape(shape4), nxt, st.step_size, bool(st.phase_only))
            satisfied = True  # ApplyConstraints (SolverBase.cc:174-190)
            for c in self.constraints:
                satisfied = c.Satisfied() and satisfied
                c.PrepareIteration(has_prev, iteration, iteration + 1 >= st.max_iterations)
                c.Apply(nxt, time)
            acc = st.constraint_accuracy if not satisfied else st.accuracy
            mag, has_converged = assign_solutions(arr, nxt.reshape(arr.shape), n_pol,
                                                  st.step_size, acc)
            mags.append(mag)
            iteration += 1
            has_prev = has_converged or has_prev
            # ReachedStoppingCriterion / DetectStall (SolverBase.h:274-285,
            # SolverBase.cc:63-86)
            stalled = False
            if st.detect_stalling and satisfied:
                if iteration == 1:
                    n_var, mean, var = 1, mag, 0.0
                else:
                    n_var += 1
                    d1 = mag - mean
                    mean += d1 / n_var
                    var += d1 * (mag - mean)
                stalled = iteration >= 30 and mean < st.step_diff_sigma * np.sqrt(var / n_var)
            ready = (iteration >= st.max_iterations or (has_converged and satisfied) or stalled)
            if iteration >= st.min_iterations and ready:
                break
        self._store(solutions, arr)
        if stat_stream is not None:
            for i, m in enumerate(mags):
                stat_stream.write(f"{i + 1} {m!r}\n")
        # MakeResult (SolverBase.cc:192-213)
        its = iteration if (has_converged and satisfied) else iteration + 1
        c_its = iteration + 1 if not satisfied else 0
        return SolveResult(its, c_its, [c.GetResult() for c in self.constraints],
                           bool(has_converged), bool(stalled), np.array(mags))

    def PerformIteration(self, data: SolveData, solutions):
        """next_solutions of one direction-iterative pass (num / den), as the
        reference computes before SolverBase::Step."""
        ctx = self._upload(data)
        arr = self._solutions_array(solutions)
        nxt = ctx.perform_iteration(arr)
        if isinstance(solutions, np.ndarray):
            return nxt.reshape(solutions.shape)
        return [nxt[cb] for cb in range(self.n_channel_blocks)]


class IterativeDiagonalSolver(SolverBase):
    """IterativeDiagonalSolver<MC2x2FDiag / MC2x2F>
    (ddecal/gain_solvers/IterativeDiagonalSolver.h:13-35)."""

    def NSolutionPolarizations(self):
        return 2

    def SupportsDdSolutionIntervals(self):
        return True


class IterativeScalarSolver(SolverBase):
    """IterativeScalarSolver<complex<float> / MC2x2FDiag / MC2x2F>
    (ddecal/gain_solvers/IterativeScalarSolver.h:16-44)."""

    def NSolutionPolarizations(self):
        return 1

    def SupportsDdSolutionIntervals(self):
        return True


class IterativeFullJonesSolver(SolverBase):
    """IterativeFullJonesSolver (ddecal/gain_solvers/IterativeFullJonesSolver.h:
    15-47): 2x2 gains on 4-correlation data (MC2x2F), solutions [.., 4] in
    the order XX XY YX YY. The loop runs on the device; host constraints are
    not supported for this solver here."""

    def NSolutionPolarizations(self):
        return 4

    def SupportsDdSolutionIntervals(self):
        return True

    def Solve(self, data, solutions, time=0.0, stat_stream=None):
        if self.constraints:
            raise NotImplementedError("constraints with the full-Jones solver")
        return super().Solve(data, solutions, time, stat_stream)
