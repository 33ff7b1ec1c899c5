"""`evolve` — the reference's highest-level driver for MCWF runs on the device.

Mirrors ``evolve(psi, sys, pe)`` (high/Evolution_.h:174-209) dispatching to
``cppqedutils::run`` (Trajectory.h:310-339, main loop :560-595):

* ``--evol single``: one trajectory; dc mode (stream every dc steps) when ``--dc`` is
  nonzero, else Dt mode / NDt mode;
* ``--evol ensemble``: nTraj trajectories; Dt or NDt mode (an Ensemble has no step, so
  dc mode does not apply, StochasticTrajectory.h:193-256); every stream carries the
  ensemble average of the linear observables and the mean dtDid.

Each streamed row is ``[t, dtDid, averages...]`` after ``Averaged::process``.
``--evol master`` runs the master equation on the device (cqg_master_*), with the same
dc / Dt / NDt loops (a Master trajectory has a step, so dc mode applies).

``ensemble_log`` writes the end-of-run log of an ensemble (mcwf::EnsembleLogger::stream,
MCWF_TrajectoryLogger.cc:79-121) and ``trajectory_log`` that of one trajectory
(mcwf::Logger::onEnd, :19-33), from the device's logger counters and jump records.
"""
import numpy as np

from . import _abi as A
from .engine import Ensemble, Master, Model, System


def _row(model, t, sums, n_traj, linear=None):
    row = np.empty(2 + model.n_avr)
    row[0] = t
    row[1] = sums[-1] / n_traj
    avr = np.asarray(sums[:-1]) / n_traj
    if linear is not None:
        linear.append(avr.copy())
    row[2:] = model.process(avr)
    return row


def evolve(script, args=(), rng=None, precision=None, n_traj=None, resume=None, _linear=None):
    """Runs the script's system as the reference's trajectory::run would.

    resume: a checkpoint (Ensemble.save) to continue from, as --continue does; the
    continued run streams no initial row (Trajectory.h:585).
    Returns (rows, ensemble, model); rows has one line per stream."""
    model = Model(script, args)
    rp = model.run_pars()
    if rp.evol == A.EVOL_MASTER:
        return _evolve_master(model, rp)
    pars = rp.mcwf
    if rng is not None:
        pars.rng = rng
    if precision is not None:
        pars.precision = precision
    if n_traj is None:
        n_traj = 1 if rp.evol == A.EVOL_SINGLE else int(rp.n_traj)
    system = System(model.desc)
    ens = Ensemble(system, model.initial_state(), n_traj, pars)

    def front_time():
        return ens.times()[0][0]

    if resume is not None:
        ens.load(resume)
        rows = []
    else:
        rows = [_row(model, 0.0, ens.steps(0, rp.T), n_traj, _linear)]
    if rp.evol == A.EVOL_SINGLE and rp.dc:
        T = rp.T
        while front_time() < T:
            sums = ens.steps(rp.dc, T)
            rows.append(_row(model, front_time(), sums, n_traj, _linear))
    elif rp.NDt:
        t = front_time()
        sums = ens.run(rp.Dt, int(rp.NDt))
        for k in range(int(rp.NDt)):
            t = t + rp.Dt
            rows.append(_row(model, t, sums[k], n_traj, _linear))
    else:
        T, Dt = rp.T, rp.Dt
        t = front_time()
        while t < T:
            # consecutive full Dt intervals go to the device in one launch; each
            # trajectory advances to t + Dt exactly as cppqedutils::advance does
            n, tt, ts = 0, t, []
            while tt < T and min(Dt, T - tt) == Dt:
                tt = tt + Dt
                ts.append(tt)
                n += 1
            if n:
                sums = ens.run(Dt, n)
                for k in range(n):
                    rows.append(_row(model, ts[k], sums[k], n_traj, _linear))
                t = ts[-1]
            else:
                delta = T - t
                sums = ens.run(delta, 1)
                t = t + delta
                rows.append(_row(model, t, sums[0], n_traj, _linear))
    return np.array(rows), ens, model


def ensemble_log_values(ens):
    """The numbers of mcwf::EnsembleLogger::stream: averages over the trajectories of the
    accepted steps, dpLimit and dpTolerance overshoots and jumps; maxima over the
    trajectories of the overshoots and of |norm - 1|."""
    c = ens.counters().astype(np.float64)
    mo, mt, mn = ens.logger_maxima()
    return {"average_steps": c[:, 0].mean(), "average_overshot": c[:, 4].mean(), "max_overshoot": mo.max(),
            "average_tolerance_overshot": c[:, 5].mean(), "max_tolerance_overshoot": mt.max(),
            "max_norm_deviation": mn.max(), "average_jumps": c[:, 6].mean(), "total_jumps": int(c[:, 6].sum())}


def _density(samples, n_bins):
    """Histogram of boost::accumulators' density feature with the whole sample as its
    cache: n_bins equal bins between the sample's minimum and maximum, one underflow and one
    overflow bin in front and behind; each bin as (lower edge, fraction of the samples)."""
    lo, hi = min(samples), max(samples)
    width = (hi - lo) / n_bins
    edges = [lo + (i - 1) * width for i in range(n_bins + 2)]
    counts = [0] * (n_bins + 2)
    for x in samples:
        if x < edges[1]:
            counts[0] += 1
        elif x >= edges[n_bins + 1]:
            counts[n_bins + 1] += 1
        else:
            k = 1
            while k < n_bins + 1 and x >= edges[k + 1]:
                k += 1
            counts[k] += 1
    return [(edges[i], counts[i] / len(samples)) for i in range(n_bins + 2)]


def ensemble_log(ens, n_bins=0, n_jumps_per_bin=50):
    """Text of mcwf::EnsembleLogger::stream (numbers in the stream's default 6 digits).  The
    histogram is built from the jump records the device keeps (the last 64 of each
    trajectory)."""
    v = ensemble_log_values(ens)
    g = "{:.6g}".format
    out = ["", "Average number of total steps: " + g(v["average_steps"]), "",
           "On average, dpLimit overshot: %s times, maximal overshoot: %s" % (g(v["average_overshot"]),
                                                                             g(v["max_overshoot"])),
           "On average, dpTolerance overshot: %s times, maximal overshoot: %s" % (
               g(v["average_tolerance_overshot"]), g(v["max_tolerance_overshoot"])), "",
           "Maximal deviation of norm from 1: " + g(v["max_norm_deviation"])]
    total = v["total_jumps"]
    if not n_bins and total < 2 * n_jumps_per_bin:
        out += ["", "Too few jumps for a histogram"]
    else:
        bins = n_bins if n_bins else total // n_jumps_per_bin
        times = []
        for i in range(ens.n_traj):
            t, _ = ens.jumps(i, 1 << 20)
            times.extend(t.tolist())
        out += ["", "Histogram of jumps. Number of bins=%d" % (bins + 2)]
        out += ["%s\t%s" % (g(a), g(b)) for a, b in _density(times, bins)]
    out += ["", "Average number of total jumps: " + g(total / ens.n_traj)]
    return "\n".join(out) + "\n"


def trajectory_log(ens, i=0):
    """Text of mcwf::Logger::onEnd for trajectory i (log level > 0)."""
    c = ens.counters()[i]
    mo, mt, mn = ens.logger_maxima()
    t, l = ens.jumps(i, 1 << 20)
    g = "{:.6g}".format
    out = ["", "Total number of MCWF steps: %d" % c[0], "",
           "dpLimit overshot: %d times, maximal overshoot: %s" % (c[4], g(mo[i])),
           "dpTolerance overshot: %d times, maximal overshoot: %s" % (c[5], g(mt[i])), "",
           "Maximal deviation of norm from 1: " + g(mn[i]), "", "MCWF Trajectory:"]
    out += ["%s\t%d" % (g(a), b) for a, b in zip(t, l)]
    return "\n".join(out) + "\n\n"


def _evolve_master(model, rp):
    """trajectory::run of a Master trajectory (Trajectory.h:462-610) on the device."""
    system = System(model.desc)
    m = Master(system, model.initial_state(), rp.mcwf)
    n = model.n_avr

    def row(t, vals):
        r = np.empty(2 + n)
        r[0] = t
        r[1] = vals[n]
        r[2:] = model.process(np.asarray(vals[:n]))
        return r

    rows = [row(0.0, m.steps(0, rp.T, n))]
    if rp.dc:  # dc mode: a row every dc steps until T
        while m.times()[0] < rp.T:
            vals = m.steps(rp.dc, rp.T, n)
            rows.append(row(m.times()[0], vals))
    elif rp.NDt:  # NDt intervals of Dt
        t = m.times()[0]
        for vals in m.run(rp.Dt, int(rp.NDt), n):
            t = t + rp.Dt
            rows.append(row(t, vals))
    else:  # Dt intervals up to T, the last one shortened
        T, Dt = rp.T, rp.Dt
        t = m.times()[0]
        while t < T:
            delta = min(Dt, T - t)
            vals = m.run(delta, 1, n)[0]
            t = t + delta
            rows.append(row(t, vals))
    return np.array(rows), m, model


def time_averaged(script, args=(), relaxation_time=0.0, **kw):
    """quantumtrajectory::TimeAveragingMCWF_Trajectory (TimeAveragingMCWF_Trajectory.h:35-90):
    the run of ``evolve`` with, at every stream after the relaxation time, the running mean
    of the unprocessed averages, averages = (averages * n + now) / (n + 1), without step-size
    weighting.  Returns (rows, processed time averages or None, number of samples, ensemble,
    model); the reference prints the processed averages in its end-of-run log ("Time
    averages after relaxation time ...")."""
    linear = []
    rows, ens, model = evolve(script, args, _linear=linear, **kw)
    acc = np.zeros(model.n_avr)
    n = 0
    for t, now in zip(rows[:, 0], linear):
        if t > relaxation_time:
            acc = (acc * n + now) / (n + 1)
            n += 1
    return rows, (model.process(acc.copy()) if n else None), n, ens, model
