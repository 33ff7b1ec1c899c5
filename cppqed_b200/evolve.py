"""`evolve` — the reference's highest-level driver for MCWF runs on the device.

Mirrors ``evolve(psi, sys, pe)`` (high/Evolution_.h:174-209) dispatching to
``cppqedutils::run`` (Trajectory.h:310-339, main loop :560-595):

* ``--evol single``: one trajectory; dc mode (stream every dc steps) when ``--dc`` is
  nonzero, else Dt mode / NDt mode;
* ``--evol ensemble``: nTraj trajectories; Dt or NDt mode (an Ensemble has no step, so
  dc mode does not apply, StochasticTrajectory.h:193-256); every stream carries the
  ensemble average of the linear observables and the mean dtDid.

Each streamed row is ``[t, dtDid, averages...]`` after ``Averaged::process``.  The
master equation (``--evol master``) is not run on the device.
"""
import numpy as np

from . import _abi as A
from .engine import Ensemble, Model, System


def _row(model, t, sums, n_traj):
    row = np.empty(2 + model.n_avr)
    row[0] = t
    row[1] = sums[-1] / n_traj
    row[2:] = model.process(np.asarray(sums[:-1]) / n_traj)
    return row


def evolve(script, args=(), rng=None, precision=None, n_traj=None):
    """Runs the script's system as the reference's trajectory::run would.

    Returns (rows, ensemble, model); rows has one line per stream."""
    model = Model(script, args)
    rp = model.run_pars()
    if rp.evol == A.EVOL_MASTER:
        raise NotImplementedError("the master equation is not run on the device")
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

    rows = [_row(model, 0.0, ens.steps(0, rp.T), n_traj)]
    if rp.evol == A.EVOL_SINGLE and rp.dc:
        T = rp.T
        while front_time() < T:
            sums = ens.steps(rp.dc, T)
            rows.append(_row(model, front_time(), sums, n_traj))
    elif rp.NDt:
        t = front_time()
        sums = ens.run(rp.Dt, int(rp.NDt))
        for k in range(int(rp.NDt)):
            t = t + rp.Dt
            rows.append(_row(model, t, sums[k], n_traj))
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
                    rows.append(_row(model, ts[k], sums[k], n_traj))
                t = ts[-1]
            else:
                delta = T - t
                sums = ens.run(delta, 1)
                t = t + delta
                rows.append(_row(model, t, sums[0], n_traj))
    return np.array(rows), ens, model
