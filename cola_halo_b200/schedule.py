"""COLA time-step schedule and snapshot windows of the reference driver.

Restates ``main.c:67-206``: a realization computes the PM force at the
current position time ``apos0``, writes every output whose scale factor lies
in ``[avel0, apos0]``, kicks the velocity to ``avel1``, writes outputs in
``(apos0, avel1]``, then drifts the positions to ``apos1``.

The reference hard-wires ``a_init = da = a_final/nsteps`` (``main.c:71-72``)
and starts the velocity clock at ``a_v = da`` (``main.c:145``).  The general
form used here keeps those semantics for any ``a_init``:

    apos0(i) = a_init + (i-1) da      avel0(i) = a_init + (i-1.5) da
    apos1(i) = a_init +  i    da      avel1(i) = a_init + (i-0.5) da

with ``a_v = a_init`` at the start.  ``Schedule.reference(nsteps)`` is the
reference's schedule (``nloop = nsteps`` force evaluations, the last one at
``a_final``); ``Schedule.linear(a_init, a_final, nsteps)`` takes ``nsteps``
drifts from ``a_init`` to ``a_final`` (``nsteps + 1`` force evaluations).
"""
from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Schedule:
    a_init: float
    da: float
    nloop: int
    a_final: float

    @classmethod
    def reference(cls, nsteps, a_final=1.0):
        da = a_final / nsteps
        return cls(a_init=da, da=da, nloop=nsteps, a_final=a_final)

    @classmethod
    def linear(cls, a_init, a_final, nsteps):
        da = (a_final - a_init) / nsteps
        return cls(a_init=a_init, da=da, nloop=nsteps + 1, a_final=a_final)

    def times(self, istep):
        """(avel0, apos0, avel1, apos1) in double precision (``main.c:174-178``)."""
        a0, da = self.a_init, self.da
        return (a0 + (istep - 1.5) * da, a0 + (istep - 1.0) * da,
                a0 + (istep - 0.5) * da, a0 + istep * da)


def output_scale_factors(zout):
    """``aout[i] = (float)(1/(1+z_i))`` (``main.c:107-111``): single precision."""
    return [float(np.float32(1.0 / (1.0 + z))) for z in zout]


def run_time_loop(sched, aout, *, move, force, kick, drift, snapshot, kick_drift=None):
    """Drive one realization's time loop with the reference's control flow.

    ``move()``, ``force()``, ``kick(avel1)``, ``drift(apos1)`` and
    ``snapshot(aout, iout)`` are the per-step actions (``main.c:167-205``).
    ``kick_drift(avel1, apos1)``, when given, replaces a kick and the drift
    that follows it whenever no output falls between them.
    Returns the list of (event, a) pairs in the order they happened.
    """
    events = []
    nout = len(aout)
    iout = 0
    if not (nout > 0 and sched.nloop > 1 and sched.a_final > sched.a_init):
        return events
    for istep in range(1, sched.nloop + 1):
        move()
        force()
        avel0, apos0, avel1, apos1 = sched.times(istep)
        events.append(("force", apos0))
        while iout < nout and avel0 <= aout[iout] <= apos0:
            snapshot(aout[iout], iout)
            events.append(("snapshot", aout[iout]))
            iout += 1
        if iout >= nout:
            break
        if kick_drift is not None and not (iout < nout and apos0 < aout[iout] <= avel1):
            kick_drift(avel1, apos1)
            events.append(("kick", avel1))
            events.append(("drift", apos1))
            continue
        kick(avel1)
        events.append(("kick", avel1))
        while iout < nout and apos0 < aout[iout] <= avel1:
            snapshot(aout[iout], iout)
            events.append(("snapshot", aout[iout]))
            iout += 1
        if iout >= nout:
            break
        drift(apos1)
        events.append(("drift", apos1))
    return events
