"""update!-style stepping of a model handle through its setter entry points, one TimeStep! per
snapshot selection (src/Simulation/update.jl:11-48): before each step the velocity, PARF and
temperature snapshots that update! would pick at model.t are set, then the step runs.

Works with any object that has get_time/set_velocity/set_PARF/set_temp/time_step (the native
model handle of either precision)."""
import math


def forcing_indices(t, wl):
    """Snapshot indices (0-based) that update! selects at model time t (update.jl:14-26)."""
    tv = int(math.floor(t / wl.dT_vel))
    tp = int(math.floor(t / wl.dT_PAR))
    tt = int(math.floor(t / wl.dT_temp))
    return tv, tp, tt


class VelCache:
    """Velocity snapshots of a workload, built once each."""

    def __init__(self, wl):
        self.wl, self.cache = wl, {}

    def __call__(self, i):
        if i not in self.cache:
            self.cache[i] = self.wl.velocity(i)
        return self.cache[i]


def drive(model, wl, steps, vel=None):
    """`steps` steps of update!(sim) with vels, one step at a time through the setters."""
    vel = vel or VelCache(wl)
    for _ in range(steps):
        _, t = model.get_time()
        tv, tp, tt = forcing_indices(t, wl)
        model.set_velocity(*vel(tv))
        model.set_PARF(wl.parf[:, :, tp])
        model.set_temp(wl.temp[:, :, :, tt])
        model.time_step(wl.dT)
