"""The reference program's time loop (src/main.cpp:358-522) over a
Simulation, with its output schedule:

* before the loop: both field-plot series at t = 0 (unless restarting), a
  statistics row stamped t + dt and one line-field file (main.cpp:362-387);
* per iteration: the two TE/TM half steps, then on plot steps
  (it % plot_modulus == plot_modulus - 1) both plot series at t + dt, on
  statistics steps the statistics row at t + dt and the energy-change
  bookkeeping, on line steps the line-field file (with the window's current
  only if the same iteration plotted, as copyFields copies it only then),
  and last the window move (main.cpp:390-506);
* after the loop: energyChangeAfter.dat (main.cpp:516-519).

Iterations without output run as captured CUDA-graph steps; output
iterations run the half steps and the window move one by one so that the
output sees the state between them, as in the reference."""
import os

from .diagnostics import DataSink, EnergyChange, LineFieldSink, VtkSink


def run(sim, cfg, steps, start=0, plot_modulus=100000, stat_modulus=100000, line_modulus=100000,
        directory="Data", restart=False, t0=0.0):
    """Runs iterations start .. start + steps - 1 of the reference loop on
    `sim` (a loaded Simulation; cfg its RunConfig) writing the reference's
    files under `directory`; returns the simulated time reached."""
    os.makedirs(directory, exist_ok=True)
    dt = sim.info()["dt"]
    pavc = VtkSink(sim, base="c", directory=directory)
    mmpavc = VtkSink(sim, base="mm", directory=directory, source="window")
    if not restart:
        pavc.execute(0.0)
        mmpavc.execute(0.0)
    energy = EnergyChange(sim, cfg, stat_modulus, directory)
    t = t0
    with DataSink(sim, os.path.join(directory, "maxwadis.stat")) as dsc:
        dsc.execute(t + dt)
        semfc = LineFieldSink(sim, directory)
        semfc.execute()
        quiet = 0  # iterations owed as graph steps
        for it in range(start, start + steps):
            plot = it % plot_modulus == plot_modulus - 1
            stat = it % stat_modulus == stat_modulus - 1
            line = it % line_modulus == line_modulus - 1
            if not (plot or stat or line):
                quiet += 1
                t += dt
                continue
            if quiet:
                sim.step(quiet)
                quiet = 0
            sim.step_first()
            sim.step_second()
            if plot:
                pavc.execute(t + dt)
                mmpavc.execute(t + dt)
            if stat:
                dsc.execute(t + dt)
                energy.execute()
            if line:
                semfc.with_current = plot
                semfc.execute()
            sim.move()
            t += dt
        if quiet:
            sim.step(quiet)
        energy.finish()
    return t
