"""A TEM pulse in the pipe travelling towards one of its open ends (shared
by the CPU and GPU absorbing-layer tests).

Ey = E0 exp(-((x - xc) / s)^2) on the inside cells and Hz = +-Ey / Z0 at the
Hz positions, all of it in the x part Hzx (the split field's y part changes
only with d Ex / dy, zero for this wave): between the parallel pipe walls
this is the TEM mode moving along +-x.  With the reference's PEC end the
pulse comes back whole; an absorbing layer at the end should swallow it.
A zero-charge bunch in the middle of the mesh (the loop needs one; it is
never pushed) keeps the window away from both ends."""
import numpy as np

from csrst_b200.workloads import BunchSpec, workload

Z0 = 376.730313461
EPS0, MU0 = 8.854187817e-12, 1.256637061e-06
BACK, WIDTH = 80, 8       # pulse centre: cells from the last / first inside column; 1/e half width
ROUND_TRIP = 480          # steps at CFL 0.5: to the end and 160 cells back


def zero_bunch(cfg, ox, oy, hx, hy):
    spec = BunchSpec(n=64, gamma=1000.0, sigma_s=3 * hx, sigma_x=3 * hy, energy_spread=0.0, charge=0.0,
                     x0=ox + (cfg.Nx // 2) * hx, y0=oy + (cfg.Ny // 2) * hy, seed=5)
    return spec


def pulse_fields(inside, hx, ox, end):
    """Static-mesh fields (Ex, Ey, Hzx, Hzy) of the pulse heading for `end`
    ("exit" or "entry"), and the column range where it is after ROUND_TRIP
    steps when the end reflects it."""
    Ny, Nx = inside.shape
    cols = np.nonzero(inside[Ny // 2])[0]
    first, last = cols.min(), cols.max()
    sgn = 1.0 if end == "exit" else -1.0
    c0 = last - BACK if end == "exit" else first + BACK
    xc = ox + c0 * hx
    s = WIDTH * hx
    i = np.arange(Nx)
    ey = 1e6 * np.exp(-((ox + i * hx - xc) / s) ** 2)[None, :] * inside
    hz = sgn * (1e6 / Z0) * np.exp(-((ox + (i + 0.5) * hx - xc) / s) ** 2)[None, :] * inside
    zero = np.zeros_like(ey)
    back = int(c0 - sgn * BACK)            # a reflected pulse after 240 cells: BACK in, 160 back
    return [zero, ey, hz, zero], (back - 30, back + 30)


def energy(fields):
    ex, ey, hx, hy = fields
    return 0.5 * EPS0 * (ex ** 2 + ey ** 2) + 0.5 * MU0 * (hx + hy) ** 2
