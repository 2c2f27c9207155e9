"""The oracle's absorbing layers (its own FP64 restatement of the
convolutional PML of csrst_set_pml) on the CPU: a TEM pulse sent into
either open end of the small bend comes back whole from the reference's
PEC end and is absorbed by the layer, and a long run with the layers stays
bounded (no late-time growth)."""
import numpy as np
import pytest

import pml_pulse as PP
from csrst_b200.workloads import make_bunch, workload


def setup(oracle, name="small-1"):
    cfg, _ = workload(name)
    d = cfg.dict()
    d["order"] = cfg.shape_order
    inside, _ = oracle.geometry(cfg.Nx, cfg.Ny, cfg.length_before, cfg.length_after, cfg.width, cfg.phi_deg,
                                cfg.ekin_mev, cfg.bz)
    geo = oracle.bend(cfg.Nx, cfg.Ny, cfg.length_before, cfg.length_after, cfg.width, cfg.phi_deg, cfg.ekin_mev,
                      cfg.bz)
    return cfg, d, inside.reshape(cfg.Ny, cfg.Nx), geo


def run(oracle, d, fields, bunch, pml, steps):
    o = oracle.Sim(d)
    o.set_static(*fields)
    o.load(*bunch)
    if pml:
        o.set_pml(pml)
    for _ in range(steps):
        o.half_h(); o.update_e(0); o.half_h(); o.update_e(1)
    return o


@pytest.mark.parametrize("end", ["exit", "entry"])
def test_layer_absorbs_what_the_pec_end_reflects(oracle, end):
    cfg, d, inside, geo = setup(oracle)
    fields, (a, b) = PP.pulse_fields(inside, geo["hx"], geo["ox"], end)
    bunch = make_bunch(PP.zero_bunch(cfg, geo["ox"], geo["oy"], geo["hx"], geo["hy"]))
    e0 = PP.energy(fields).sum()
    back = {}
    for pml in (0, 10):
        o = run(oracle, d, fields, bunch, pml, PP.ROUND_TRIP)
        back[pml] = PP.energy(o.get_static())[:, a:b].sum() / e0
    assert back[0] > 0.97            # the PEC end sends the pulse back
    assert back[10] < 2e-3           # the layer: below 2e-3 of the pulse's energy (measured 5e-4 exit, 1e-3 entry)
    assert o.pml_cells() > 0


def test_layer_stays_bounded(oracle):
    """6000 steps with both layers (the slanted exit wall's cut cells next
    to the layer once made the update grow without bound)."""
    cfg, d, inside, geo = setup(oracle)
    fields, _ = PP.pulse_fields(inside, geo["hx"], geo["ox"], "exit")
    bunch = make_bunch(PP.zero_bunch(cfg, geo["ox"], geo["oy"], geo["hx"], geo["hy"]))
    e0 = PP.energy(fields).sum()
    o = run(oracle, d, fields, bunch, 10, 6000)
    w = PP.energy(o.get_static())
    assert np.isfinite(w).all() and w.sum() < 0.05 * e0
