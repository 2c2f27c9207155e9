"""Absorbing layers at the open ends (csrst_set_pml) on the GPU.

 * FP64: with the layers on, the loop stays bit-identical to the oracle's
   restatement (its own FP64 CPML), fields, window and particles, for a
   bunch in the straight section and one entering the dipole;
 * the layer cells and the regular sweep's row ranges equal the oracle's
   construction;
 * FP64 and FP32 mode: a TEM pulse sent into the exit comes back whole from
   the reference's PEC end and below 2e-3 of its energy with a 10-cell
   layer, and 2000 steps with the layers stay bounded."""
import numpy as np
import pytest

import pml_pulse as PP
from csrst_b200 import Simulation
from csrst_b200.workloads import make_bunch, workload
from test_gpu_parity import assert_same_state, pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["small-1", "small-2-bend"])
def test_pml_steps_bit_exact(gpu_lib, oracle, name):
    cfg, g, o = pair(name, oracle, fields=True, seed=4)
    g.set_pml(10)
    o.set_pml(10)
    n, rows = g.pml()
    assert n == o.pml_cells() and n > 0
    assert (rows[:, 0] > 0).any() and (rows[:, 1] < cfg.Nx).any()
    g.step(12)
    o.step(12)
    assert_same_state(g, o)
    g.close()


def test_pml_off_is_the_reference_path(gpu_lib, oracle):
    cfg, g, o = pair("small-1", oracle, fields=True, seed=5)
    g.set_pml(10)
    g.set_pml(0)                      # off again: the reference's PEC ends
    assert g.pml()[0] == 0
    g.step(6)
    o.step(6)
    assert_same_state(g, o)
    g.close()


@pytest.mark.parametrize("fp32", [False, True])
def test_pml_absorbs_an_outgoing_pulse(gpu_lib, fp32):
    cfg, _ = workload("small-1")
    back, e0, bounded = {}, None, None
    for pml in (0, 10):
        s = Simulation(cfg, fp32=fp32)
        info = s.info()
        inside, _ = s.geometry()
        fields, (a, b) = PP.pulse_fields(inside, info["hx"], info["ox"], "exit")
        e0 = PP.energy(fields).sum()
        s.set_static(*fields)
        s.load(*make_bunch(PP.zero_bunch(cfg, info["ox"], info["oy"], info["hx"], info["hy"])))
        if pml:
            s.set_pml(pml)
        for k in range(2000):
            s.half_h(); s.update_e(0); s.half_h(); s.update_e(1)
            if k + 1 == PP.ROUND_TRIP:
                back[pml] = PP.energy(s.get_static())[:, a:b].sum() / e0
        if pml:
            bounded = PP.energy(s.get_static()).sum() / e0
        s.close()
    assert back[0] > 0.97
    assert back[10] < 2e-3
    assert np.isfinite(bounded) and bounded < 0.05
