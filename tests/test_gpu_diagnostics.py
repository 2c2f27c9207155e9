"""Run statistics on the GPU: a statistics file written during a run holds,
row by row, the GPU moments of that step and the field energy of the
reference's formula; in FP32 mode the field sums stay within FP32 rounding of
the FP64 path's."""
import numpy as np
import pytest

from csrst_b200 import Simulation
from csrst_b200.diagnostics import DataSink, read_sdds
from csrst_b200.workloads import make_bunch, workload

pytestmark = pytest.mark.gpu


def test_statistics_file_follows_the_run(gpu_lib, tmp_path):
    cfg, spec = workload("small-1")
    s = Simulation(cfg)
    s.load(*make_bunch(spec))
    s.initial_fields()
    dt = s.info()["dt"]
    path = tmp_path / "maxwadis.stat"
    expect = []
    with DataSink(s, str(path)) as ds:
        for k in range(3):
            s.step(4)
            m = s.moments()
            expect.append(ds.execute((k + 1) * 4 * dt))
            assert np.array_equal(np.array(expect[-1])[[1, 2, 3, 12, 13, 14]], m[[14, 4, 5, 16, 17, 15]])
    names, rows = read_sdds(str(path))
    assert rows.shape == (3, 16) and np.allclose(rows, np.array(expect), rtol=1e-14, atol=0)
    assert np.all(rows[:, 15] > 0) and np.all(np.diff(rows[:, 0]) > 0)


def test_fp32_field_sums_close_to_fp64(gpu_lib):
    cfg, spec = workload("small-1")
    out = []
    for fp32 in (False, True):
        s = Simulation(cfg, fp32=fp32)
        s.load(*make_bunch(spec))
        s.initial_fields()
        s.step(10)
        out.append(s.field_energy(True))
    assert np.all(np.abs(out[1] - out[0]) <= 1e-4 * np.abs(out[0]))
