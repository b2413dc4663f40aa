"""The bulk-staged pushes wait on an mbarrier for each particle tile, and
that wait is bounded.  With the test hook that issues no tile copies
(PIC_PUSH_SKIP_COPIES=1) every wait runs out after PIC_PUSH_WAIT_LIMIT polls:
the kernel records the failure and returns, the step reports it as an error
(no GPU fault, no hang), and a new simulation on the same device runs
normally afterwards."""
import numpy as np
import pytest

from pic_b200 import api, deck
from pic_b200.simulation import Simulation

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [api.PIC_PREC_FP64, api.PIC_PREC_MIXED])
def test_push_tile_wait_runs_out_and_is_reported(precision, monkeypatch):
    monkeypatch.setenv("PIC_PUSH_SKIP_COPIES", "1")
    monkeypatch.setenv("PIC_PUSH_WAIT_LIMIT", "2000")
    cfg = deck.config("cfg1", precision=precision)
    sim = Simulation(cfg)
    try:
        sim.initial_fields()
        with pytest.raises(api.PicError, match="push tile copy did not complete"):
            sim.step()
    finally:
        sim.close()
    monkeypatch.delenv("PIC_PUSH_SKIP_COPIES")
    monkeypatch.delenv("PIC_PUSH_WAIT_LIMIT")
    sim = Simulation(cfg)
    try:
        sim.initial_fields()
        st = sim.step()
        assert st.pushed > 0 and np.isfinite(sim.field("phi")).all()
    finally:
        sim.close()
