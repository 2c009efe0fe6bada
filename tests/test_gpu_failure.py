"""Failure paths on the device, without a GPU fault (through the C ABI):
a bounded wait that nothing completes ends with LMC_ETIMEOUT in the
handle's status word and leaves the context usable; a run that goes
non-finite reports LMC_ENAN from its diagnostics."""
import numpy as np
import pytest

from loma_phd_b200 import Lomacte
from loma_phd_b200 import lomacte as lm
from tests.helpers import FIELDS, case, oracle_for, rel_l2

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives(gpu):
    p, y, st = case(24, 24, 33)
    g = Lomacte(p, y)
    g.load_state(st)
    g.step(1)
    assert g.status() == lm.LMC_OK
    g.wait_selftest(1000)  # an mbarrier nothing arrives on, 1000 polls
    assert g.status() == lm.LMC_ETIMEOUT
    g.close()
    # the context is intact: a fresh case still steps and matches the oracle
    h = Lomacte(p, y)
    h.load_state(st)
    h.step(1)
    assert h.status() == lm.LMC_OK
    o = oracle_for(p, y, st)
    o.step(1)
    sg, so = h.get_state(), o.get_state()
    for k in FIELDS:
        assert rel_l2(sg[k], so[k]) < 1e-10, k
    h.close()


def test_non_finite_run_reports_enan(gpu):
    p, y, st = case(24, 24, 33)
    bad = {k: (np.array(v, copy=True) if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    bad["phi"][1, 2, 10] = np.nan
    g = Lomacte(p, y)
    g.load_state(bad)
    g.step(1)
    with pytest.raises(lm.LomacteError) as e:
        g.diag()
    assert e.value.code == lm.LMC_ENAN
    assert g.status() == lm.LMC_ENAN
    g.close()
