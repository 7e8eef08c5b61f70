"""The L2 read-bandwidth probe behind the round kernel's L2 roofline
(emp_measure_l2_read): a finite rate above the device's HBM copy rate, since
the buffer is served from L2."""
import json
import math
import os

import pytest

import empanada_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.gpu
def test_l2_read_rate_is_above_hbm():
    gbs = empanada_b200.measure_l2_read(64 << 20, 0)
    assert math.isfinite(gbs) and gbs > 0
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    hbm = float(json.load(open(p))["hbm_gbs"]) if os.path.exists(p) else 6650.0
    assert gbs > hbm, (gbs, hbm)
