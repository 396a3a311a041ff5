"""Host-side pieces of bench.py's JSON line (no GPU): the FLOP models
behind the roofline entry, the workload block, the drift measure and the
HBM denominator's fallback."""
import math
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_flop_models():
    n = 24**3
    fft = 5.0 * n * math.log2(n)
    # packed algorithm: M Nrho + Nrho + 2 transforms and 8 n per (p, q)
    assert bench.q_flops_per_eval(24, 12, 12) == pytest.approx(158 * fft + 8 * 144 * n)
    assert bench.q_flops_per_eval(24, 12, 12) == pytest.approx(1.661e8, rel=1e-3)
    # the reference's 3 M Nrho + 3 transforms per Q (scattering.py:239-281)
    assert bench.q_flops_reference_equivalent(24, 12, 12) == pytest.approx(435 * fft)
    assert bench.q_flops_reference_equivalent(24, 12, 12) == pytest.approx(4.136e8, rel=1e-3)
    assert bench.q_flops_reference_equivalent(24, 12, 12) > 2.4 * bench.q_flops_per_eval(24, 12, 12)


def test_config_block_names_the_workload():
    one, four = bench.config_block(1), bench.config_block(4)
    for c in (one, four):
        assert 'workload' in c and '2048 DOFs' in c['workload'] and 'Nv=24^3' in c['workload']
        assert c['ndof'] == 2048 and (c['Nv'], c['Nrho'], c['M']) == (24, 12, 12)
        assert 'l2' in c and 'model' not in c
    assert one['parallelism'] == 'single GPU' and 'weak scaling' in four['parallelism']


def test_drift_is_relative():
    before = [2.0, 0.0, 0.0, 0.0, 10.0]
    after = [2.0 + 2e-10, 1e-12, 0.0, 0.0, 10.0 - 1e-9]
    d = bench.drift(before, after)
    assert d['mass'] == pytest.approx(1e-10)
    assert d['momentum_x'] == pytest.approx(5e-13)        # relative to the mass
    assert d['energy'] == pytest.approx(1e-10)


def test_hbm_peak_has_a_fallback():
    peak = bench.hbm_peak_gbs()
    assert peak > 1000.0
    if not os.path.exists(os.path.join(os.path.dirname(bench.__file__), 'MEASURED_PEAKS.json')):
        assert peak == 6650.0
