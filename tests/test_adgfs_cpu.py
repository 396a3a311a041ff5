"""CPU checks of the BGK / ARS oracle: the IMEX tables reach their stated
order on a relaxation problem with a linear explicit part, and the BGK
relaxation drives a distribution to its Maxwellian."""
import numpy as np
import pytest

from oracle.bgk import ARS, maxwellian, moments5, nu, step_ars
from oracle.fr import velocities


def _grid(N=12, L=5.0):
    c0 = np.linspace(-L + L / N, L - L / N, N)
    return velocities(c0), (2 * L / N)**3


def _f0(cv, seed=0):
    rng = np.random.default_rng(seed)
    u = np.array([0.3, -0.1, 0.05])[:, None]
    f = np.exp(-np.sum((cv - u)**2, axis=0) / 1.1) / (np.pi * 1.1)**1.5
    return f * (1 + 0.2 * np.sin(cv[0]) * np.cos(cv[1])) * (1 + 0.01 * rng.uniform(-1, 1, cv.shape[1]))


@pytest.mark.parametrize('scheme,order', [('adgfs-ars-111', 1), ('adgfs-ars-222', 2),
                                          ('adgfs-ars-443', 3)])
def test_ars_order(scheme, order):
    """df/dt = -k f + nu (M[f] - f) on one velocity cube: error vs a fine
    reference falls with the scheme's order."""
    cv, cw = _grid()
    f0 = _f0(cv)[None]
    L = lambda f: -0.7 * f
    prefac, omega, T = 2.0, 0.81, 0.4

    def run(n):
        f = f0.copy()
        for _ in range(n):
            f = step_ars(f, T / n, L, scheme, prefac, omega, cv, cw)
        return f
    ref = run(512)
    e1 = np.linalg.norm(run(8) - ref)
    e2 = np.linalg.norm(run(16) - ref)
    rate = np.log2(e1 / e2)
    assert rate > order - 0.3, rate


def test_bgk_relaxes_to_maxwellian():
    cv, cw = _grid()
    f = _f0(cv, 1)[None]
    U0 = moments5(f, cv, cw)
    for _ in range(40):
        f = step_ars(f, 0.5, lambda g: 0 * g, 'adgfs-ars-222', 2.0, 0.81, cv, cw)
    M = maxwellian(moments5(f, cv, cw), cv)
    assert np.linalg.norm(f - M) < 1e-4 * np.linalg.norm(M)       # 12^3 grid quadrature
    # moments stay within the grid's quadrature error of the initial ones
    assert np.allclose(moments5(f, cv, cw), U0, rtol=1e-4, atol=1e-4)


def test_ars_tables_consistent():
    for name, (Ae, Ai) in ARS.items():
        Ae, Ai = np.array(Ae), np.array(Ai)
        c_e, c_i = Ae.sum(1), Ai.sum(1)
        assert np.allclose(c_e, c_i), name          # same stage times
        assert np.isclose(Ae[-1].sum(), 1.0) and np.isclose(Ai[-1].sum(), 1.0)
    assert nu(np.array([1.0, 0, 0, 0, 1.5]), 2.0, 0.81) == pytest.approx(2.0)
