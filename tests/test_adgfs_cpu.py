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


# ---------------------------------------------------------------------------
# ES-BGK ('esbgk-direct-gll')

def test_es_gaussian_is_maxwellian_at_pr_one_and_for_maxwellians():
    from oracle.bgk import es_gaussian, es_tensor, moments11
    cv, cw = _grid(16, 6.0)
    f = _f0(cv, 2)[None]
    U = moments11(f, cv, cw)
    assert np.allclose(es_gaussian(U, 1.0, cv), maxwellian(U[..., :5], cv), rtol=1e-12, atol=0)
    # a Maxwellian's ES tensor is T I for every Pr
    M = maxwellian(U[..., :5], cv)
    _, _, T, Tij = es_tensor(moments11(M, cv, cw), 2.0 / 3.0)
    assert np.allclose(Tij[0], T[0] * np.eye(3), atol=1e-6)


def test_esbgk_moments_follow_the_stage_moments():
    """With L = 0, ARS-111: the 11 moments of f_1 equal the stage moments U_1
    (second moments relaxed at nu/Pr) up to the grid's quadrature error, and
    the deviatoric stress decays by 1/(1 + dt nu/Pr)."""
    from oracle.bgk import _es_targets, moments11, step_ars_es
    cv, cw = _grid(16, 6.0)
    f = _f0(cv, 3)[None]
    Pr, prefac, omega, dt = 2.0 / 3.0, 2.0, 0.81, 0.3
    U0 = moments11(f, cv, cw)
    f1 = step_ars_es(f, dt, lambda g: 0 * g, 'adgfs-ars-111', prefac, omega, Pr, cv, cw)
    U1 = moments11(f1, cv, cw)
    assert np.allclose(U1[..., :5], U0[..., :5], rtol=1e-6, atol=1e-8)
    w = dt * nu(U0[..., :5], prefac, omega) / Pr
    dev0 = U0[..., 5:] - _es_targets(U0)
    dev1 = U1[..., 5:] - _es_targets(U1)
    assert np.allclose(dev1, dev0 / (1 + w[..., None]), rtol=1e-4, atol=1e-7)


@pytest.mark.parametrize('scheme,order', [('adgfs-ars-111', 1), ('adgfs-ars-222', 2)])
def test_esbgk_ars_order(scheme, order):
    from oracle.bgk import step_ars_es
    cv, cw = _grid()
    f0 = _f0(cv)[None]
    L = lambda f: -0.7 * f
    prefac, omega, T, Pr = 2.0, 0.81, 0.4, 2.0 / 3.0

    def run(n):
        f = f0.copy()
        for _ in range(n):
            f = step_ars_es(f, T / n, L, scheme, prefac, omega, Pr, cv, cw)
        return f
    ref = run(512)
    rate = np.log2(np.linalg.norm(run(8) - ref) / np.linalg.norm(run(16) - ref))
    assert rate > order - 0.3, rate


def test_esbgk_prefactor():
    from oracle.bgk import bgk_prefactor, esbgk_prefactor
    a = (1e-3, 337.0, 273.0, 1e20, 0.81, 2.117e-5, 273.0)
    assert esbgk_prefactor(*a, 2.0 / 3.0) == pytest.approx(bgk_prefactor(*a) * 2.0 / 3.0)


# ---------------------------------------------------------------------------
# Shakov ('shakov-direct-gll')

def test_shakov_target_moments():
    """S keeps the conserved moments and the Maxwellian's second moments and
    carries the heat flux (1 - Pr) q; at Pr = 1 it is the Maxwellian."""
    from oracle.bgk import heat_flux, moments14, shakov_target
    cv, cw = _grid(16, 6.0)
    f = _f0(cv, 4)[None]
    U = moments14(f, cv, cw)
    Pr = 2.0 / 3.0
    US = moments14(shakov_target(U, Pr, cv), cv, cw)
    UM = moments14(maxwellian(U[..., :5], cv), cv, cw)
    assert np.allclose(US[..., :11], UM[..., :11], rtol=0, atol=1e-7)
    assert np.allclose(US[..., :5], U[..., :5], rtol=0, atol=2e-7)
    assert np.allclose(heat_flux(US), (1 - Pr) * heat_flux(U), rtol=0, atol=3e-6)
    assert abs(heat_flux(U)).max() > 1e-2
    assert np.allclose(shakov_target(U, 1.0, cv), maxwellian(U[..., :5], cv), rtol=1e-13, atol=0)


def test_shakov_heat_flux_relaxes_at_nu_pr():
    """With L = 0, ARS-111: q decays by 1/(1 + dt nu Pr), the deviatoric
    stress by 1/(1 + dt nu), and the moments of f_1 follow U_1."""
    from oracle.bgk import _es_targets, heat_flux, moments14, step_ars_sk
    cv, cw = _grid(16, 6.0)
    f = _f0(cv, 5)[None]
    Pr, prefac, omega, dt = 2.0 / 3.0, 2.0, 0.81, 0.3
    U0 = moments14(f, cv, cw)
    f1 = step_ars_sk(f, dt, lambda g: 0 * g, 'adgfs-ars-111', prefac, omega, Pr, cv, cw)
    U1 = moments14(f1, cv, cw)
    n0 = nu(U0[..., :5], prefac, omega)[..., None]
    assert np.allclose(heat_flux(U1), heat_flux(U0) / (1 + dt * n0 * Pr), rtol=0, atol=3e-6)
    dev0 = U0[..., 5:11] - _es_targets(U0)
    dev1 = U1[..., 5:11] - _es_targets(U1)
    assert np.allclose(dev1, dev0 / (1 + dt * n0), rtol=1e-4, atol=1e-7)


@pytest.mark.parametrize('scheme,order', [('adgfs-ars-111', 1), ('adgfs-ars-222', 2)])
def test_shakov_ars_order(scheme, order):
    from oracle.bgk import step_ars_sk
    cv, cw = _grid()
    f0 = _f0(cv)[None]
    L = lambda f: -0.7 * f
    prefac, omega, T, Pr = 2.0, 0.81, 0.4, 2.0 / 3.0

    def run(n):
        f = f0.copy()
        for _ in range(n):
            f = step_ars_sk(f, T / n, L, scheme, prefac, omega, Pr, cv, cw)
        return f
    ref = run(512)
    rate = np.log2(np.linalg.norm(run(8) - ref) / np.linalg.norm(run(16) - ref))
    assert rate > order - 0.3, rate


@pytest.mark.parametrize('q', [2, 3])
@pytest.mark.parametrize('model', ['bgk', 'esbgk', 'shakov'])
def test_bdf_order(q, model):
    """The oracle BDF-q stepper (ARS-222 start-up) reaches order q."""
    from oracle.bgk import run_bdf
    cv, cw = _grid()
    f0 = _f0(cv)[None]
    L = lambda f: -0.7 * f
    T = 0.4

    def run(n):
        return run_bdf(f0, T / n, L, n, q, 2.0, 0.81, 2.0 / 3.0, cv, cw, model)
    ref = run(128)
    rate = np.log2(np.linalg.norm(run(16) - ref) / np.linalg.norm(run(32) - ref))
    assert rate > q - 0.3, rate


@pytest.mark.parametrize('model', ['bgk', 'esbgk', 'shakov'])
@pytest.mark.parametrize('scheme', ['adgfs-ars-111', 'adgfs-ars-222', 'adgfs-ars-443'])
def test_oracle_ars_step_equals_reference_kernels(model, scheme):
    """One ARS step of the oracle's steppers against the reference's own
    bgk-, esbgk- and shakov-direct-gll kernels (rendered; the call sequence
    of frfs/integrators/std/steppers.py:538-585; golden vectors written by
    tests/golden/make_reference_ars.py on a GPU): 2 of its 32 seeded
    distributions on a 16^3 grid, a given explicit part L, dt nu ~ 1, FP64."""
    import os
    import sys
    from oracle.bgk import step_ars, step_ars_es, step_ars_sk
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), 'golden'))
    from make_reference_ars import grid, inputs
    d = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'reference_ars.npz'))
    cv, cw = grid()
    rows = d['rows']
    f0, L = inputs(cv)                      # the generator's seeded inputs
    f0, L = f0[rows], L[rows]
    assert np.allclose(f0.sum(1), d['f0_rows_sum'], rtol=1e-15, atol=0)
    dt, prefac = float(d['dt']), float(d['prefac'])
    Lf = lambda f: L
    if model == 'bgk':
        got = step_ars(f0, dt, Lf, scheme, prefac, 0.81, cv, cw)
    elif model == 'esbgk':
        got = step_ars_es(f0, dt, Lf, scheme, prefac, 0.81, 2.0 / 3.0, cv, cw)
    else:
        got = step_ars_sk(f0, dt, Lf, scheme, prefac, 0.81, 2.0 / 3.0, cv, cw)
    want = d[f'{model}:{scheme}']
    # relative to the change the step makes
    err = np.linalg.norm(got - want) / np.linalg.norm(want - f0)
    assert err < 1e-12, err


@pytest.mark.parametrize('model', ['bgk', 'esbgk', 'shakov'])
@pytest.mark.parametrize('q', [2, 3])
def test_oracle_bdf_update_equals_reference_kernels(model, q):
    """One IMEX-BDF-q update of the oracle (oracle/bgk.py:bdf_update)
    against the reference's own updateMom{q}_BDF / cmaxwellian /
    updateDistribution{q}_BDF kernels of the *-direct-gll templates (the
    call sequence of BDF2AstdStepper.step, frfs/integrators/std/
    steppers.py:700-760; golden vectors of tests/golden/
    make_reference_ars.py): new moments and distribution, FP64."""
    import os
    import sys
    from oracle.bgk import BDF, MODELS, bdf_update
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), 'golden'))
    from make_reference_ars import bdf_inputs, grid
    d = np.load(os.path.join(os.path.dirname(__file__), 'golden', 'reference_ars.npz'))
    cv, cw = grid()
    rows = d['rows']
    fs, Ls = bdf_inputs(cv, q)
    fs, Ls = fs[:, rows], Ls[:, rows]
    mom = MODELS[model][0]
    A, G, b, _ = BDF[q]
    Pr = 1.0 if model == 'bgk' else 2.0 / 3.0
    U, f = bdf_update(list(fs), list(Ls), [mom(x, cv, cw) for x in fs], [mom(x, cv, cw) for x in Ls],
                      A, [-x for x in G], b, float(d['dt']), float(d['prefac']), 0.81, Pr, cv, model)
    wf, wU = d[f'{model}:bdf{q}:f'], d[f'{model}:bdf{q}:U']
    assert np.linalg.norm(f - wf) / np.linalg.norm(wf - fs[-1]) < 1e-12
    assert np.abs(U - wU).max() / np.abs(wU).max() < 1e-13
