"""CPU checks of the oracle itself, pinned to the reference's own numbers.

Pins (no reference test suite exists; these are the numbers its logs print):
  * Newell self-coupling N(0) for thickness 1, printed by every FFT run,
    e.g. src/irregular/2d_fft/2d_i1/scaling_logs/fft_1536x512.txt:8-9 and
    2d_i1/result.txt:10-11: diag(-4.5733e+00, -4.5733e+00, -3.4198e+00),
    off-diagonal tab = -1.10e-17, tac = tbc = 0; strength-scaled (x2)
    -9.1465e+00 / -6.8397e+00 (fft_1536x512.txt:13).
  * FFT demag equals the direct O(N^2) convolution (the reference's only
    quantitative cross-check, 2d_i1/result.txt FFT vs direct).
"""
import json
import os

import numpy as np
import pytest

import llg
from conftest import rel_err

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load_gold(name):
    with open(os.path.join(GOLD, name)) as f:
        return json.load(f)


def test_newell_self_coupling_matches_reference_logs(oracle_lib):
    g = load_gold("reference_log_pins.json")
    n = oracle_lib.newell_avg(1.0, 0, 0)
    for comp, key in ((0, "nxx0_unscaled"), (4, "nyy0_unscaled"), (8, "nzz0_unscaled")):
        # printed with %.4e → half a unit in the 4th decimal of the mantissa
        assert abs(n[comp] - g[key]) <= 0.5e-4 * abs(g[key]) + 1e-12, (comp, n[comp], g[key])
    assert abs(n[1] - g["tab_offdiag"]) < 0.006e-17
    assert n[2] == 0.0 and n[5] == 0.0
    assert abs(n[0] + n[4] + n[8] + 4 * np.pi) < 1e-3  # trace -4 pi (reference comment)


def test_self_coupling_scaled_by_strength(oracle_lib):
    g = load_gold("reference_log_pins.json")
    p = llg.default_params(16, 16, demag_mode=llg.DEMAG_PERIODIC, demag_strength=2.0, bc=llg.BC_PERIODIC)
    o = oracle_lib.Oracle(p)
    s = o.demag_self()
    for v, key in zip(s, ("nxx0_strength2", "nyy0_strength2", "nzz0_strength2")):
        assert abs(v - g[key]) <= 0.5e-4 * abs(g[key])


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 8, 12, 37, 60, 64, 96, 1024, 3072])
def test_oracle_fft_matches_numpy(oracle_lib, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert rel_err(oracle_lib.fft(x), np.fft.fft(x)) < 1e-13
    assert rel_err(oracle_lib.fft(x, +1), np.fft.ifft(x) * n) < 1e-13


@pytest.mark.parametrize("mode,ng,ny", [(llg.DEMAG_PERIODIC, 13, 7), (llg.DEMAG_PERIODIC, 16, 8),
                                        (llg.DEMAG_OPEN, 12, 9), (llg.DEMAG_OPEN, 7, 5)])
def test_demag_fft_equals_direct(oracle_lib, mode, ng, ny):
    p = llg.default_params(ng, ny, demag_mode=mode, demag_strength=2.5, bc=llg.BC_PERIODIC)
    o = oracle_lib.Oracle(p)
    y = np.random.default_rng(1).standard_normal(3 * ng * ny)
    assert rel_err(o.demag(y), o.demag(y, direct=True)) < 1e-12


def test_uniform_film_demag_is_local_limit(oracle_lib):
    """Open boundaries, uniform in-plane m: field at the centre approaches the
    thin-film limit (h_x ~ 0 far from edges, h_z ~ -strength*4pi*m_z)."""
    ng = ny = 64
    p = llg.default_params(ng, ny, demag_mode=llg.DEMAG_OPEN, demag_strength=1.0, bc=llg.BC_PERIODIC)
    o = oracle_lib.Oracle(p)
    n = ng * ny
    y = np.zeros(3 * n)
    y[2 * n:] = 1.0
    h = o.demag(y)
    c = (ny // 2) * ng + ng // 2
    assert h[2 * n + c] < -0.9 * 4 * np.pi
    assert abs(h[c]) < 1e-9 and abs(h[n + c]) < 1e-9


@pytest.mark.parametrize("aniso", [llg.ANISO_LINEAR, llg.ANISO_CUBIC])
@pytest.mark.parametrize("windowed", [0, 1])
@pytest.mark.parametrize("bc", [llg.BC_PERIODIC, llg.BC_FREE])
def test_jv_is_exact_derivative_without_demag(oracle_lib, aniso, windowed, bc):
    ng, ny = 9, 6
    p = llg.default_params(ng, ny, aniso_kind=aniso, chb=0.3, bc=bc, jv_mode=llg.JV_FULL_FIELD,
                           msk=(1, 1, 1) if aniso == llg.ANISO_CUBIC else (1, 0, 0), windowed=windowed)
    o = oracle_lib.Oracle(p)
    rng = np.random.default_rng(7)
    n = ng * ny
    if windowed:
        o.set_window(rng.uniform(0, 1, n), rng.standard_normal(3 * n), rng.standard_normal(3 * n))
    y = rng.standard_normal(3 * n)
    v = rng.standard_normal(3 * n)
    eps = 1e-6
    fd = (o.rhs(y + eps * v) - o.rhs(y - eps * v)) / (2 * eps)
    assert rel_err(o.jtv(v, y), fd) < 1e-8


def test_reference_jv_omits_applied_field(oracle_lib):
    """The reference Jv builds h from exchange + anisotropy only (2d_i2/jtv.cu:87-97)."""
    ng, ny = 8, 5
    p_ref = llg.default_params(ng, ny, happ=(0.0, 0.0, 0.3))
    p_full = llg.default_params(ng, ny, happ=(0.0, 0.0, 0.3), jv_mode=llg.JV_FULL_FIELD)
    y = np.random.default_rng(2).standard_normal(3 * ng * ny)
    v = np.random.default_rng(3).standard_normal(3 * ng * ny)
    a = oracle_lib.Oracle(p_ref).jtv(v, y)
    b = oracle_lib.Oracle(p_full).jtv(v, y)
    assert np.abs(a - b).max() > 1e-3


@pytest.mark.parametrize("aniso", [llg.ANISO_LINEAR, llg.ANISO_CUBIC])
def test_block_jacobi_inverts_local_block(oracle_lib, aniso):
    """P^-1 (I - gamma J_local) = I per cell, J_local by finite differences of f
    in the cell's own m with neighbours and demag frozen."""
    ng, ny = 6, 5
    p = llg.default_params(ng, ny, aniso_kind=aniso, bc=llg.BC_PERIODIC, chb=0.2,
                           msk=(1, 1, 1) if aniso == llg.ANISO_CUBIC else (1, 0, 0))
    o = oracle_lib.Oracle(p)
    n = ng * ny
    rng = np.random.default_rng(11)
    y = rng.standard_normal(3 * n)
    gamma = 0.37
    o.rhs(y.copy())
    o.psetup(y, gamma)
    P = o.pinv().reshape(9, n)
    cell = 13
    J = np.zeros((3, 3))
    eps = 1e-6
    for b in range(3):
        yp = y.copy(); yp[b * n + cell] += eps
        ym = y.copy(); ym[b * n + cell] -= eps
        fp = o.rhs(yp); fm = o.rhs(ym)
        J[:, b] = (fp[[cell, n + cell, 2 * n + cell]] - fm[[cell, n + cell, 2 * n + cell]]) / (2 * eps)
    A = np.eye(3) - gamma * J
    Pi = P[:, cell].reshape(3, 3)
    assert np.abs(Pi @ A - np.eye(3)).max() < 1e-7


def test_rhs_preserves_norm_direction(oracle_lib):
    """m · dm/dt = alpha (m·h)(1 - |m|^2) → 0 for unit m (torque is orthogonal)."""
    ng, ny = 10, 7
    p = llg.default_params(ng, ny, bc=llg.BC_PERIODIC, demag_mode=llg.DEMAG_OPEN, demag_strength=1.0)
    o = oracle_lib.Oracle(p)
    n = ng * ny
    y = np.random.default_rng(5).standard_normal(3 * n).reshape(3, n)
    y /= np.linalg.norm(y, axis=0)
    yd = o.rhs(y.ravel().copy()).reshape(3, n)
    assert np.abs((y * yd).sum(axis=0)).max() < 1e-12


def test_oracle_integrator_config0_runs(oracle_lib):
    """Config 0 (128x64, t 0→2 here) integrates with CVODE-like counters."""
    p = llg.default_params(128, 64)
    o = oracle_lib.Oracle(p)
    geo = oracle_lib.build_geometry(llg.default_geom(128, 64, ic_jitter_eps=0.01))
    o.integrator_init(geo["y0"], llg.default_solver_opts())
    t = 0.0
    for k in range(20):
        rc, t, y = o.integrate(0.1 * (k + 1))
        assert rc == 0
    st = o.stats()
    assert st["nst"] > 10 and st["nfe"] >= st["nst"] and st["nli"] > 0
    assert np.isfinite(y).all()
    assert abs(t - 2.0) < 1e-12


def test_integrator_flags_nonfinite_state(oracle_lib):
    """A NaN planted in y is caught by the WRMS-norm check (CV_BAD_STATE),
    not by a fault."""
    p = llg.default_params(16, 8)
    o = oracle_lib.Oracle(p)
    geo = oracle_lib.build_geometry(llg.default_geom(16, 8, ic_jitter_eps=0.01))
    y0 = geo["y0"].copy()
    y0[5] = np.nan
    o.integrator_init(y0, llg.default_solver_opts())
    rc, t, y = o.integrate(0.1)
    assert rc == -40   # CV_BAD_STATE: the weights of a NaN state are not "non-positive"
