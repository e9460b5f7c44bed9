"""Solution export (nrpyell_interpolate_solution): the SinhSymTP inverse map
and the Lagrange interpolation reproduce polynomials of the interpolation
order exactly, grid values at grid points, and the ADM assembly has the
conformally flat structure and the known Bowen-York answer on the axis of a
boosted puncture."""
import ctypes as C

import numpy as np
import pytest

from nrpyelliptic_b200 import _lib
from nrpyelliptic_b200.export import interpolate
from nrpyelliptic_b200.problem import CONFIGS, Config, DeviceState, Problem, Punctures, with_grid

pytestmark = pytest.mark.gpu


def to_cart(p, xx0, xx1, xx2):
    A = p.AMAX * np.sinh(xx0 / p.SINHWAA) / np.sinh(1.0 / p.SINHWAA)
    return np.stack([A * np.sin(xx1) * np.cos(xx2), A * np.sin(xx1) * np.sin(xx2),
                     np.sqrt(A * A + p.bScale ** 2) * np.cos(xx1)], axis=-1)


@pytest.fixture(scope="module")
def lib():
    lib = _lib.load()
    lib.nrpyell_clear_status()
    return lib


def test_polynomials_of_the_order_are_reproduced(lib):
    prob = Problem(with_grid(CONFIGS["shipped_64x64x8"], (48, 32, 8)), lib=lib)
    ds = DeviceState(prob, lib=lib)
    x0, x1, x2 = prob.xx_arrays()
    X0, X1, X2 = np.meshgrid(x0, x1, x2, indexing="ij")
    f = lambda a, b, c: 1 + 2 * a - 0.7 * b ** 2 + 0.3 * a * b * c + 0.05 * c ** 4 + a ** 4 * b ** 3
    y = prob.zero_state()
    y[:prob.Ntot] = f(X0, X1, X2).transpose(2, 1, 0).ravel()  # i0 fastest
    ds.set_state(y)
    rng = np.random.default_rng(1)
    n = 500
    q0 = rng.uniform(x0[5], x0[-6], n)
    q1 = rng.uniform(x1[5], x1[-6], n)
    q2 = rng.uniform(-3.0, 3.0, n)
    uu, _, _, _ = interpolate(prob, ds, to_cart(prob.params, q0, q1, q2), order=4)
    ref = f(q0, q1, q2)
    assert np.max(np.abs(uu - ref)) < 1e-9 * np.max(np.abs(ref))
    ds.free()


def test_grid_values_at_grid_points(lib):
    prob = Problem(CONFIGS["shipped_64x64x8"], lib=lib)
    ds = DeviceState(prob, lib=lib)
    steps, fin = C.c_int(0), C.c_double(0)
    lib.nrpyell_relax(C.byref(ds.g), prob.dt, -8.0, 4000, 100.0, C.byref(steps), C.byref(fin), None)
    _lib.check(lib)
    x0, x1, x2 = prob.xx_arrays()
    u = ds.download("y_n", prob.Ntot).reshape(prob.N[2], prob.N[1], prob.N[0])
    rng = np.random.default_rng(2)
    i0 = rng.integers(8, prob.N[0] - 8, 200)
    i1 = rng.integers(8, prob.N[1] - 8, 200)
    i2 = rng.integers(5, prob.N[2] - 5, 200)
    uu, psi, gamma, K = interpolate(prob, ds, to_cart(prob.params, x0[i0], x1[i1], x2[i2]), order=4)
    ref = u[i2, i1, i0]
    assert np.max(np.abs(uu - ref)) < 1e-10 * np.max(np.abs(u))
    assert np.allclose(gamma[:, [1, 2, 4]], 0) and np.allclose(gamma[:, 0], psi ** 4, rtol=1e-15)
    assert np.allclose(gamma[:, 3], gamma[:, 0]) and np.allclose(gamma[:, 5], gamma[:, 0])
    trK = K[:, 0] + K[:, 3] + K[:, 5]
    assert np.max(np.abs(trK)) < 1e-12 * np.max(np.abs(K))
    ds.free()


def test_boosted_puncture_on_its_axis(lib):
    """One puncture at the origin with momentum P along x (the other with zero
    mass, momentum and spin, far away): on the x axis Abar_xx = 3 P x / r^3."""
    pu = Punctures(m0=0.5, m1=0.0, pos0=(0.0, 0.0, 0.0), pos1=(0.0, 0.0, -50.0), P0=(0.2, 0.0, 0.0),
                   P1=(0.0, 0.0, 0.0), S0=(0.0, 0.0, 0.0), S1=(0.0, 0.0, 0.0))
    prob = Problem(Config("boosted", (32, 16, 8), pu, bScale=5.0), lib=lib)
    ds = DeviceState(prob, lib=lib)  # uu = 0
    xs = np.array([1.5, 3.0, 7.0])
    pts = np.stack([xs, 0 * xs, 0 * xs], axis=1)
    uu, psi, _, K = interpolate(prob, ds, pts, order=4)
    assert np.allclose(uu, 0.0)
    assert np.allclose(psi, 1 + 0.5 / (2 * xs), rtol=1e-14)
    assert np.allclose(K[:, 0], 3 * 0.2 * xs / xs ** 3 / psi ** 2, rtol=1e-12)
    ds.free()


def test_initial_lapse_options_match_their_formulas(lib):
    """nrpyell_initial_lapse against the thorn's two formulas written out in
    numpy (conformally_flat_BBH_lapse_power_of_psi_initial_data.c,
    conformally_flat_BBH_lapse_averaged_initial_data.c), at random points
    and with uu interpolated from a relaxed solution."""
    from nrpyelliptic_b200.export import initial_lapse
    prob = Problem(CONFIGS["shipped_64x64x8"], lib=lib)
    ds = DeviceState(prob, lib=lib)
    st, fin = C.c_int(0), C.c_double(0)
    assert lib.nrpyell_relax(C.byref(ds.g), prob.dt, -10.0, 4000, 100.0, C.byref(st), C.byref(fin), None) == 0
    p = prob.params
    rng = np.random.default_rng(5)
    xyz = rng.uniform(-8.0, 8.0, (200, 3))
    uu = interpolate(prob, ds, xyz)[0]
    r0 = np.linalg.norm(xyz - [p.puncture_0_x, p.puncture_0_y, p.puncture_0_z], axis=1)
    r1 = np.linalg.norm(xyz - [p.puncture_1_x, p.puncture_1_y, p.puncture_1_z], axis=1)
    s = 0.5 * p.bare_mass_0 / r0 + 0.5 * p.bare_mass_1 / r1
    for n in (-2.0, 1.5):
        a = initial_lapse(prob, xyz, uu, mode="psi^n", exponent=n)
        np.testing.assert_allclose(a, (1.0 + s + uu) ** n, rtol=1e-13)
    a = initial_lapse(prob, xyz, mode="averaged")
    np.testing.assert_allclose(a, 0.5 * (1.0 - s) / (1.0 + s) + 0.5, rtol=1e-14)
    # an unknown mode is an error
    out = np.zeros(1)
    P = lambda v: v.ctypes.data_as(C.POINTER(C.c_double))
    assert lib.nrpyell_initial_lapse(C.byref(p), 1, P(xyz[:1].copy()), P(uu[:1].copy()), 7, 0.0, P(out)) == -1
    lib.nrpyell_clear_status()
    ds.free()
