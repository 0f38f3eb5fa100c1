"""Known-answer checks on the GPU that need no reference run (the reference
has no test suite; these are the properties its schemes promise):

* free-stream preservation: a uniform moving state stays uniform, for every
  flux family and precision form;
* the circular Sod problem of fv_up7 keeps its symmetry under the
  transposition x <-> y and the mirror x -> 1 - x;
* the isentropic vortex with mean flow (1, 1) on a periodic [-5, 5]^2
  returns to its initial state after one period (t = 10), with an error
  that falls with resolution.
"""
from __future__ import annotations

import numpy as np
import pytest

import fvstuff_b200 as F
from cases import vortex

pytestmark = pytest.mark.gpu

# (flux, precision, order, extra solver options)
FREESTREAM = [
    ("up_ducros", "f64", 7), ("up_ducros", "f64", 3), ("up_ducros", "f32", 7), ("up_ducros", "f32c", 7),
    ("up_ducros_hll", "f64", 7), ("up_ducros_roe", "f64", 7), ("keep", "f64", 7), ("rec3", "f64", 7),
    ("up_hllc_d2av", "f64", 5), ("up_ducros", "f64", 9), ("up_hllc_d2av", "f64", 9),
]


@pytest.mark.parametrize("flux,prec,order", FREESTREAM)
def test_free_stream_is_preserved(flux, prec, order):
    n, steps = 48, 30
    s = F.Solver(n, order=order, flux=flux, precision=prec, bc="periodic", cfl=0.4)
    s.init_case("uniform", rho=1.3, u=0.7, v=-0.4, p=2.1)
    U0 = s.get_state(layout="prim", interior=True)
    s.step(steps)
    st = s.sync()
    assert st.status == 0 and st.steps == steps
    U = s.get_state(layout="prim", interior=True)
    tol = 1e-13 if prec == "f64" else 2e-6
    for q in range(4):
        assert np.max(np.abs(U[q] - U0[q])) <= tol * max(1.0, np.max(np.abs(U0[q]))), (flux, prec, q)


@pytest.mark.parametrize("prec", ["f64", "f32c"])
def test_circular_sod_keeps_its_symmetry(prec):
    n, steps = 128, 60
    s = F.Solver(n, precision=prec)  # fv_up7's defaults: UP7, reflecting walls, CFL 0.4
    s.init_case("sod")
    s.step(steps)
    assert s.sync().status == 0
    rho, u, v, p = s.get_state(layout="prim", interior=True)   # [j, i]
    tol = (1e-10 if prec == "f64" else 1e-5) * rho.max()
    assert np.max(np.abs(rho - rho.T)) <= tol                     # x <-> y
    assert np.max(np.abs(rho - rho[:, ::-1])) <= tol              # x -> 1 - x
    assert np.max(np.abs(u - v.T)) <= tol * 10                    # velocities swap with the axes
    assert np.max(np.abs(u + u[:, ::-1])) <= tol * 10             # and change sign in the mirror
    assert rho.max() > 2.0 and rho.min() < 1.0                    # the waves have moved


def _vortex_error(n):
    s = F.Solver(n, bc="periodic", x0=-5.0, y0=-5.0, length=10.0, cfl=0.5)
    w0 = vortex(n)
    s.set_state(w0, layout="prim", interior=True)
    st = s.advance(10.0)
    assert st.status == 0 and abs(st.t - 10.0) < 1e-12
    w = s.get_state(layout="prim", interior=True)
    return float(np.sqrt(np.mean((w[0] - w0[0]) ** 2)))


def test_vortex_returns_after_one_period():
    e64, e128 = _vortex_error(64), _vortex_error(128)
    print("isentropic vortex, one period: L2(rho) %.3e at 64^2, %.3e at 128^2 (ratio %.1f)" % (e64, e128, e64 / e128))
    assert e128 < 2e-3
    assert e64 / e128 > 3.0
