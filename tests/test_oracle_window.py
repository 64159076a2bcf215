"""CPU checks of the oracle's adjoint chained over a window of steps, the
reference the window adjoint's GPU tests are held to: four unlimited
tracer steps, each with its own winds and densities, and a tendency held
for every step (as a surface emission is).  The chain of one-step
adjoints in reverse, with the tendencies' adjoint summed over the steps,
must satisfy <y, x_N> = <lam_0, x_0> + <sum_k lam_sct_k, E> (the window is
linear in the initial tracers x_0 and the tendency E for fixed winds), and
a central difference along a seeded direction must equal the gradient's
projection on it."""
import numpy as np
import pytest

import oracle_lib
from olam_b200 import abi

NSTEPS, NTR = 4, 2


@pytest.fixture(scope="module")
def window():
    from olam_b200.synth.grid import build_grid, stretched_levels
    from olam_b200.synth.state import transport_state
    g = build_grid(5, stretched_levels(10, 100.0, 30000.0), seed=8)
    states = [transport_state(g, 1800.0, NTR, seed=20 + k) for k in range(NSTEPS)]
    return g, states, abi.make_opts(1800.0, nrk_scal=3)


def _forward(g, states, opts, x0, e):
    fg = abi.FortranGrid(g)
    x = [np.asarray(t, np.float64) for t in x0]
    for st in states:
        x = list(oracle_lib.scalar_transport(fg, opts, x, e, st, fp64=True))
    return x


def _adjoint(g, states, opts, y):
    fg = abi.FortranGrid(g)
    lam = [np.asarray(t, np.float64) for t in y]
    lsum = [np.zeros((g.mwa, g.mza)) for _ in range(NTR)]
    for st in reversed(states):
        la, ls = oracle_lib.scalar_transport_adjoint(fg, opts, lam, st, fp64=True)
        lam = list(la)
        lsum = [a + b for a, b in zip(lsum, ls)]
    return lam, lsum


def _fields(g, rng, scale=1.0):
    out = []
    for _ in range(NTR):
        a = scale * rng.standard_normal((g.mwa, g.mza))
        a[0] = 0.0          # the dummy column
        a[:, 0] = 0.0       # the level below ground
        out.append(a)
    return out


def test_window_chain_identity(window):
    g, states, opts = window
    rng = np.random.default_rng(3)
    x0, e, y = _fields(g, rng), _fields(g, rng, 1e-4), _fields(g, rng)
    xn = _forward(g, states, opts, x0, e)
    lam0, lsum = _adjoint(g, states, opts, y)
    lhs = sum(float(np.vdot(xn[n], y[n])) for n in range(NTR))
    rhs = sum(float(np.vdot(x0[n], lam0[n]) + np.vdot(e[n], lsum[n])) for n in range(NTR))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs), (lhs, rhs)


def test_window_chain_against_central_differences(window):
    g, states, opts = window
    rng = np.random.default_rng(5)
    x0, e, y = _fields(g, rng), _fields(g, rng, 1e-4), _fields(g, rng)
    lam0, lsum = _adjoint(g, states, opts, y)

    def J(x, ee):
        xn = _forward(g, states, opts, x, ee)
        return sum(float(np.vdot(xn[n], y[n])) for n in range(NTR))
    for _ in range(3):
        dx, de = _fields(g, rng), _fields(g, rng, 1e-4)
        h = 0.25
        fd = (J([a + h * b for a, b in zip(x0, dx)], [a + h * b for a, b in zip(e, de)])
              - J([a - h * b for a, b in zip(x0, dx)], [a - h * b for a, b in zip(e, de)])) / (2 * h)
        proj = sum(float(np.vdot(lam0[n], dx[n]) + np.vdot(lsum[n], de[n])) for n in range(NTR))
        assert abs(fd - proj) <= 1e-10 * abs(fd), (fd, proj)
