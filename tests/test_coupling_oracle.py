"""Particle-level DEM-SPH coupling in the oracle (CPU): the marker layout
of a ball, Newton's third law between the fluid and the balls (total linear
momentum of a free fluid block and a ball moving through it is conserved
to rounding), and a ball's force from a still tank (hydrostatic buoyancy
points up and is of the order of the displaced weight)."""
import math

import numpy as np

from this_studio_b200 import scenes

from .helpers import coupled_momentum, oracle_coupled


def _expected_counts(R, dx, h):
    out = []
    l = 0
    while l * dx < 2.0 * h:
        r = R - (l + 0.5) * dx
        if not r > 0.25 * dx:
            break
        out.append((r, max(1, int(round(4.0 * math.pi * r * r / (dx * dx))))))
        l += 1
    return out


def test_marker_shells(oracle_lib):
    sc = scenes.balls_in_tank(nx=12, ny=12, depth=12, balls=((0.5, 0.5, 0.5, 4.0, 500.0),
                                                          (0.2, 0.2, 0.3, 0.5, 500.0)))
    f, d = oracle_coupled(sc)
    m = f.markers()
    dx, h = sc.marker_spacing, sc.marker_h
    shells = _expected_counts(4 * dx, dx, h)
    assert [n for _, n in shells] == [154, 79, 28]
    assert (m["ball"] == 0).sum() == sum(n for _, n in shells)
    # a ball of radius dx/2 has no shell: one marker at its centre
    assert (m["ball"] == 1).sum() == 1
    off = m["pos"] - sc.dem.position[m["ball"]]
    r = np.linalg.norm(off, axis=1)
    k = 0
    for rl, n in shells:
        assert np.allclose(r[k:k + n], rl, rtol=0, atol=1e-15)
        k += n
    big = m["ball"] == 0
    assert np.allclose(np.linalg.norm(m["normal"][big], axis=1), 1.0, atol=1e-15)
    assert np.allclose(m["normal"][big] * r[big, None], off[big], atol=1e-15)
    assert np.all(m["normal"][~big] == 0)
    # balls at rest: markers at rest
    assert np.all(m["vel"] == 0)


def test_momentum_exchange_is_exact(oracle_lib):
    """No gravity, no walls: the fluid's momentum changes only through the
    markers, and the balls receive the exact negative."""
    v0 = np.array([[0.8, -0.3, 0.2]])
    sc = scenes.balls_in_tank(nx=14, ny=14, depth=14, balls=((0.5, 0.5, 0.5, 3.0, 800.0),), ball_velocity=v0,
                              gravity=(0.0, 0.0, 0.0), walls=False)
    f, d = oracle_coupled(sc)
    p0 = coupled_momentum(sc, np.zeros((len(sc.sph.fluid), 3)), v0)
    f.couple_step(d, 6, sc.dem_substeps)
    st, b = f.state(), d.balls()
    p1 = coupled_momentum(sc, st["vel"], b["vel"])
    ball, F, T = f.coupling(d, 1)
    mb = sc.dem.density[0] * (4.0 / 3.0) * math.pi * sc.dem.radius[0] ** 3
    # the ball was slowed by the fluid, and the fluid carries what it lost
    assert np.linalg.norm(F) > 0 and np.dot(F[0], v0[0]) < 0
    drift = np.linalg.norm(p1 - p0) / (mb * np.linalg.norm(v0))
    print(f"momentum drift over 6 coupled steps: {drift:.2e}")
    assert drift < 1e-12


def hydrostatic(sc):
    """(rho, p, drho) of the fluid at rest under gravity: p = rho0 g (H - z)."""
    sp = sc.sph
    H = sp.fluid[:, 2].max() + 0.5 * sp.spacing
    p = sp.density * 9.81 * (H - sp.fluid[:, 2])
    drho = p / sp.sound_speed ** 2
    return sp.density + drho, p, drho


def test_still_tank_buoyancy(oracle_lib):
    """A ball in still water at hydrostatic pressure: the fluid pushes it up
    by roughly the weight of the water it displaces."""
    sc = scenes.balls_in_tank(nx=16, ny=16, depth=20, balls=((0.5, 0.5, 0.45, 4.0, 1000.0),))
    f, d = oracle_coupled(sc)
    rho, p, drho = hydrostatic(sc)
    f.set_state(rho=rho, p=p, drho=drho)
    f.couple_step(d, 1, sc.dem_substeps)
    _, F, _ = f.coupling(d, 1)
    R = sc.dem.radius[0]
    W = sc.sph.density * 9.81 * (4.0 / 3.0) * math.pi * R ** 3
    print(f"buoyancy {F[0]}, displaced weight {W:.4g}")
    assert F[0, 2] > 0.3 * W and F[0, 2] < 3.0 * W
    assert abs(F[0, 0]) < 0.2 * W and abs(F[0, 1]) < 0.2 * W
