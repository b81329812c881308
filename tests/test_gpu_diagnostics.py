"""FP64 conservation diagnostics computed on the device
(demsph_dem_diagnostics, demsph_sph_diagnostics) against the same sums
taken on the host from the state read back, and the balances they exist
for: fluid mass constant to the last bit, ball-ball and bond forces summing
to zero, momentum of an isolated pack conserved."""
import numpy as np
import pytest

from this_studio_b200 import scenes
from this_studio_b200.scenes import build_dem, build_sph

pytestmark = pytest.mark.gpu


def _close(a, b, tol, scale=None):
    a, b = np.atleast_1d(a), np.atleast_1d(b)
    s = scale if scale is not None else max(np.linalg.norm(b), 1e-300)
    return np.linalg.norm(a - b) / s < tol


def _world_inverse_inertia(q, inv6):
    """R I^-1 R^T for the clump orientation q = (q0, q1, q2, q3) and the
    body-frame inverse inertia (xx, yy, zz, xy, xz, yz)."""
    q0, q1, q2, q3 = q
    R = np.array([[1 - 2 * q2 * q2 - 2 * q3 * q3, 2 * (q1 * q2 - q0 * q3), 2 * (q1 * q3 + q0 * q2)],
                  [2 * (q1 * q2 + q0 * q3), 1 - 2 * q1 * q1 - 2 * q3 * q3, 2 * (q2 * q3 - q0 * q1)],
                  [2 * (q1 * q3 - q0 * q2), 2 * (q2 * q3 + q0 * q1), 1 - 2 * q1 * q1 - 2 * q2 * q2]])
    xx, yy, zz, xy, xz, yz = inv6
    Ii = np.array([[xx, xy, xz], [xy, yy, yz], [xz, yz, zz]])
    return R @ Ii @ R.T


def test_dem_diagnostics_match_host_sums(gpu):
    sc = scenes.dem_pack(n_side=8)
    rng = np.random.default_rng(3)
    r = 0.004
    for k in range(6):  # free clumps above the pack, spinning
        c = np.array([0.01 + 0.015 * k, 0.02, 0.2])
        ax = rng.normal(size=3)
        ax /= np.linalg.norm(ax)
        m = 3 * 4 / 3 * np.pi * r ** 3 * 2500
        I = np.array([0.4 * m / 3 * r * r * 3 + 2 * m / 3 * (1.5 * r) ** 2, 0.4 * m / 3 * r * r * 3, 0.5e-8])
        sc.clumps.append(dict(point=c + np.outer([-1, 0, 1], ax) * 1.5 * r, radius=[r, r, r], centroid=c,
                              velocity=tuple(rng.normal(0, 0.1, 3)), angularVelocity=tuple(rng.normal(0, 20, 3)),
                              mass=m, inertia=(I[0], I[1], I[2], 1e-12, -2e-12, 3e-12), material=0))
    sc.maxb = (sc.maxb[0], sc.maxb[1], 0.25)
    g = build_dem(sc, "fp64")
    g.step(7)
    d = g.diagnostics()
    b, cl = g.getBall(), g.getClump()
    nb = sc.position.shape[0]
    m = 4.0 / 3.0 * np.pi * sc.radius ** 3 * sc.density
    v, w, x = b["velocity"][:nb], b["angularVelocity"][:nb], b["position"][:nb]
    P = (m[:, None] * v).sum(0)
    L = (np.cross(x, m[:, None] * v) + (0.4 * m * sc.radius ** 2)[:, None] * w).sum(0)
    KE = 0.5 * (m * (v * v).sum(1)).sum()
    KR = 0.5 * (0.4 * m * sc.radius ** 2 * (w * w).sum(1)).sum()
    M = m.sum()
    for k, c in enumerate(sc.clumps):
        mc = c["mass"]
        xx, yy, zz, xy, xz, yz = c["inertia"]
        Ib = np.array([[xx, xy, xz], [xy, yy, yz], [xz, yz, zz]])
        inv = np.linalg.inv(Ib)
        Iw = np.linalg.inv(_world_inverse_inertia(cl["orientation"][k],
                                                  (inv[0, 0], inv[1, 1], inv[2, 2], inv[0, 1], inv[0, 2], inv[1, 2])))
        vc, wc, xc = cl["velocity"][k], cl["angularVelocity"][k], cl["position"][k]
        P += mc * vc
        L += np.cross(xc, mc * vc) + Iw @ wc
        KE += 0.5 * mc * vc @ vc
        KR += 0.5 * wc @ Iw @ wc
        M += mc
    print(f"P {d['momentum']} L {d['angularMomentum']} KE {d['kineticEnergy']:.6e} KR {d['rotationalEnergy']:.6e}")
    assert _close(d["mass"], M, 1e-13)
    assert _close(d["momentum"], P, 1e-11, scale=M * np.abs(v).max())
    assert _close(d["angularMomentum"], L, 1e-10)
    assert _close(d["kineticEnergy"], KE, 1e-12)
    assert _close(d["rotationalEnergy"], KR, 1e-10)
    assert _close(d["forceSum"], b["force"].sum(0), 1e-12, scale=np.abs(b["force"]).sum())


def test_dem_isolated_pack_conserves_momentum(gpu):
    sc = scenes.dem_pack(n_side=10)
    sc.gravity = (0.0, 0.0, 0.0)
    g = build_dem(sc, "fp64")
    d0 = g.diagnostics()
    g.step(40)
    d1 = g.diagnostics()
    scale = d0["mass"] * np.abs(sc.velocity).max()
    drift = np.linalg.norm(d1["momentum"] - d0["momentum"]) / scale
    f = g.getBall()["force"]
    print(f"isolated pack: momentum drift {drift:.2e}, force sum {np.linalg.norm(d1['forceSum']):.2e} "
          f"of {np.abs(f).sum():.2e}, KE {d0['kineticEnergy']:.4e} -> {d1['kineticEnergy']:.4e}")
    assert drift < 1e-12
    assert np.linalg.norm(d1["forceSum"]) < 1e-12 * np.abs(f).sum()


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_sph_diagnostics_match_host_sums_and_mass_is_constant(gpu, prec):
    sc = scenes.dam_break_reference()
    g = build_sph(sc, prec)
    d0 = g.diagnostics()
    g.step(25)
    d = g.diagnostics()
    s = g.getSPH()
    n = sc.fluid.shape[0]
    m = np.full(n, sc.spacing ** 3 * sc.density)
    gv = np.array(sc.gravity)
    v = s["velocity"]
    host = {"mass": m.sum(), "momentum": (m[:, None] * v).sum(0), "kineticEnergy": 0.5 * (m * (v * v).sum(1)).sum(),
            "potentialEnergy": -(m * (s["position"] @ gv)).sum(), "densityChangeSum": s["densityChange"].sum(),
            "volume": (m / s["density"]).sum()}
    print(f"{prec}: {d}")
    assert d["mass"] == d0["mass"]  # masses never change: the same bits
    assert _close(d["mass"], host["mass"], 1e-13)
    assert _close(d["momentum"], host["momentum"], 1e-11, scale=host["mass"] * np.abs(v).max())
    assert _close(d["kineticEnergy"], host["kineticEnergy"], 1e-12)
    assert _close(d["potentialEnergy"], host["potentialEnergy"], 1e-12)
    assert _close(d["densityChangeSum"], host["densityChangeSum"], 1e-11, scale=np.abs(s["densityChange"]).sum())
    assert _close(d["volume"], host["volume"], 1e-13)
    # the column starts to fall: potential energy goes into kinetic energy
    assert d["potentialEnergy"] < d0["potentialEnergy"] and d["kineticEnergy"] > d0["kineticEnergy"]
