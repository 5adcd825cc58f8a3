"""Seeded synthetic planetary systems written in the reference's own initials formats.

Every system is emitted as the text files the reference loader reads
(src/modules/mass_loader.cpp:67-294 for the config, :324-561 for the Initial/Extra files,
src/physics/geopotential.cpp:8-127 and src/physics/ring.cpp:25-108 for the model files; the formats
are documented in initials/README.md). Both the reference oracle and this package's loader then
ingest identical bytes. Numbers are printed with Python's shortest round-trip repr, so `%lf`
parsing recovers every double exactly.

Workloads (sizes from the benchmark definitions; no public dataset is involved):
  * ``config1``  seed 1001: star + 8 planets + 24 moons (33 bodies), Newtonian + 1PN only.
  * ``config2``  seed 2002: full-shape solar system of 504 bodies with geopotentials (J2-J6 zonal,
                 degree/order-4 tesseral) on the star and 8 planets, time-lagged planet/moon tides,
                 one ringed planet, soft Kuiper-belt masses, radiation pressure and mass loss.
  * ``small_full`` any seed: the config2 recipe scaled down (default 48 bodies) so that every force
                 term is exercised at sizes a scalar CPU oracle finishes in seconds.
"""
from __future__ import annotations

import copy
import math
import os
from dataclasses import dataclass, field

import numpy as np

AU = 1.495978707e11
GM_SUN = 1.32712440018e20
G = 6.67430e-11            # src/math/basic_math.h:21
M_SUN = GM_SUN / G
DAY = 86400.0
DEG = math.pi / 180.0


@dataclass
class Body:
    name: str
    sid: str
    GM: float
    R_km: float               # negative: soft mass (initials/README.md, Radius)
    inertia: float = 0.4
    k2: float = 0.0
    k2r: float = 0.0
    td: float = 0.0
    j2: float = 0.0
    c21: float = 0.0
    c22: float = 0.0
    s21: float = 0.0
    s22: float = 0.0
    tdf: float = 1.0
    gp_factor: float = 0.0
    ring_factor: float = 0.0
    r: tuple = (0.0, 0.0, 0.0)
    v: tuple = (0.0, 0.0, 0.0)
    x_axis: tuple = (1.0, 0.0, 0.0)
    z_axis: tuple = (0.0, 0.0, 1.0)
    w: tuple = (0.0, 0.0, 0.0)


@dataclass
class System:
    bodies: list
    extras: list = field(default_factory=list)     # (sid, key, value)
    geopotentials: dict = field(default_factory=dict)  # sid -> (Nz, Nt, [(n, m, C, S)])
    rings: dict = field(default_factory=dict)        # sid -> [(name, rin_km, rout_km, thick_km, GM)]
    delta_t: float = 4320.0
    tdb: int = 0


def _kepler_state(mu, a, e, inc, node, argp, M):
    """Position and velocity of a Keplerian orbit (standard two-body relations)."""
    E = M
    for _ in range(60):
        dE = (E - e * math.sin(E) - M) / (1.0 - e * math.cos(E))
        E -= dE
        if abs(dE) < 1e-16:
            break
    cE, sE = math.cos(E), math.sin(E)
    b = math.sqrt(1.0 - e * e)
    r = a * (1.0 - e * cE)
    px, py = a * (cE - e), a * b * sE
    f = math.sqrt(mu * a) / r
    vx, vy = -f * sE, f * b * cE
    cO, sO = math.cos(node), math.sin(node)
    ci, si = math.cos(inc), math.sin(inc)
    cw, sw = math.cos(argp), math.sin(argp)
    # rotation R3(node) R1(inc) R3(argp) applied to the perifocal frame
    P = np.array([cO * cw - sO * sw * ci, sO * cw + cO * sw * ci, sw * si])
    Q = np.array([-cO * sw - sO * cw * ci, -sO * sw + cO * cw * ci, cw * si])
    return px * P + py * Q, vx * P + vy * Q


def _radius_km(GM, rho=2000.0):
    m = GM / G
    return (3.0 * m / (4.0 * math.pi * rho)) ** (1.0 / 3.0) / 1000.0


def _loguniform(rng, lo, hi):
    return math.exp(rng.uniform(math.log(lo), math.log(hi)))


def _unit(v):
    v = np.asarray(v, dtype=float)
    return v / np.linalg.norm(v)


def _perp(z, phase):
    """A unit vector perpendicular to z, rotated by `phase` about z."""
    ref = np.array([0.0, 0.0, 1.0]) if abs(z[2]) < 0.9 else np.array([1.0, 0.0, 0.0])
    x0 = _unit(np.cross(ref, z))
    y0 = np.cross(z, x0)
    return math.cos(phase) * x0 + math.sin(phase) * y0


def _spin_frame(rng, orbit_normal, obliquity, period_s):
    n = _unit(orbit_normal)
    tilt_dir = _perp(n, rng.uniform(0, 2 * math.pi))
    z = _unit(math.cos(obliquity) * n + math.sin(obliquity) * tilt_dir)
    x = _perp(z, rng.uniform(0, 2 * math.pi))
    w = z * (2.0 * math.pi / period_s)
    return tuple(x), tuple(z), tuple(w)


def _synchronous_frame(r_rel, v_rel):
    h = np.cross(r_rel, v_rel)
    z = _unit(h)
    x = -np.asarray(r_rel) / np.linalg.norm(r_rel)
    x = _unit(x - np.dot(x, z) * z)
    rate = np.linalg.norm(h) / np.dot(r_rel, r_rel)
    return tuple(x), tuple(z), tuple(z * rate)


def _barycentric(bodies):
    gm = np.array([b.GM for b in bodies])
    r = np.array([b.r for b in bodies])
    v = np.array([b.v for b in bodies])
    rc = (gm[:, None] * r).sum(0) / gm.sum()
    vc = (gm[:, None] * v).sum(0) / gm.sum()
    for b in bodies:
        b.r = tuple(np.asarray(b.r) - rc)
        b.v = tuple(np.asarray(b.v) - vc)


def _moon(rng, idx, host, host_R_km, ratio, a_range, e_max, inc_max, prefix, tidal):
    gm = host.GM * ratio
    a = rng.uniform(*a_range) * host_R_km * 1000.0
    e = rng.uniform(0, e_max)
    inc = rng.uniform(0, inc_max)
    r_rel, v_rel = _kepler_state(host.GM + gm, a, e, inc, rng.uniform(0, 2 * math.pi),
                                 rng.uniform(0, 2 * math.pi), rng.uniform(0, 2 * math.pi))
    m = Body(name=f"{prefix}{idx:03d}", sid=f"{prefix}{idx:03d}", GM=gm, R_km=_radius_km(gm),
             inertia=0.38)
    m.r = tuple(np.asarray(host.r) + r_rel)
    m.v = tuple(np.asarray(host.v) + v_rel)
    if tidal:
        m.k2 = rng.uniform(0.1, 0.5)
        m.k2r = m.k2
        m.td = rng.uniform(1.0, 600.0)
        m.x_axis, m.z_axis, m.w = _synchronous_frame(r_rel, v_rel)
        # The loader subtracts the initial tidal + rotational deformation from the given degree-2
        # harmonics (mass_loader.cpp:544-551) and requires J2 >= 0 afterwards (mass_loader.cpp:50),
        # so the given J2/C22 are the equilibrium deformation plus a small static residual.
        R3_GM = (m.R_km * 1000.0) ** 3 / m.GM
        q = host.GM * R3_GM / float(np.dot(r_rel, r_rel)) ** 1.5
        w2 = float(np.dot(m.w, m.w))
        m.j2 = m.k2r * w2 * R3_GM / 3.0 + m.k2 * q / 2.0 + rng.uniform(1e-5, 1e-4)
        m.c22 = m.k2 * q / 4.0 + rng.uniform(0.0, 1e-5)
    return m


def _add_rotational_j2(b):
    """Given J2 = equilibrium rotational deformation + the drawn static residual (see _moon)."""
    w2 = float(np.dot(b.w, b.w))
    b.j2 += b.k2r * w2 * (b.R_km * 1000.0) ** 3 / b.GM / 3.0


def make_config1(seed: int = 1001) -> System:
    """Star + 8 planets + 24 moons, point-mass Newtonian + 1PN only (33 bodies)."""
    rng = np.random.default_rng(seed)
    star = Body(name="Star", sid="S0", GM=GM_SUN, R_km=6.96e5, inertia=0.4)
    bodies = [star]
    planets = []
    for k in range(8):
        gm = _loguniform(rng, 1e-9, 1e-3) * GM_SUN
        a = _loguniform(rng, 0.4, 30.0) * AU
        r, v = _kepler_state(GM_SUN + gm, a, rng.uniform(0, 0.1), rng.uniform(0, 3 * DEG),
                             rng.uniform(0, 2 * math.pi), rng.uniform(0, 2 * math.pi),
                             rng.uniform(0, 2 * math.pi))
        p = Body(name=f"Planet{k + 1}", sid=f"P{k + 1}", GM=gm, R_km=_radius_km(gm), r=tuple(r), v=tuple(v))
        planets.append(p)
        bodies.append(p)
    for k in range(24):
        host = planets[2 + k % 6]
        ratio = _loguniform(rng, 1e-8, 1e-4)
        bodies.append(_moon(rng, k + 1, host, host.R_km, ratio, (5, 60), 0.05, 3 * DEG, "M", tidal=False))
    _barycentric(bodies)
    return System(bodies=bodies)


def make_ensemble_member(seed: int, n_bodies: int, sigma: float = 1e-9) -> System:
    """The config1 recipe at any size: a star, ceil(n/4) planets and the rest moons (cycled over the
    planets from the third on, or over all planets when there are at most two), point-mass Newtonian +
    1PN. Every planet and moon position and velocity component is then scaled by (1 + sigma * N(0, 1))."""
    rng = np.random.default_rng(seed)
    n_planets = max(1, math.ceil(n_bodies / 4))
    n_moons = max(0, n_bodies - 1 - n_planets)
    star = Body(name="Star", sid="S0", GM=GM_SUN, R_km=6.96e5, inertia=0.4)
    bodies = [star]
    planets = []
    for k in range(n_planets):
        gm = _loguniform(rng, 1e-9, 1e-3) * GM_SUN
        a = _loguniform(rng, 0.4, 30.0) * AU
        r, v = _kepler_state(GM_SUN + gm, a, rng.uniform(0, 0.1), rng.uniform(0, 3 * DEG),
                             rng.uniform(0, 2 * math.pi), rng.uniform(0, 2 * math.pi),
                             rng.uniform(0, 2 * math.pi))
        p = Body(name=f"Planet{k + 1}", sid=f"P{k + 1}", GM=gm, R_km=_radius_km(gm), r=tuple(r), v=tuple(v))
        planets.append(p)
        bodies.append(p)
    first = 2 if n_planets > 2 else 0
    for k in range(n_moons):
        host = planets[first + k % (n_planets - first)]
        ratio = _loguniform(rng, 1e-8, 1e-4)
        bodies.append(_moon(rng, k + 1, host, host.R_km, ratio, (5, 60), 0.05, 3 * DEG, "M", tidal=False))
    for b in bodies[1:]:
        b.r = tuple(np.asarray(b.r) * (1 + sigma * rng.standard_normal(3)))
        b.v = tuple(np.asarray(b.v) * (1 + sigma * rng.standard_normal(3)))
    _barycentric(bodies)
    return System(bodies=bodies)


def make_ensemble(n_sys: int = 512, seed: int = 3003, n_range=(8, 300), steps=(500, 20000)):
    """A batched ensemble: n_sys members of log-uniform size in n_range (member s seeded seed*10^6 + s)
    and integration lengths uniform in `steps`. Returns [(System, n_steps)]."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n_sys):
        n = int(round(_loguniform(rng, *n_range)))
        k = int(rng.integers(steps[0], steps[1] + 1))
        out.append((make_ensemble_member(seed * 1_000_000 + s, n), k))
    return out


def _gp_model(rng, nz=6, nt=4):
    terms = []
    for n in range(3, nz + 1):
        terms.append((n, 0, rng.normal(0, 1e-6) / n, 0.0))
    for n in range(3, nt + 1):
        for m in range(1, n + 1):
            terms.append((n, m, rng.normal(0, 1e-6) / n, rng.normal(0, 1e-6) / n))
    return (nz, nt, terms)


def make_config2(seed: int = 2002, n_planet_moons: int = 77, n_dwarfs: int = 5, n_dwarf_moons: int = 8,
                 n_asteroids: int = 342, n_tno: int = 27, n_kuiper: int = 36) -> System:
    """Full-shape synthetic solar system (504 bodies with the default counts).

    Star + 8 planets carry J2..J6 zonal and degree/order-4 tesseral harmonics; planet and moon tides
    are time-lagged (k2 = k2r ~ U(0.1, 0.5), td ~ U(1, 600) s); planet 6 has a ring annulus of
    1.2-2.3 radii; 36 soft masses form a Kuiper ring at 44 AU.
    """
    rng = np.random.default_rng(seed)
    sysm = System(bodies=[])
    bodies = sysm.bodies
    star = Body(name="Star", sid="S0", GM=GM_SUN, R_km=6.96e5, inertia=0.07, k2=0.03, k2r=0.027, td=0.1)
    star.j2 = rng.uniform(1e-3, 2e-2)
    star.c21, star.c22, star.s21, star.s22 = (rng.normal(0, 1e-6) / 2 for _ in range(4))
    star.x_axis, star.z_axis, star.w = _spin_frame(rng, (0, 0, 1), 7.25 * DEG, 25.38 * DAY)
    star.gp_factor = 1.0
    _add_rotational_j2(star)
    sysm.geopotentials["S0"] = _gp_model(rng)
    bodies.append(star)
    sysm.extras += [("S0", "MassRate", -0.3784717910405785), ("S0", "Luminosity", 3.828e26)]

    planets = []
    a_grid = np.sort(np.array([_loguniform(rng, 0.4, 30.0) for _ in range(8)]))
    for k in range(8):
        gm = _loguniform(rng, 1e-9, 1e-3) * GM_SUN
        a = a_grid[k] * AU
        r, v = _kepler_state(GM_SUN + gm, a, rng.uniform(0, 0.1), rng.uniform(0, 3 * DEG),
                             rng.uniform(0, 2 * math.pi), rng.uniform(0, 2 * math.pi),
                             rng.uniform(0, 2 * math.pi))
        R_km = _radius_km(gm, rho=1300.0 if gm > 1e-6 * GM_SUN else 5000.0)
        p = Body(name=f"Planet{k + 1}", sid=f"P{k + 1}", GM=gm, R_km=R_km, inertia=0.3,
                 r=tuple(r), v=tuple(v))
        p.k2 = rng.uniform(0.1, 0.5)
        p.k2r = p.k2
        p.td = rng.uniform(1.0, 600.0)
        p.j2 = rng.uniform(1e-3, 2e-2)
        p.c21, p.c22, p.s21, p.s22 = (rng.normal(0, 1e-6) / 2 for _ in range(4))
        p.x_axis, p.z_axis, p.w = _spin_frame(rng, np.cross(r, v), rng.uniform(0, 30 * DEG),
                                              rng.uniform(10, 30) * 3600.0)
        p.gp_factor = 1.0
        _add_rotational_j2(p)
        sysm.geopotentials[p.sid] = _gp_model(rng)
        planets.append(p)
        bodies.append(p)
    sysm.extras += [("P3", "Receptance", 1.4), ("P3", "J2Rate", -1.5e-18), ("P4", "Receptance", 1.2)]
    ringed = planets[5]
    ringed.ring_factor = 1.0
    sysm.rings[ringed.sid] = [("Annulus", 1.2 * ringed.R_km, 2.3 * ringed.R_km, 2.0, 3e-8 * ringed.GM)]

    for k in range(n_planet_moons):
        host = planets[2 + k % 6]
        ratio = _loguniform(rng, 1e-8, 1e-4)
        m = _moon(rng, k + 1, host, host.R_km, ratio, (5, 60), 0.05, 3 * DEG, "M", tidal=True)
        bodies.append(m)
        if k % 5 == 0:
            sysm.extras.append((m.sid, "Receptance", 1.1))

    dwarfs = []
    for k in range(n_dwarfs):
        gm = _loguniform(rng, 1e-9, 5e-9) * GM_SUN
        a = rng.uniform(35.0, 68.0) * AU
        r, v = _kepler_state(GM_SUN + gm, a, rng.uniform(0, 0.3), rng.uniform(0, 20 * DEG),
                             rng.uniform(0, 2 * math.pi), rng.uniform(0, 2 * math.pi),
                             rng.uniform(0, 2 * math.pi))
        d = Body(name=f"Dwarf{k + 1}", sid=f"D{k + 1}", GM=gm, R_km=_radius_km(gm), inertia=0.34,
                 r=tuple(r), v=tuple(v))
        dwarfs.append(d)
        bodies.append(d)
    for k in range(n_dwarf_moons):
        host = dwarfs[k % len(dwarfs)] if dwarfs else planets[7]
        ratio = _loguniform(rng, 1e-4, 1e-1)
        bodies.append(_moon(rng, k + 1, host, host.R_km, ratio, (5, 60), 0.05, 30 * DEG, "DM", tidal=False))

    for k in range(n_asteroids):
        gm = _loguniform(rng, 1e-16, 1e-10) * GM_SUN
        a = rng.uniform(2.1, 3.3) * AU
        r, v = _kepler_state(GM_SUN + gm, a, rng.uniform(0, 0.25), rng.uniform(0, 20 * DEG),
                             rng.uniform(0, 2 * math.pi), rng.uniform(0, 2 * math.pi),
                             rng.uniform(0, 2 * math.pi))
        ast = Body(name=f"Asteroid{k + 1}", sid=f"A{k + 1:04d}", GM=gm, R_km=_radius_km(gm),
                   r=tuple(r), v=tuple(v))
        bodies.append(ast)
        if k % 17 == 0:
            sysm.extras.append((ast.sid, "Receptance", 1.0))

    for k in range(n_tno):
        gm = _loguniform(rng, 1e-12, 1e-9) * GM_SUN
        a = rng.uniform(35.0, 50.0) * AU
        r, v = _kepler_state(GM_SUN + gm, a, rng.uniform(0, 0.2), rng.uniform(0, 20 * DEG),
                             rng.uniform(0, 2 * math.pi), rng.uniform(0, 2 * math.pi),
                             rng.uniform(0, 2 * math.pi))
        bodies.append(Body(name=f"TNO{k + 1}", sid=f"T{k + 1:03d}", GM=gm, R_km=_radius_km(gm),
                           r=tuple(r), v=tuple(v)))

    for k in range(n_kuiper):
        gm = 2.5e11
        lon = 2 * math.pi * k / max(n_kuiper, 1)
        r, v = _kepler_state(GM_SUN + gm, 44.0 * AU, 0.0, 0.0, 0.0, 0.0, lon)
        bodies.append(Body(name=f"Kuiper{k + 1}", sid=f"K{k + 1:03d}", GM=gm, R_km=-5.584e8, inertia=0.36,
                           r=tuple(r), v=tuple(v)))
    _barycentric(bodies)
    return sysm


def make_ringed_subsystem(seed: int = 6006, n_moons: int = 4, ring_ratio: float = 0.05,
                          gp_scale: float = 3.0) -> System:
    """An isolated planetary subsystem for conservation checks: a spinning, oblate, tidally deformable
    planet with J3..J6 / degree-4 geopotential (scaled by gp_scale), a massive ring annulus of 1.2-2.3
    radii (ring_ratio of the planet's GM) and n_moons synchronous, tidally locked moons. The subsystem's
    barycentre sits at 9.5 AU and moves at 9.6 km/s, so its total momenta are far from zero."""
    rng = np.random.default_rng(seed)
    sysm = System(bodies=[], delta_t=900.0)
    gm = 3.7931e16
    p = Body(name="Planet", sid="P6", GM=gm, R_km=58232.0, inertia=0.22, k2=0.34, k2r=0.34, td=600.0)
    p.j2 = 0.0163
    p.c21, p.c22, p.s21, p.s22 = (rng.normal(0, 1e-6) / 2 for _ in range(4))
    p.x_axis, p.z_axis, p.w = _spin_frame(rng, (0, 0, 1), 26.7 * DEG, 10.6 * 3600.0)
    p.gp_factor = gp_scale
    _add_rotational_j2(p)
    sysm.geopotentials[p.sid] = _gp_model(rng)
    p.ring_factor = 1.0
    sysm.rings[p.sid] = [("Annulus", 1.2 * p.R_km, 2.3 * p.R_km, 2.0, ring_ratio * gm)]
    bodies = [p]
    for k in range(n_moons):
        bodies.append(_moon(rng, k + 1, p, p.R_km, _loguniform(rng, 1e-6, 1e-4), (3, 20), 0.02, 1 * DEG, "M",
                            tidal=True))
    _barycentric(bodies)
    bulk_r, bulk_v = np.array([9.5 * AU, 0.0, 0.0]), np.array([0.0, 9.6e3, 0.4e3])
    for b in bodies:
        b.r = tuple(np.asarray(b.r) + bulk_r)
        b.v = tuple(np.asarray(b.v) + bulk_v)
    sysm.bodies = bodies
    return sysm


def make_config5(seed: int = 5005, n_particles: int = 2_000_000, j2: float = 2e-4, particle_seed: int | None = None):
    """Massless test particles against 9 perturbers: the star and the 8 planets of make_config1(1001)
    (its moons left out, the nine re-centred on their barycentre), the star given a static J2 and a zonal
    J3-J4 geopotential (coefficients N(0, 1e-6) / n drawn from `seed`); Newtonian + 1PN otherwise.
    Particles: a ~ U(1.5, 50) AU, e ~ U(0, 0.3), i ~ U(0, 20 deg), angles uniform, on heliocentric Kepler
    orbits about the star (drawn from `seed`, or from `particle_seed` when given: shards of one workload
    share the perturbers and differ in particles). Returns (perturber System, particles [6][n]:
    x, y, z, vx, vy, vz)."""
    base = make_config1(1001)
    bodies = [copy.deepcopy(b) for b in base.bodies[:9]]
    star = bodies[0]
    star.j2 = j2
    star.gp_factor = 1.0
    _barycentric(bodies)
    rng = np.random.default_rng(seed)
    sysm = System(bodies=bodies, delta_t=43200.0)
    sysm.geopotentials["S0"] = (4, 0, [(n, 0, rng.normal(0, 1e-6) / n, 0.0) for n in (3, 4)])
    if particle_seed is not None:
        rng = np.random.default_rng(particle_seed)
    n = n_particles
    a = rng.uniform(1.5, 50.0, n) * AU
    return sysm, kepler_cloud(rng, GM_SUN, a, rng.uniform(0.0, 0.3, n), rng.uniform(0.0, 20 * DEG, n), star.r, star.v)


def kepler_cloud(rng, gm: float, a, e, inc, center_r, center_v) -> np.ndarray:
    """Particles on Kepler orbits of semi-major axes a, eccentricities e and inclinations inc (arrays) about
    a centre of mass gm at (center_r, center_v); node, argument of pericentre and mean anomaly uniform.
    Returns [6][n]: x, y, z, vx, vy, vz."""
    n = len(a)
    node, argp, M = (rng.uniform(0, 2 * math.pi, n) for _ in range(3))
    E = M.copy()   # Kepler's equation by Newton iteration, vectorised
    for _ in range(30):
        E = E - (E - e * np.sin(E) - M) / (1 - e * np.cos(E))
    cE, sE = np.cos(E), np.sin(E)
    px, py = a * (cE - e), a * np.sqrt(1 - e * e) * sE
    nmot = np.sqrt(gm / a ** 3)
    vx, vy = -a * nmot * sE / (1 - e * cE), a * nmot * np.sqrt(1 - e * e) * cE / (1 - e * cE)
    cO, sO, cw, sw, ci, si = np.cos(node), np.sin(node), np.cos(argp), np.sin(argp), np.cos(inc), np.sin(inc)
    P = np.array([cO * cw - sO * sw * ci, sO * cw + cO * sw * ci, sw * si])
    Q = np.array([-cO * sw - sO * cw * ci, -sO * sw + cO * cw * ci, cw * si])
    pos = px * P + py * Q + np.asarray(center_r, np.float64)[:, None]
    vel = vx * P + vy * Q + np.asarray(center_v, np.float64)[:, None]
    return np.concatenate([pos, vel]).astype(np.float64)


def with_test_bodies(sysm: System, particles: np.ndarray, gm: float = 1e-20) -> System:
    """The perturbers plus the particles as bodies of negligible mass (the reference's equivalent of
    massless particles), appended after the perturbers."""
    bodies = list(sysm.bodies)
    for k in range(particles.shape[1]):
        bodies.append(Body(name=f"T{k}", sid=f"T{k}", GM=gm, R_km=1e-3, inertia=0.4,
                           r=tuple(particles[0:3, k]), v=tuple(particles[3:6, k])))
    return System(bodies=bodies, extras=sysm.extras, geopotentials=sysm.geopotentials, rings=sysm.rings,
                  delta_t=sysm.delta_t, tdb=sysm.tdb)


def make_small_full(seed: int = 7007, n_bodies: int = 48) -> System:
    """The config2 recipe at reduced counts: every force term present, ~n_bodies bodies."""
    rest = max(n_bodies - 9, 8)
    moons = max(rest * 77 // 495, 6)
    return make_config2(seed, n_planet_moons=moons, n_dwarfs=1, n_dwarf_moons=1,
                        n_asteroids=max(rest - moons - 6, 1), n_tno=2, n_kuiper=2)


def _fmt(x) -> str:
    return repr(float(x))


def write_system(sysm: System, directory: str, integrator: str = "GPU_RK12", cadence: float | None = None) -> str:
    """Write config, Initial, Extra, Geopotentials/ and Rings/ files; returns the config path."""
    os.makedirs(directory, exist_ok=True)
    init_lines = ["#Name\tID\tGM\tRadius(km)\tinertia\tk2\tk2r\ttd\tJ2\tC21\tC22\tS21\tS22\tTidalDelayFactor\t"
                  "Geopotential\tRing\tx\ty\tz\tvx\tvy\tvz\talpha\tdelta\tw\tperiod(h)\txx\txy\txz\tzx\tzy\tzz\twx\twy\twz"]
    for b in sysm.bodies:
        vals = [b.GM, b.R_km, b.inertia, b.k2, b.k2r, b.td, b.j2, b.c21, b.c22, b.s21, b.s22, b.tdf,
                b.gp_factor, b.ring_factor, *b.r, *b.v, 0.0, 90.0, 0.0, 1.0, *b.x_axis, *b.z_axis, *b.w]
        init_lines.append("\t".join([b.name, b.sid] + [_fmt(x) for x in vals]))
    with open(os.path.join(directory, "Initial.txt"), "w") as f:
        f.write("\n".join(init_lines) + "\n")
    cfg = ["#synthetic system written by ephemeris_b200.synth", "Initial\tInitial.txt"]
    if sysm.extras:
        with open(os.path.join(directory, "Extra.txt"), "w") as f:
            f.write("#sid\tparam\tvalue\n")
            for sid, key, val in sysm.extras:
                f.write(f"{sid}\t{key}\t{_fmt(val)}\n")
        cfg.append("Extra\tExtra.txt")
    if sysm.geopotentials:
        gdir = os.path.join(directory, "Geopotentials")
        os.makedirs(gdir, exist_ok=True)
        for sid, (nz, nt, terms) in sysm.geopotentials.items():
            with open(os.path.join(gdir, f"{sid}.txt"), "w") as f:
                f.write(f"{nz}\t{nt}\n")
                for n, m, c, s in terms:
                    f.write(f"{n}\t{m}\t{_fmt(c)}\t{_fmt(s)}\n")
        cfg.append("Geopotentials\tGeopotentials")
    if sysm.rings:
        rdir = os.path.join(directory, "Rings")
        os.makedirs(rdir, exist_ok=True)
        for sid, annuli in sysm.rings.items():
            with open(os.path.join(rdir, f"{sid}.txt"), "w") as f:
                f.write("#name\tRin(km)\tRout\tThick\tGM\n")
                for name, rin, rout, thick, gm in annuli:
                    f.write(f"{name}\t{_fmt(rin)}\t{_fmt(rout)}\t{_fmt(thick)}\t{_fmt(gm)}\n")
        cfg.append("Rings\tRings")
    dt = sysm.delta_t
    cfg += [f"TDB\t{int(sysm.tdb)}", f"Integrator\t{integrator}", f"Delta_t\t{_fmt(dt)}",
            f"Cadence\t{_fmt(cadence if cadence else dt * 20)}", "Max_Ephemeris_Length\t631152000"]
    path = os.path.join(directory, "Config.txt")
    with open(path, "w") as f:
        f.write("\n".join(cfg) + "\n")
    return path


WORKLOADS = {
    "config1": make_config1,
    "config2": make_config2,
    "small_full": make_small_full,
}


def write_workload(name: str, directory: str, seed: int | None = None, **kw) -> str:
    maker = WORKLOADS[name]
    sysm = maker(seed, **kw) if seed is not None else maker(**kw)
    return write_system(sysm, directory)


def make_config4_system(seed: int = 4004) -> System:
    """Perturbers of the serving workload: the config2 recipe (seeded) with every moon merged into its
    host (GM summed, barycentric position and velocity), all bodies point masses (Newtonian + 1PN).
    A 1-day-knot B-spline cannot follow a moon's hours-to-days orbit, so the ephemeris carries the
    planetary (and dwarf) system barycentres, as small-body ephemerides do."""
    full = make_config2(seed)
    hosts = [b for b in full.bodies if b.sid[0] in "SPDAKT" and not b.sid.startswith("DM")]
    moons = [b for b in full.bodies if b.sid.startswith("M") or b.sid.startswith("DM")]
    groups = {b.sid: [b] for b in hosts}
    cand = [b for b in hosts if b.sid[0] in "PD"]
    for m in moons:
        host = min(cand, key=lambda h: float(np.sum((np.asarray(h.r) - np.asarray(m.r)) ** 2)))
        groups[host.sid].append(m)
    bodies = []
    for h in hosts:
        g = groups[h.sid]
        gm = sum(b.GM for b in g)
        r = sum(b.GM * np.asarray(b.r) for b in g) / gm
        v = sum(b.GM * np.asarray(b.v) for b in g) / gm
        bodies.append(Body(name=h.name, sid=h.sid, GM=gm, R_km=h.R_km, inertia=0.4, r=tuple(r), v=tuple(v)))
    return System(bodies=bodies, delta_t=43200.0)


def make_requests(rng, count: int, span: float, p_max: int = 4096, a_range=(0.5, 50.0), e_max: float = 0.6,
                  inc_max_deg: float = 20.0, years=(1.0, 100.0), star_r=(0.0, 0.0, 0.0), star_v=(0.0, 0.0, 0.0)):
    """Serving requests: P = round(log-U(1, p_max)) particles with a ~ U(a_range) AU, e ~ U(0, e_max),
    i ~ U(0, inc_max) on Kepler orbits about the star's state (star_r, star_v) at the ephemeris start, and a
    duration log-U(years) in years (capped to the span) from that start. Returns [(particles [6][P], t_end)]."""
    out = []
    for _ in range(count):
        p = int(round(_loguniform(rng, 1.0, float(p_max))))
        a = rng.uniform(*a_range, p) * AU
        parts = kepler_cloud(rng, GM_SUN, a, rng.uniform(0, e_max, p), rng.uniform(0, inc_max_deg * DEG, p), star_r, star_v)
        out.append((parts, min(_loguniform(rng, *years) * 365.25 * 86400.0, span)))
    return out
