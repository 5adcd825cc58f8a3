"""Record the compressed-ephemeris golden fixtures (tests/golden/ephemeris/*.npz).

Synthetic orbital sample series (two-body orbits of several shapes, a perturbed orbit and non-Keplerian
tracks) go through the reference's own compressor, `ephemeris_compressor::compress_orbital_data`
(src/modules/ephemeris_compressor.cpp:164-399), and rotational series (a fast principal spin, a slow tumble,
a tidally locked moon with its orbit) through `compress_rotational_data` (ephemeris_compressor.cpp:401-530),
via oracle/_ref/ephc (built by `make -C oracle ephc` from
the reference sources). Each fixture keeps the compressed record exactly as the reference writes it, the
time span, evaluation times, and the reference interpolator's {r, v, GM} at those times
(ephemeris_compressor.cpp:1036-1053), on the B-spline form as loaded and after expand().

Run from the repository root: python tests/golden/make_ephemeris_golden.py
(EPH_GOLDEN_EPHEMERIS_DIR writes the fixtures elsewhere, for the reproducibility test.)
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
EPHC = os.path.join(ROOT, "oracle", "_ref", "ephc")
OUT = os.environ.get("EPH_GOLDEN_EPHEMERIS_DIR", os.path.join(HERE, "ephemeris"))
DAY = 86400.0


def kepler_states(gm, a, e, inc, node, argp, m0, ts):
    """Two-body states (r, v) at times ts of an elliptic orbit (Kepler's equation by Newton steps)."""
    n = np.sqrt(gm / a ** 3)
    M = m0 + n * ts
    E = M.copy()
    for _ in range(60):
        E -= (E - e * np.sin(E) - M) / (1 - e * np.cos(E))
    cE, sE = np.cos(E), np.sin(E)
    b = a * np.sqrt(1 - e * e)
    xp, yp = a * (cE - e), b * sE
    rdot = n * a / (1 - e * cE)
    vxp, vyp = -a * sE * rdot / a, b * cE * rdot / a
    co, so, ci, si, cw, sw = np.cos(node), np.sin(node), np.cos(inc), np.sin(inc), np.cos(argp), np.sin(argp)
    R = np.array([[co * cw - so * sw * ci, -co * sw - so * cw * ci, so * si],
                  [so * cw + co * sw * ci, -so * sw + co * cw * ci, -co * si],
                  [sw * si, cw * si, ci]])
    r = np.stack([xp, yp, np.zeros_like(xp)], 1) @ R.T
    v = np.stack([vxp, vyp, np.zeros_like(xp)], 1) @ R.T
    return r, v


def hyperbolic_states(gm, q, e, inc, node, argp, t_peri, ts):
    """Two-body states of a hyperbolic orbit (periapsis distance q, eccentricity e > 1, periapsis at t_peri)."""
    a = q / (e - 1)
    n = np.sqrt(gm / a ** 3)
    M = n * (ts - t_peri)
    H = np.arcsinh(M / e)
    for _ in range(80):
        H -= (e * np.sinh(H) - H - M) / (e * np.cosh(H) - 1)
    ch, sh = np.cosh(H), np.sinh(H)
    b = a * np.sqrt(e * e - 1)
    xp, yp = a * (e - ch), b * sh
    hdot = n / (e * ch - 1)
    vxp, vyp = -a * sh * hdot, b * ch * hdot
    co, so, ci, si, cw, sw = np.cos(node), np.sin(node), np.cos(inc), np.sin(inc), np.cos(argp), np.sin(argp)
    R = np.array([[co * cw - so * sw * ci, -co * sw - so * cw * ci, so * si],
                  [so * cw + co * sw * ci, -so * sw + co * cw * ci, -co * si],
                  [sw * si, cw * si, ci]])
    r = np.stack([xp, yp, np.zeros_like(xp)], 1) @ R.T
    v = np.stack([vxp, vyp, np.zeros_like(xp)], 1) @ R.T
    return r, v


def cases():
    rng = np.random.default_rng(2024)
    gm_earth, gm_sun = 3.986004418e14, 1.32712440018e20
    out = []
    # near-circular moon orbit, two revolutions
    ts = np.linspace(0, 54 * DAY, 433)
    out.append(("moon_circular", ts, *kepler_states(gm_earth, 3.844e8, 0.0549, 0.09, 2.1, 0.6, 0.3, ts)))
    # eccentric planet orbit over half a revolution
    ts = np.linspace(0, 600 * DAY, 301)
    out.append(("planet_eccentric", ts, *kepler_states(gm_sun, 2.77 * 1.496e11, 0.62, 0.18, 1.3, 4.0, 0.2, ts)))
    # comet-like orbit near perihelion
    ts = np.linspace(0, 120 * DAY, 241)
    out.append(("comet_perihelion", ts, *kepler_states(gm_sun, 18.0 * 1.496e11, 0.967, 2.83, 1.02, 1.94, -0.02, ts)))
    # Kepler orbit with a small periodic perturbation (GM inferred, elements slowly varying)
    ts = np.linspace(0, 30 * DAY, 361)
    r, v = kepler_states(gm_earth, 4.2164e7, 0.01, 0.02, 0.5, 0.1, 0.0, ts)
    w = 2 * np.pi / (13.7 * DAY)
    amp = 2.0e3
    r = r + amp * np.stack([np.sin(w * ts), np.cos(w * ts), 0.3 * np.sin(2 * w * ts)], 1)
    v = v + amp * w * np.stack([np.cos(w * ts), -np.sin(w * ts), 0.6 * np.cos(2 * w * ts)], 1)
    out.append(("geo_perturbed", ts, r, v))
    # non-Keplerian track (no central mass fits): a drifting, gently curving path
    ts = np.linspace(0, 10 * DAY, 201)
    r = np.stack([1.0e9 + 3.0e3 * ts, -2.0e8 + 50.0 * ts + 1.0e7 * np.sin(ts / (3 * DAY)), 4.0e6 * np.cos(ts / (5 * DAY))], 1)
    v = np.stack([np.full_like(ts, 3.0e3), 50.0 + 1.0e7 / (3 * DAY) * np.cos(ts / (3 * DAY)),
                  -4.0e6 / (5 * DAY) * np.sin(ts / (5 * DAY))], 1)
    out.append(("drift_track", ts, r, v))
    # a track accelerated away from the origin (no positive GM fits): state-vector record
    ts = np.linspace(0, 4 * DAY, 161)
    r0, v0, acc = np.array([2.0e9, 1.0e9, -5.0e8]), np.array([1.0e3, -4.0e3, 2.0e2]), np.array([2.0e-2, 1.0e-2, -5.0e-3])
    r = r0 + np.outer(ts, v0) + 0.5 * np.outer(ts * ts, acc) + 1.0e5 * np.stack(
        [np.sin(ts / DAY), np.cos(ts / (2 * DAY)), np.sin(ts / (3 * DAY))], 1)
    v = v0 + np.outer(ts, acc) + 1.0e5 * np.stack(
        [np.cos(ts / DAY) / DAY, -np.sin(ts / (2 * DAY)) / (2 * DAY), np.cos(ts / (3 * DAY)) / (3 * DAY)], 1)
    out.append(("outward_track", ts, r, v))
    # hyperbolic flyby through periapsis, and a mildly hyperbolic interstellar-like comet
    ts = np.linspace(0, 8 * DAY, 321)
    out.append(("flyby_hyperbolic", ts, *hyperbolic_states(gm_earth, 7.0e6, 1.8, 0.7, 0.4, 1.1, 4 * DAY, ts)))
    ts = np.linspace(0, 200 * DAY, 401)
    out.append(("comet_hyperbolic", ts, *hyperbolic_states(gm_sun, 0.25 * 1.496e11, 1.2, 2.2, 0.3, 2.0, 90 * DAY, ts)))
    # near-parabolic comets through perihelion (e = 0.9995 and 1.0005)
    ts = np.linspace(0, 60 * DAY, 241)
    q = 0.4 * 1.496e11
    out.append(("comet_near_parabolic_e", ts, *kepler_states(gm_sun, q / (1 - 0.9995), 0.9995, 1.9, 0.5, 2.4,
                                                             -np.sqrt(gm_sun / (q / 0.0005) ** 3) * 30 * DAY, ts)))
    out.append(("comet_near_parabolic_h", ts, *hyperbolic_states(gm_sun, q, 1.0005, 1.9, 0.5, 2.4, 30 * DAY, ts)))
    # short series: few samples (low B-spline degree)
    ts = np.linspace(0, 2 * DAY, 5)
    out.append(("moon_short", ts, *kepler_states(gm_earth, 3.844e8, 0.0549, 0.09, 2.1, 0.6, 1.0, ts)))
    rng.random()
    return out


def rot(axis, ang):
    """Rotation matrices [len(ang)][3][3] about a unit axis by angles ang (Rodrigues)."""
    a = np.asarray(axis, float) / np.linalg.norm(axis)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    ang = np.atleast_1d(ang)
    return np.eye(3) + np.sin(ang)[:, None, None] * K + (1 - np.cos(ang))[:, None, None] * (K @ K)


def rotational_cases():
    """(name, times, w, x, z, orbital (r, v) or None): body-frame axes x, z and angular velocity w."""
    out = []
    R0 = rot([0.3, -0.5, 0.8], [0.7])[0]
    # fast principal spin (about 0.6 turn per sample): only the axial form applies
    ts = np.linspace(0, 10 * DAY, 41)
    n, om = np.array([0.1, 0.2, 0.97]) / np.linalg.norm([0.1, 0.2, 0.97]), 2 * np.pi / (10 * 3600.0)
    R = rot(n, om * ts) @ R0
    out.append(("spin_fast", ts, np.tile(om * n, (len(ts), 1)), R[:, :, 0], R[:, :, 2], None))
    # slow tumbling (precession about a perpendicular axis): the body-frame spin axis wanders
    ts = np.linspace(0, 2 * DAY, 97)
    n1, n2, Om, om = np.array([0.0, 0.0, 1.0]), np.array([1.0, 0.0, 0.0]), 2 * np.pi / (1.1 * DAY), 2 * np.pi / (0.9 * DAY)
    A, B = rot(n1, Om * ts), rot(n2, om * ts)
    R = A @ B @ R0
    w = Om * n1 + om * (A @ n2)
    out.append(("tumble_slow", ts, w, R[:, :, 0], R[:, :, 2], None))
    # tidally locked moon with a small libration about the orbit normal
    ts = np.linspace(0, 27 * DAY, 325)
    r, v = kepler_states(3.986004418e14, 3.844e8, 0.0549, 0.09, 2.1, 0.6, 0.3, ts)
    h = np.cross(r, v)
    zh = h / np.linalg.norm(h, axis=1)[:, None]
    xh = -r / np.linalg.norm(r, axis=1)[:, None]
    yh = np.cross(zh, xh)
    lib_n = 2 * np.pi / (27.5 * DAY)
    lam, dlam = 0.02 * np.sin(lib_n * ts), 0.02 * lib_n * np.cos(lib_n * ts)
    x = np.cos(lam)[:, None] * xh + np.sin(lam)[:, None] * yh
    w = h / np.einsum("ij,ij->i", r, r)[:, None] + dlam[:, None] * zh
    out.append(("moon_locked", ts, w, x, zh, (r, v)))
    return out


def eval_times(span, rng):
    t = np.concatenate([[0.0, span], span * np.array([1e-6, 0.003, 0.01, 0.02, 0.5, 0.98, 0.99, 0.997, 1 - 1e-6]),
                        np.sort(rng.uniform(0, span, 48))])
    return np.clip(t, 0.0, span)


def main():
    if not os.path.exists(EPHC):
        sys.exit("oracle/_ref/ephc is missing: run make -C oracle ephc")
    os.makedirs(OUT, exist_ok=True)
    rng = np.random.default_rng(77)
    with tempfile.TemporaryDirectory() as td:
        for name, ts, r, v in cases():
            span = float(ts[-1] - ts[0])
            tev = eval_times(span, rng)
            raw = np.concatenate([r, v], 1).astype(np.float64)
            fin, fblob, fev = (os.path.join(td, x) for x in ("in", "blob", "ev"))
            with open(fin, "wb") as f:
                f.write(np.int64(len(ts)).tobytes() + np.float64(span).tobytes() + raw.tobytes()
                        + np.int64(len(tev)).tobytes() + tev.tobytes())
            subprocess.run([EPHC, "orbital", fin, fblob, fev], check=True)
            blob = np.fromfile(fblob, np.uint8)
            ev = np.fromfile(fev, np.uint8)
            level, fmt = np.frombuffer(ev[:16].tobytes(), np.int64)
            vals = np.frombuffer(ev[16:].tobytes(), np.float64).reshape(2, len(tev), 7) if level > 0 else np.zeros((2, 0, 7))
            np.savez_compressed(os.path.join(OUT, name + ".npz"), blob=blob, span=span, times=tev, level=level,
                                format=fmt, loaded=vals[0], expanded=vals[1])
            print(f"{name:18s} level {level} format {fmt} blob {len(blob)} bytes")
        for name, ts, w, x, z, orbit in rotational_cases():
            span = float(ts[-1] - ts[0])
            tev = eval_times(span, rng)
            raw = np.concatenate([w, x, z], 1).astype(np.float64)
            fin, fblob, fev, forb = (os.path.join(td, s) for s in ("in", "blob", "ev", "orb"))
            with open(fin, "wb") as f:
                f.write(np.int64(len(ts)).tobytes() + np.float64(span).tobytes() + raw.tobytes()
                        + np.int64(len(tev)).tobytes() + tev.tobytes())
            cmd = [EPHC, "rotational", fin, fblob, fev]
            if orbit is not None:
                with open(forb, "wb") as f:
                    f.write(np.int64(len(ts)).tobytes() + np.float64(span).tobytes()
                            + np.concatenate(orbit, 1).astype(np.float64).tobytes())
                cmd.append(forb)
            subprocess.run(cmd, check=True)
            blob = np.fromfile(fblob, np.uint8)
            ev = np.fromfile(fev, np.uint8)
            level, fmt = np.frombuffer(ev[:16].tobytes(), np.int64)
            vals = np.frombuffer(ev[16:].tobytes(), np.float64).reshape(2, len(tev), 15) if level > 0 else np.zeros((2, 0, 15))
            np.savez_compressed(os.path.join(OUT, name + ".npz"), blob=blob, span=span, times=tev, level=level,
                                format=fmt, loaded=vals[0], expanded=vals[1])
            print(f"{name:18s} level {level} format {fmt} blob {len(blob)} bytes")


if __name__ == "__main__":
    main()
