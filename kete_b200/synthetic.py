"""Seeded synthetic inputs: populations of orbital states and a DAF/SPK type-2 ephemeris.

No real planetary ephemeris (DE440s) or survey data is available offline, so every
workload is generated here from a seed:

* ``write_synthetic_spk`` fits degree-13 Chebyshev records to seeded Keplerian orbits
  for the Sun, the eight planetary barycentres, the Earth-Moon barycentre, the Earth and
  the Moon, and writes them as a little-endian DAF/SPK file with type-2 segments.  The
  centre tree copies DE440s: bodies 1-8 and 10 are given relative to the solar-system
  barycentre (0); the Earth (399) and Moon (301) relative to the Earth-Moon barycentre
  (3); positions are km in the J2000 equatorial frame (frame code 1), times are TDB
  seconds past J2000 -- the NAIF SPK type-2 layout ("Chebyshev, position only").
* ``main_belt`` / ``neo`` / ``mixed`` draw orbital elements with the distributions of the
  benchmark configurations and convert them to heliocentric ecliptic states with the
  cometary-elements conversion of kete (kete_core/elements.rs:190-264).
"""
from __future__ import annotations

import struct

import numpy as np

GMS = 0.00029591220828411956
GMS_SQRT = 0.01720209894996
AU_KM = 149597870.7
OBLIQUITY = 0.40909280422232897
J2000 = 2451545.0
EPOCH = 2460000.5

# mass ratios (fraction of the Sun) of the perturbers, kete_core/constants/gravity.rs:43-134
MASS_RATIO = {
    1: 1.66012082548908e-07,
    2: 2.44783828779694e-06,
    399: 3.00348961546514e-06,
    301: 3.69430335010988e-08,
    4: 3.22715608291416e-07,
    5: 0.0009547919099414246,
    6: 0.00028588567002459455,
    7: 4.36624961322212e-05,
    8: 5.15138377265457e-05,
}
PLANET_A = {1: 0.387, 2: 0.723, 3: 1.0, 4: 1.524, 5: 5.203, 6: 9.537, 7: 19.19, 8: 30.07}


# ---------------------------------------------------------------------------------------------
# Kepler helpers (vectorised numpy; input generation only)
# ---------------------------------------------------------------------------------------------
def _ecc_anomaly(m, e):
    m = np.mod(m, 2 * np.pi)
    E = np.where(e < 0.8, m, np.pi * np.ones_like(m))
    for _ in range(60):
        f = E - e * np.sin(E) - m
        E = E - f / (1 - e * np.cos(E))
    return E


def _rotation(inc, lan, argp):
    cw, sw = np.cos(argp), np.sin(argp)
    co, so = np.cos(lan), np.sin(lan)
    ci, si = np.cos(inc), np.sin(inc)
    P = np.stack([cw * co - sw * so * ci, cw * so + sw * co * ci, sw * si])
    Q = np.stack([-sw * co - cw * so * ci, -sw * so + cw * co * ci, cw * si])
    return P, Q


def kepler_state(a, e, inc, lan, argp, m0, epoch, t, mu=GMS):
    """Heliocentric ecliptic position/velocity (AU, AU/day) of an elliptic orbit at t."""
    a, e = np.asarray(a, float), np.asarray(e, float)
    n = np.sqrt(mu / a**3)
    m = m0 + n * (np.asarray(t, float) - epoch)
    E = _ecc_anomaly(m, e)
    cE, sE = np.cos(E), np.sin(E)
    b = a * np.sqrt(1 - e * e)
    x, y = a * (cE - e), b * sE
    edot = n / (1 - e * cE)
    xd, yd = -a * sE * edot, b * cE * edot
    P, Q = _rotation(inc, lan, argp)
    if P.ndim == 1:
        P, Q = P[:, None], Q[:, None]
    return x * P + y * Q, xd * P + yd * Q


def ecl_to_eq(v):
    c, s = np.cos(OBLIQUITY), np.sin(OBLIQUITY)
    v = np.asarray(v, float)
    return np.stack([v[0], c * v[1] - s * v[2], s * v[1] + c * v[2]])


def elements_to_state(epoch, ecc, incl, lon_asc, peri_time, peri_arg, peri_dist):
    """Vectorised elliptic CometElements::to_pos_vel (kete_core/elements.rs:190-264)."""
    ecc = np.asarray(ecc, float)
    a = peri_dist / (1.0 - ecc)
    mean_motion = np.abs(a) ** -1.5 * GMS_SQRT
    mean_anom = mean_motion * (epoch - peri_time)
    E = _ecc_anomaly(mean_anom, ecc)
    sE, cE = np.sin(E), np.cos(E)
    e_dot = a**1.5 * (1.0 - ecc * cE)
    b = a * np.sqrt(1.0 - ecc**2)
    x, y = a * (cE - ecc), b * sE
    xd = -a / e_dot * sE * GMS_SQRT
    yd = b / e_dot * cE * GMS_SQRT
    P, Q = _rotation(incl, lon_asc, peri_arg)
    return x * P + y * Q, xd * P + yd * Q


# ---------------------------------------------------------------------------------------------
# populations
# ---------------------------------------------------------------------------------------------
def _finish(rng, n, a, e, inc, epoch):
    lan = rng.uniform(0, 2 * np.pi, n)
    argp = rng.uniform(0, 2 * np.pi, n)
    m = rng.uniform(0, 2 * np.pi, n)
    peri_dist = a * (1 - e)
    peri_time = epoch - m / (a**-1.5 * GMS_SQRT)
    return elements_to_state(epoch, e, inc, lan, peri_time, argp, peri_dist)


def main_belt(n, seed=0, epoch=EPOCH):
    """a ~ U(2.1, 3.3) AU, e ~ Rayleigh(0.1) clipped < 0.4, i ~ Rayleigh(10 deg)."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(2.1, 3.3, n)
    e = np.minimum(rng.rayleigh(0.1, n), 0.3999)
    inc = np.radians(rng.rayleigh(10.0, n))
    return _finish(rng, n, a, e, inc, epoch)


def neo(n, seed=0, epoch=EPOCH):
    """a ~ U(0.8, 2.5) AU, e ~ U(0.1, 0.7), i ~ Rayleigh(15 deg)."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.8, 2.5, n)
    e = rng.uniform(0.1, 0.7, n)
    inc = np.radians(rng.rayleigh(15.0, n))
    return _finish(rng, n, a, e, inc, epoch)


def mixed(n, seed=0, neo_frac=0.1, nongrav_frac=0.05, epoch=EPOCH):
    """90 % main belt + 10 % NEO; a fraction carries JPL comet A1/A2 non-grav terms.

    Returns pos (3,n), vel (3,n), nongrav (10,n) rows (kind, a1, a2, a3, alpha, r0, m, n, k, dt).
    """
    rng = np.random.default_rng(seed)
    n_neo = int(round(n * neo_frac))
    pm, vm = main_belt(n - n_neo, seed=seed + 1, epoch=epoch)
    pn, vn = neo(n_neo, seed=seed + 2, epoch=epoch)
    pos = np.concatenate([pm, pn], axis=1)
    vel = np.concatenate([vm, vn], axis=1)
    perm = rng.permutation(n)
    pos = np.ascontiguousarray(pos[:, perm])
    vel = np.ascontiguousarray(vel[:, perm])
    ng = np.zeros((10, n))
    has = rng.random(n) < nongrav_frac
    k = int(has.sum())
    ng[0, has] = 1.0
    ng[1, has] = rng.normal(0.0, 1e-8, k)
    ng[2, has] = rng.normal(0.0, 1e-9, k)
    ng[3, has] = 0.0
    ng[4, has], ng[5, has], ng[6, has] = 0.1112620426, 2.808, 2.15
    ng[7, has], ng[8, has], ng[9, has] = 5.093, 4.6142, 0.0
    return pos, vel, ng


def comet_nongrav(a1, a2, a3=0.0):
    """NonGravModel::new_jpl_comet_default as a non-grav row (kete_core/propagation/nongrav.rs:97-109)."""
    return np.array([1.0, a1, a2, a3, 0.1112620426, 2.808, 2.15, 5.093, 4.6142, 0.0])


# ---------------------------------------------------------------------------------------------
# synthetic planetary ephemeris
# ---------------------------------------------------------------------------------------------
def _planet_elements(seed):
    rng = np.random.default_rng(seed)
    el = {}
    for pid, a in PLANET_A.items():
        el[pid] = dict(
            a=a,
            e=rng.uniform(0.0, 0.21) if pid != 3 else 0.0167,
            inc=np.radians(rng.uniform(0.0, 7.0)) if pid != 3 else 0.0,
            lan=rng.uniform(0, 2 * np.pi),
            argp=rng.uniform(0, 2 * np.pi),
            m0=rng.uniform(0, 2 * np.pi),
        )
    return el


def synthetic_bodies(t_jd, seed=2024):
    """Positions/velocities (km, km/s, J2000 equatorial) of the synthetic solar system.

    Returns dict naif_id -> (pos (3,n), vel (3,n), center)."""
    t_jd = np.asarray(t_jd, float)
    el = _planet_elements(seed)
    helio = {}
    for pid, p in el.items():
        helio[pid] = kepler_state(p["a"], p["e"], p["inc"], p["lan"], p["argp"], p["m0"], EPOCH,
                                  t_jd)
    m_emb = MASS_RATIO[399] + MASS_RATIO[301]
    masses = {1: MASS_RATIO[1], 2: MASS_RATIO[2], 3: m_emb, 4: MASS_RATIO[4], 5: MASS_RATIO[5],
              6: MASS_RATIO[6], 7: MASS_RATIO[7], 8: MASS_RATIO[8]}
    total = 1.0 + sum(masses.values())
    sun_p = -sum(masses[k] * helio[k][0] for k in masses) / total
    sun_v = -sum(masses[k] * helio[k][1] for k in masses) / total
    out = {10: (sun_p, sun_v, 0)}
    for pid in masses:
        out[pid] = (helio[pid][0] + sun_p, helio[pid][1] + sun_v, 0)
    # Moon about the Earth: a = 384400 km, e = 0.055, i = 5.1 deg to the ecliptic
    a_m = 384400.0 / AU_KM
    mp, mv = kepler_state(a_m, 0.055, np.radians(5.1), 2.1, 0.7, 1.3, EPOCH, t_jd,
                          mu=GMS * m_emb)
    f_moon = MASS_RATIO[399] / m_emb
    out[399] = (-(1 - f_moon) * mp, -(1 - f_moon) * mv, 3)
    out[301] = (f_moon * mp, f_moon * mv, 3)
    # the five large asteroids kete adds with include_asteroids (gravity.rs:104-133), given
    # relative to the Sun (10) as asteroid SPKs are
    rng = np.random.default_rng(seed + 7)
    for aid in ASTEROIDS:
        a_, e_, i_ = rng.uniform(2.2, 3.2), rng.uniform(0.05, 0.25), np.radians(rng.uniform(2, 20))
        lan, argp, m0 = rng.uniform(0, 2 * np.pi, 3)
        ap, av = kepler_state(a_, e_, i_, lan, argp, m0, EPOCH, t_jd)
        out[aid] = (ap, av, 10)
    res = {}
    for k, (p, v, c) in out.items():
        res[k] = (ecl_to_eq(p) * AU_KM, ecl_to_eq(v) * AU_KM / 86400.0, c)
    return res


def _cheb_nodes(m):
    k = np.arange(m)
    return np.cos(np.pi * (k + 0.5) / m)


def fit_type2_segment(body, jd_start, jd_end, record_days, n_coef=14, seed=2024):
    """Least-squares Chebyshev fit of every type-2 record of one body at once.

    Returns (DAF array data, center id)."""
    n_rec = int(np.ceil((jd_end - jd_start) / record_days))
    nodes = _cheb_nodes(3 * n_coef)
    mids = jd_start + (np.arange(n_rec) + 0.5) * record_days
    rad = record_days / 2.0
    tj = (mids[:, None] + rad * nodes[None, :]).ravel()
    p, _, center = synthetic_bodies(tj, seed)[body]
    vander = np.polynomial.chebyshev.chebvander(nodes, n_coef - 1)  # (m, n_coef)
    pinv = np.linalg.pinv(vander)  # (n_coef, m)
    recs = np.empty((n_rec, 2 + 3 * n_coef))
    recs[:, 0] = (mids - J2000) * 86400.0
    recs[:, 1] = rad * 86400.0
    for c in range(3):
        vals = p[c].reshape(n_rec, nodes.size)
        recs[:, 2 + c * n_coef:2 + (c + 1) * n_coef] = vals @ pinv.T
    tail = np.array([(jd_start - J2000) * 86400.0, record_days * 86400.0, 2 + 3 * n_coef, n_rec])
    return np.concatenate([recs.ravel(), tail]), center


def fit_type3_segment(body, jd_start, jd_end, record_days, n_coef=12, seed=2024):
    """Type-3 records (Chebyshev position and velocity series fitted separately) of one body.

    Returns (DAF array data, center id)."""
    n_rec = int(np.ceil((jd_end - jd_start) / record_days))
    nodes = _cheb_nodes(3 * n_coef)
    mids = jd_start + (np.arange(n_rec) + 0.5) * record_days
    rad = record_days / 2.0
    tj = (mids[:, None] + rad * nodes[None, :]).ravel()
    p, v, center = synthetic_bodies(tj, seed)[body]
    pinv = np.linalg.pinv(np.polynomial.chebyshev.chebvander(nodes, n_coef - 1))
    recs = np.empty((n_rec, 2 + 6 * n_coef))
    recs[:, 0] = (mids - J2000) * 86400.0
    recs[:, 1] = rad * 86400.0
    for c, arr in enumerate((p[0], p[1], p[2], v[0], v[1], v[2])):
        vals = arr.reshape(n_rec, nodes.size)
        recs[:, 2 + c * n_coef:2 + (c + 1) * n_coef] = vals @ pinv.T
    tail = np.array([(jd_start - J2000) * 86400.0, record_days * 86400.0, 2 + 6 * n_coef, n_rec])
    return np.concatenate([recs.ravel(), tail]), center


def read_daf_segments(path):
    """The segments of a DAF/SPK file: list of (target, center, frame, type, start_s, end_s,
    data array), in the file's summary order."""
    buf = open(path, "rb").read()
    e = "<" if buf[88:96] == b"LTL-IEEE" else ">"
    nd, ni = struct.unpack(e + "2i", buf[8:16])
    ss = nd + (ni + 1) // 2
    nxt = struct.unpack(e + "i", buf[76:80])[0]
    out = []
    while nxt:
        off = 1024 * (nxt - 1)
        nxt_d, _, nsum = struct.unpack(e + "3d", buf[off:off + 24])
        for k in range(int(nsum)):
            o = off + 24 + k * ss * 8
            s0, s1 = struct.unpack(e + "2d", buf[o:o + 16])
            tgt, ctr, frm, typ, a0, a1 = struct.unpack(e + "6i", buf[o + 16:o + 40])
            data = np.frombuffer(buf[8 * (a0 - 1):8 * a1], dtype=e + "f8").astype(np.float64)
            out.append((tgt, ctr, frm, typ, s0, s1, data))
        nxt = int(nxt_d)
    return out


def write_daf_spk(path, segments, internal_name="kete_b200 synthetic ephemeris"):
    """Write a little-endian DAF/SPK.  segments: list of (target, center, frame, type,
    start_s, end_s, data)."""
    nd, ni = 2, 6
    ss = nd + (ni + 1) // 2  # summary size in doubles
    assert len(segments) <= (125 - 3) // ss
    # record 1 file record, 2 summary record, 3 name record, data from record 4
    addr = 3 * 128 + 1
    summaries = []
    blobs = []
    for tgt, ctr, frm, typ, s0, s1, data in segments:
        data = np.asarray(data, dtype="<f8")
        start, end = addr, addr + data.size - 1
        summaries.append((s0, s1, tgt, ctr, frm, typ, start, end))
        blobs.append(data)
        addr = end + 1
    free = addr
    rec1 = bytearray(1024)
    rec1[0:8] = b"DAF/SPK "
    rec1[8:12] = struct.pack("<i", nd)
    rec1[12:16] = struct.pack("<i", ni)
    rec1[16:76] = internal_name.ljust(60)[:60].encode()
    rec1[76:80] = struct.pack("<i", 2)
    rec1[80:84] = struct.pack("<i", 2)
    rec1[84:88] = struct.pack("<i", free)
    rec1[88:96] = b"LTL-IEEE"
    ftp = b"FTPSTR:\r:\n:\r\n:\r\x00:\x81:\x10\xce:ENDFTP"
    rec1[699:699 + len(ftp)] = ftp
    rec2 = bytearray(1024)
    rec2[0:24] = struct.pack("<3d", 0.0, 0.0, float(len(summaries)))
    for k, (s0, s1, tgt, ctr, frm, typ, a0, a1) in enumerate(summaries):
        off = 24 + k * ss * 8
        rec2[off:off + 16] = struct.pack("<2d", s0, s1)
        rec2[off + 16:off + 40] = struct.pack("<6i", tgt, ctr, frm, typ, a0, a1)
    rec3 = bytearray(1024)
    for k, s in enumerate(summaries):
        nm = f"BODY {s[2]}".ljust(ss * 8)[: ss * 8].encode()
        rec3[k * ss * 8:(k + 1) * ss * 8] = nm
    body = b"".join(b.tobytes() for b in blobs)
    pad = (-len(body)) % 1024
    with open(path, "wb") as f:
        f.write(bytes(rec1) + bytes(rec2) + bytes(rec3) + body + b"\x00" * pad)


SPK_BODIES = (10, 1, 2, 3, 399, 301, 4, 5, 6, 7, 8)
ASTEROIDS = (20000001, 20000002, 20000004, 20000010, 20000704)


def write_type3_spk(path, bodies=ASTEROIDS[:2], jd_start=2459000.5, jd_end=2461000.5,
                    record_days=16.0, n_coef=12, seed=2024):
    """An SPK of type-3 segments for some of the synthetic asteroids (centre: the Sun)."""
    segs = []
    for body in bodies:
        data, center = fit_type3_segment(body, jd_start, jd_end, record_days, n_coef, seed)
        n_rec = int(data[-1])
        s0 = (jd_start - J2000) * 86400.0
        segs.append((body, center, 1, 3, s0, s0 + n_rec * record_days * 86400.0, data))
    write_daf_spk(path, segs)
    return path


def write_synthetic_spk(path, jd_start=2457000.5, jd_end=2463000.5, record_days=32.0,
                        moon_record_days=8.0, n_coef=14, seed=2024, asteroids=False):
    """Write the synthetic perturber SPK used by the tests and the benchmark.

    n_coef: coefficients per coordinate, one count for every body or a dict body -> count
    (real ephemerides mix counts).  asteroids: also write the five large asteroids."""
    segs = []
    bodies = SPK_BODIES + (ASTEROIDS if asteroids else ())
    for body in bodies:
        rd = moon_record_days if body in (399, 301) else record_days
        nc = n_coef.get(body, 14) if isinstance(n_coef, dict) else n_coef
        data, center = fit_type2_segment(body, jd_start, jd_end, rd, nc, seed)
        n_rec = int(data[-1])
        s0 = (jd_start - J2000) * 86400.0
        s1 = s0 + n_rec * rd * 86400.0
        segs.append((body, center, 1, 2, s0, s1, data))
    write_daf_spk(path, segs)
    return path
