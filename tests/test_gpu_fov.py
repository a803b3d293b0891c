"""GPU field-of-view checks against the oracle.

FOV membership must be identical except for objects within 1e-10 rad of a field edge
(those may flip either way); states of visible objects agree to 1e-12 AU (two-body branch)
or 1e-9 AU (n-body branch)."""
import math

import numpy as np
import pytest

from kete_b200 import synthetic

pytestmark = pytest.mark.gpu
EPOCH = synthetic.EPOCH
EDGE_RAD = 1e-10


def _observer(oracle_spk, jd):
    rc, s = oracle_spk.spk_get_state(399, jd, 10, 2)  # Earth, heliocentric ecliptic
    assert rc == 0
    return s


def _population(n, seed):
    pm, vm = synthetic.main_belt(n - n // 5, seed=seed)
    pn, vn = synthetic.neo(n // 5, seed=seed + 1)
    return np.concatenate([pm, pn], axis=1), np.concatenate([vm, vn], axis=1)


def _fields(gpu, oracle_spk, pos, jds, seed, width=1.8, vel=None):
    """Fields pointed at chosen objects (so detections exist) and at random directions; with
    ``vel`` the chosen object is followed to the field's epoch (two-body)."""
    rng = np.random.default_rng(seed)
    fovs = []
    for k, jd in enumerate(jds):
        obs = _observer(oracle_spk, jd)
        if k % 2 == 0:
            i = rng.integers(pos.shape[1])
            p = pos[:, i]
            if vel is not None:
                tp, _, _, _ = oracle_spk.propagate_two_body(pos[:, i:i + 1], vel[:, i:i + 1],
                                                            np.array([EPOCH]), np.array([jd]))
                p = tp[:, 0]
            target = p - obs[:3]
        else:
            target = rng.normal(size=3)
        o = gpu.State("observer", jd, obs[:3], obs[3:], gpu.Frames.Ecliptic, 10)
        fovs.append(gpu.RectangleFOV(target, rng.uniform(0, 90), o, width, width))
    return fovs


def _edge_distance(normals, v):
    v = np.asarray(v) / np.linalg.norm(v)
    return np.min(np.abs(np.asarray(normals).reshape(4, 3) @ v))


def _oracle_check(oracle_spk, fov, pos, vel, jd, dt_limit):
    flags, out7 = oracle_spk.fov_check_visible(fov.ecliptic_column()[:7], fov.normals, pos, vel,
                                               jd, dt_limit)
    return flags, out7


@pytest.fixture(params=[0, 1], ids=["two_pass", "fused"])
def fov_form(request, gpu):
    """Both forms of the field check: linear screen then two-body pairs (default), and the
    fused one-pass kernel."""
    gpu.fov.set_fov_form(request.param)
    yield request.param
    gpu.fov.set_fov_form(0)


@pytest.mark.parametrize("offset_days", [0.5, 4.0])
def test_check_visible_vs_oracle(gpu, oracle_spk, offset_days, fov_form):
    """Linear branch (|dt| < dt_limit) and n-body branch (|dt| >= dt_limit)."""
    n = 4000
    pos, vel = _population(n, 11)
    jd_obj = np.full(n, EPOCH)
    fovs = _fields(gpu, oracle_spk, pos, EPOCH + offset_days + np.linspace(0, 1.0, 12), 12)
    table = np.stack([f.ecliptic_column() for f in fovs], axis=1)
    ff, oo, ss = gpu.fov.fov_check_visible_arrays(pos, vel, jd_obj, None, table, 3.0)
    tol = 1e-12 if offset_days < 3.0 else 1e-9
    total = 0
    for k, f in enumerate(fovs):
        flags, out7 = _oracle_check(oracle_spk, f, pos, vel, jd_obj, 3.0)
        ref = set(np.nonzero(flags)[0].tolist())
        got = set(oo[ff == k].tolist())
        for i in ref ^ got:  # disagreements only at the frame edge
            st = out7[:, i] if i in ref else ss[:, (ff == k) & (oo == i)][:, 0]
            rel = st[1:4] - f.ecliptic_column()[1:4]
            assert _edge_distance(f.normals, rel) < EDGE_RAD, (k, i)
        for i in ref & got:
            g = ss[:, (ff == k) & (oo == i)][:, 0]
            assert np.abs(g[1:4] - out7[1:4, i]).max() < tol
            assert abs(g[0] - out7[0, i]) < 1e-9
        total += len(ref & got)
    assert total >= 6  # the pointed fields do see objects


def test_fov_state_check_schedule_vs_oracle(gpu, oracle_spk):
    """kete.fov_state_check chunking, big/small re-propagation and per-field results.  The
    fields span 200 days, so both re-seeding branches of checks.rs:68-85 fire: the big-step
    copy moves on once a chunk is 50 dt_limit (150 d) from it, and the small-step population
    restarts from the big-step copy while it is 25 dt_limit (75 d) or more away."""
    n = 1500
    pos, vel = _population(n, 21)
    rng = np.random.default_rng(22)
    jds = np.sort(EPOCH + rng.uniform(0.0, 200.0, 45))
    fovs = _fields(gpu, oracle_spk, pos, jds, 23, width=4.0, vel=vel)
    states = [gpu.State(f"o{i}", EPOCH, pos[:, i], vel[:, i]) for i in range(n)]
    res = gpu.fov_state_check(states, fovs, dt_limit=3.0)
    got = {}
    for sim in res:
        got[id(sim.fov)] = {s.desig: s for s in sim.states}
    # oracle restatement of src/kete/rust/fovs/checks.rs:24-110
    dt_limit = 3.0
    chunks, chunk = [], []
    for f in sorted(fovs, key=lambda f: f.jd):
        if chunk and abs(f.jd - chunk[0].jd) >= 2 * dt_limit:
            chunks.append(chunk)
            chunk = []
        chunk.append(f)
    chunks.append(chunk)
    jd, big_jd = EPOCH, EPOCH
    cur = [pos.copy(), vel.copy(), np.ones(n, bool), EPOCH]
    big = [pos.copy(), vel.copy(), np.ones(n, bool), EPOCH]

    def prop(p, target):
        op, ov, st, _, _ = oracle_spk.propagate_n_body(p[0], p[1], p[3], target)
        return [op, ov, p[2] & (st == 0), target]

    n_fields = 0
    reseeds = resets = 0
    for chunk in chunks:
        jd_mean = (chunk[-1].jd + chunk[0].jd) / 2.0
        if abs(jd_mean - big_jd) >= dt_limit * 50:
            big_jd = jd_mean
            big = prop(big, jd)
            reseeds += 1
        if abs(jd_mean - jd) >= dt_limit:
            if abs(jd - big_jd) >= dt_limit * 25:
                cur = [big[0].copy(), big[1].copy(), big[2].copy(), big[3]]
                resets += 1
            jd = jd_mean
            cur = prop(cur, jd)
        idx = np.nonzero(cur[2])[0]
        for f in chunk:
            flags, out7 = oracle_spk.fov_check_visible(f.ecliptic_column()[:7], f.normals,
                                                       cur[0][:, idx], cur[1][:, idx],
                                                       np.full(idx.size, cur[3]), dt_limit)
            ref = {f"o{idx[j]}": out7[:, j] for j in np.nonzero(flags)[0]}
            g = got.get(id(f), {})
            for d in set(ref) ^ set(g):
                st = ref[d] if d in ref else np.concatenate([[g[d].jd], g[d].pos, g[d].vel])
                rel = st[1:4] - f.ecliptic_column()[1:4]
                assert _edge_distance(f.normals, rel) < EDGE_RAD, d
            for d in set(ref) & set(g):
                assert np.abs(g[d].pos - ref[d][1:4]).max() < 1e-9
            n_fields += bool(ref)
    assert n_fields >= 5
    assert reseeds >= 1 and resets >= 1, (reseeds, resets)
    assert len(res) == sum(1 for f in fovs if id(f) in got)


def test_fov_forms_identical(gpu, oracle_spk):
    """The two-pass and fused field checks run the same arithmetic on the same pairs: the
    visible pairs and their states are identical."""
    n = 20000
    pos, vel = _population(n, 31)
    jd_obj = np.full(n, EPOCH)
    fovs = _fields(gpu, oracle_spk, pos, EPOCH + 0.3 + np.linspace(0, 2.0, 40), 32, width=3.0)
    table = np.stack([f.ecliptic_column() for f in fovs], axis=1)
    out = {}
    try:
        for form in (0, 1):
            gpu.fov.set_fov_form(form)
            out[form] = gpu.fov.fov_check_visible_arrays(pos, vel, jd_obj, None, table, 3.0)
    finally:
        gpu.fov.set_fov_form(0)
    (f0, o0, s0), (f1, o1, s1) = out[0], out[1]
    assert len(o0) > 20
    assert np.array_equal(f0, f1) and np.array_equal(o0, o1)
    assert np.array_equal(s0, s1)
