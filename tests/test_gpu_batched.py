"""GPU parity of the batched uneven N-body configuration at its own spans, and the device
step bound.

1) Objects drawn as the 1M-object batched workload (90% main belt, 10% NEO, 5% with JPL comet
   A1/A2), each propagated to its own target epoch drawn uniform in +-5 years, against the
   oracle (kete_core/propagation/mod.rs:70-118 with RadauIntegrator::integrate,
   radau.rs:160-218, and spk_accel, acceleration.rs:121-168).  Tolerance: positions within
   1e-9 AU for every object whose closest planet approach stays above 0.01 AU; the objects
   that pass closer are counted and reported separately (their chaotic growth of
   rounding-level differences is physical, not an error of either side).
2) The bounded step loop: with a step limit of a few attempts, a one-year propagation
   returns the Timeout status and NaN states from every kernel form, and the library works
   normally afterwards (no kernel spins without end, none traps).
"""
import numpy as np
import pytest

from kete_b200 import synthetic

pytestmark = pytest.mark.gpu

EPOCH = synthetic.EPOCH
TIMEOUT = 7

# the warp-synchronous cached node kernel (persistent grid with refill, objects in work
# order; and one object per group), the warp-pooled forms, and the plain thread form
FORMS = (dict(mode=2, variant=7, refill=1), dict(mode=2, variant=7, refill=0),
         dict(mode=2, variant=9, refill=1), dict(mode=2, variant=10, refill=1),
         dict(mode=1, variant=0, refill=0))


def _population(n=4000, seed=81):
    pos, vel, ng = synthetic.mixed(n, seed=seed)
    rng = np.random.default_rng(seed + 1)
    jd0 = np.full(n, EPOCH)
    jd1 = EPOCH + rng.uniform(-5 * 365.25, 5 * 365.25, n)
    return pos, vel, ng, jd0, jd1


def test_batched_mix_five_year_spans_vs_oracle(gpu, oracle_spk):
    from kete_b200 import tune

    pos, vel, ng, jd0, jd1 = _population()
    op, ov, ost, ons, _ = oracle_spk.propagate_n_body(pos, vel, jd0, jd1, ng=ng)
    assert (ost == 0).mean() > 0.99
    try:
        for cfg in FORMS:
            tune.set_config(**cfg)
            p, v, st, det = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1, nongrav=ng,
                                                        mode=cfg["mode"], with_details=True)
            close = det["min_dist"] < 0.01
            far = ~close
            # statuses: identical for every object that stays away from the planets
            assert np.array_equal(st[far], ost[far]), cfg
            ok = (st == 0) & (ost == 0)
            err = np.linalg.norm(p - op, axis=0)
            verr = np.linalg.norm(v - ov, axis=0)
            assert err[ok & far].max() < 1e-9, (cfg, err[ok & far].max())
            assert verr[ok & far].max() < 1e-11, (cfg, verr[ok & far].max())
            # nearly the same adaptive step sequence: over five years a rounding-level
            # difference in a step-size estimate shifts the final truncated step of some
            # objects by one step
            dsteps = np.abs(det["counters"][0][ok].astype(np.int64) - ons[ok])
            assert np.mean(dsteps == 0) > 0.8 and np.mean(dsteps <= 1) > 0.98, cfg
            near = ok & close
            print(f"{cfg}: far max {err[ok & far].max():.3e} AU over {int((ok & far).sum())} "
                  f"objects; {int(close.sum())} within 0.01 AU of a planet, max "
                  f"{(err[near].max() if near.any() else 0.0):.3e} AU, "
                  f"{int((err[near] <= 1e-9).sum())} of them within 1e-9 AU")
    finally:
        tune.set_config()


def test_pooled_forms_split_at_the_fast_window(gpu, oracle, spk_path, tmp_path):
    """The warp-pooled kernels (variants 9, 10) evaluate the ephemeris only from the fast
    plan's records, whose window is the coverage of every body's first segment.  With the
    ephemeris in two files (two segments per body, meeting at JD 2460000.5), the objects whose
    span crosses into the other file's coverage are ordered after the others and integrated by
    the form with the general evaluation in a second launch.  Objects start on both sides of
    the boundary, so that both launches have work whichever segment comes first; half the
    comets have a delayed non-gravitational model (dt != 0, a two-body back-propagation per
    evaluation, which the pooled kernel makes as its one out-of-line call).  Every object
    agrees with the oracle, which searches the segments for every evaluation."""
    from kete_b200 import tune

    a, b = str(tmp_path / "early.bsp"), str(tmp_path / "late.bsp")
    synthetic.write_synthetic_spk(a, jd_start=2459000.5, jd_end=2460000.5)
    synthetic.write_synthetic_spk(b, jd_start=2460000.5, jd_end=2461000.5)
    n = 400
    pos, vel, ng = synthetic.mixed(n, seed=83, nongrav_frac=0.1)
    comets = np.flatnonzero(ng[0] == 1.0)
    ng[9, comets[::2]] = 4.0  # a delayed model for every other comet
    assert len(comets) >= 20
    rng = np.random.default_rng(84)
    jd0 = np.where(np.arange(n) % 2 == 0, 2459700.5, 2460300.5)
    jd1 = jd0 + rng.uniform(-600.0, 600.0, n)
    crossing = (np.minimum(jd0, jd1) < 2460000.5) & (np.maximum(jd0, jd1) > 2460000.5)
    assert 0.1 < crossing.mean() < 0.9
    try:
        gpu.spice.kernel_reload([a, b])
        oracle.spk_reset()
        for f in (a, b):
            oracle.spk_load_bytes(open(f, "rb").read())
        op, ov, ost, _, _ = oracle.propagate_n_body(pos, vel, jd0, jd1, ng=ng)
        assert (ost == 0).all()
        for cfg in (dict(mode=2, variant=10, refill=1), dict(mode=2, variant=9, refill=0),
                    dict(mode=2, variant=7, refill=1)):
            tune.set_config(**cfg)
            p, v, st, det = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1, nongrav=ng, mode=2,
                                                        with_details=True)
            far = det["min_dist"] >= 0.01
            assert (st == 0).all(), cfg
            err = np.linalg.norm(p - op, axis=0)
            assert err[far].max() < 1e-9, (cfg, err[far].max())
            assert far.mean() > 0.9
    finally:  # restore the session ephemeris for the tests that follow
        tune.set_config()
        gpu.spice.kernel_reload([spk_path])
        oracle.spk_reset()
        oracle.spk_load_bytes(open(spk_path, "rb").read())


def test_step_limit_returns_timeout(gpu, oracle_spk):
    from kete_b200 import tune

    n = 300
    pos, vel = synthetic.main_belt(n, seed=91)
    jd0, jd1 = np.full(n, EPOCH), np.full(n, EPOCH + 365.25)
    try:
        tune.set_step_limit(4)
        for cfg in FORMS + (dict(mode=2, variant=0, refill=0), dict(mode=2, variant=4, refill=1)):
            tune.set_config(**cfg)
            p, v, st = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1, mode=cfg["mode"])
            assert (st == TIMEOUT).all(), (cfg, np.bincount(st))
            assert np.isnan(p).all() and np.isnan(v).all()
        # a zero-length span needs no step and is not affected
        p, v, st = gpu.propagate_n_body_arrays(pos, vel, jd0, jd0)
        assert (st == 0).all()
    finally:
        tune.set_step_limit(0)
        tune.set_config()
    op, _, ost, _, _ = oracle_spk.propagate_n_body(pos, vel, jd0, jd1)
    p, v, st = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1)
    assert (st == 0).all() and np.abs(p - op).max() < 1e-9


def test_close_approaches_reported_apart(gpu, oracle_spk):
    """Objects sent past the Earth within 0.01 AU are flagged by their closest planet distance
    (min_dist) and compared apart: every object that stays away agrees with the oracle to
    1e-9 AU; the close ones are counted, their statuses agree, and their errors are reported
    (a close approach amplifies rounding-level differences; both sides integrate the same
    dynamics)."""
    n = 400
    rng = np.random.default_rng(123)
    earth = np.stack([oracle_spk.spk_get_state(399, EPOCH + 30.0, 10, 2)[1]])[0]
    # start 30 days before the encounter on the Earth's track, offset by 0.001-0.03 AU, with
    # a relative velocity of ~0.003 AU/day: the slow straight-line approach passes near the
    # Earth and stays close for days, so the accepted steps sample the closest approach
    rel_v = rng.normal(0.0, 0.003, (3, n))
    miss = rng.uniform(0.001, 0.03, n) * rng.choice([-1.0, 1.0], n)
    p30 = earth[:3, None] + np.array([[1.0], [0.0], [0.0]]) * miss
    pos = p30 - 30.0 * (earth[3:, None] + rel_v)
    vel = earth[3:, None] + rel_v
    pos, vel = np.ascontiguousarray(pos), np.ascontiguousarray(vel)
    jd0, jd1 = np.full(n, EPOCH), np.full(n, EPOCH + 365.25)
    op, ov, ost, _, _ = oracle_spk.propagate_n_body(pos, vel, jd0, jd1)
    p, v, st, det = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1, with_details=True)
    close = det["min_dist"] < 0.01
    assert close.sum() >= 10 and (~close).sum() >= 10
    assert np.array_equal(st, ost)
    ok = (st == 0) & (ost == 0)
    err = np.linalg.norm(p - op, axis=0)
    assert err[ok & ~close].max() < 1e-9
    print(f"{int(close.sum())} of {n} within 0.01 AU of a planet: max |dpos| "
          f"{err[ok & close].max():.3e} AU, median {np.median(err[ok & close]):.3e} AU; "
          f"{int((err[ok & close] <= 1e-9).sum())} within 1e-9 AU")


def test_output_arrays_and_tuner_finalists(gpu):
    """``out=`` writes the results into the caller's arrays, on the host and on the device,
    bit-identical to a call that allocates them; the tuner's finalist stage re-times the
    closest configurations on the whole population and installs the fastest there."""
    import torch
    from kete_b200 import tune

    pos, vel, ng, jd0, jd1 = _population(n=3000, seed=91)
    jd1 = EPOCH + (jd1 - EPOCH) / 20.0  # spans of up to a quarter year keep the sweep short
    n = pos.shape[1]
    try:
        tune.set_config(mode=2, variant=10, refill=1)
        ref = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1, nongrav=ng, mode=2)
        out = (np.empty((3, n)), np.empty((3, n)), np.empty(n, dtype=np.int32))
        got = gpu.propagate_n_body_arrays(pos, vel, jd0, jd1, nongrav=ng, mode=2, out=out)
        for a, b, c in zip(ref, out, got):
            assert c is b
            assert np.array_equal(a, b)
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        dev = (T(pos), T(vel), T(jd0), T(jd1), T(ng))
        dout = (torch.empty((3, n), dtype=torch.float64, device="cuda"),
                torch.empty((3, n), dtype=torch.float64, device="cuda"),
                torch.empty((n,), dtype=torch.int32, device="cuda"))
        gpu.propagate_n_body_arrays(*dev[:4], nongrav=dev[4], mode=2, out=dout)
        torch.cuda.synchronize()
        for a, b in zip(ref, dout):
            assert np.array_equal(a, b.cpu().numpy())
        with pytest.raises(ValueError):  # wrong shape
            gpu.propagate_n_body_arrays(pos, vel, jd0, jd1, nongrav=ng, mode=2,
                                        out=(out[0][:, :10], out[1], out[2]))
        with pytest.raises(ValueError):  # host outputs for device inputs
            gpu.propagate_n_body_arrays(*dev[:4], nongrav=dev[4], mode=2, out=out)

        sub = slice(0, None, 4)
        best, times = tune.autotune(*(x[..., sub].contiguous() for x in dev[:4]),
                                    nongrav=dev[4][:, sub].contiguous(), full=dev,
                                    finalists=2, within=10.0)
        full = {k: v for k, v in times.items() if k.endswith("_full")}
        assert len(full) == 2
        label = f"mode{best['mode']}_v{best['variant']}_r{best['refill']}_full"
        assert times[label] == min(full.values())
        assert {k: tune.current()[k] for k in best} == best
    finally:
        tune.set_config()
