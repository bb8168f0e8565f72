"""The learned surrogate against the method without it (the engine's FP64
solve): on held-out gratings the trained network is far closer to the solve
than the training-mean predictor and answers a query much faster; the fallback
rules route out-of-range parameters, lossless stacks that break R + T = 1 and
audited rows to the solve, which then supplies their values."""
import time

import numpy as np
import pytest

import openrcwa_b200 as o
from openrcwa_b200 import surrogate as sg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def trained():
    eng = o.Engine(0)
    rng = np.random.default_rng(0)
    nh = 2
    P = sg.sample(60000, rng)
    Y = sg.solve(eng, P, nh, chunk=4096)
    sur = sg.Surrogate(eng, nh, hidden=256, layers=4, seed=1)
    loss = sur.fit(P, Y, epochs=30, batch=512, lr=1e-3, seed=3)
    yield eng, sur, P, Y, loss, rng
    sur.close()
    eng.close()


def test_network_beats_mean_and_is_faster(trained):
    eng, sur, P, Y, loss, rng = trained
    assert loss[-1] < 0.2 * loss[0]
    Pt = sg.sample(1000, rng)
    t0 = time.perf_counter()
    Yt = sg.solve(eng, Pt, sur.nh)
    t_solve = (time.perf_counter() - t0) / len(Pt)
    Yp = sur.predict(Pt)
    rms = float(np.sqrt(np.mean((Yp - Yt) ** 2)))
    rms_mean = float(np.sqrt(np.mean((Yt - Y.mean(axis=0)) ** 2)))
    assert rms < 0.5 * rms_mean, (rms, rms_mean)
    Pbig = sg.sample(65536, rng)
    sur.predict(Pbig[:1024])
    t0 = time.perf_counter()
    sur.predict(Pbig)
    t_net = (time.perf_counter() - t0) / len(Pbig)
    assert t_solve / t_net > 10, (t_solve, t_net)


def test_fallback_rules(trained):
    eng, sur, P, Y, loss, rng = trained
    Pq = sg.sample(60, rng)
    Pq[:20, 3] = 14.0      # eps_re above the training range
    Pq[20:40, 4] = 0.0     # lossless: the energy check applies
    r = sur.query(Pq, audit=0.5, seed=4)
    src, Yq = r["source"], r["Y"]
    assert np.all(src[:20] == sg.SOURCE_HULL)
    fell = src != sg.SOURCE_NET
    # fallbacks come from the mixed-precision solve, within 1e-4 of FP64
    Ys = sg.solve(eng, Pq[fell], sur.nh, chunk=4096, precision=o.RCWA_PREC_MIXED)
    assert np.max(np.abs(Yq[fell] - Ys)) < 1e-12
    assert np.max(np.abs(Yq[fell] - sg.solve(eng, Pq[fell], sur.nh))) < 1e-4
    net_lossless = (src == sg.SOURCE_NET) & (Pq[:, 4] == 0.0)
    assert np.all(np.abs(Yq[net_lossless, 50] + Yq[net_lossless, 51] - 1.0) <= 1e-3)
    assert np.any(src == sg.SOURCE_AUDIT) and len(r["audit_err"]) == int(np.sum(src == sg.SOURCE_AUDIT))


def test_hull_rule_flags_queries_far_from_the_training_data(trained):
    # a training set on a diagonal band of the box: every parameter spans its
    # full range, so the range check passes everywhere, but a query at the
    # opposite corner of the box is far from every training row
    eng, sur, P, Y, loss, rng = trained
    lo, hi = sg.RANGES[:, 0], sg.RANGES[:, 1]
    t = rng.random((4096, 1))
    Pb = lo + (hi - lo) * np.clip(t + 0.03 * rng.standard_normal((4096, len(lo))), 0.0, 1.0)
    Pb[:, 7] = lo[7] + (hi[7] - lo[7]) * t[:, 0]
    band = sg.Surrogate(eng, sur.nh, hidden=32, layers=2, seed=2)
    band.fit(Pb, sg.solve(eng, Pb, sur.nh, chunk=4096), epochs=1, batch=512, lr=1e-3, seed=5)
    on_band = lo + (hi - lo) * np.clip(rng.random((32, 1)) + np.zeros((32, len(lo))), 0.05, 0.95)
    off_band = lo + (hi - lo) * np.where(np.arange(len(lo)) % 2 == 0, 0.1, 0.9)[None, :].repeat(32, axis=0)
    r = band.query(np.vstack([on_band, off_band]), audit=0.0)
    assert np.all(r["source"][32:] == sg.SOURCE_HULL)
    assert np.mean(r["source"][:32] == sg.SOURCE_NET) > 0.9
    band.close()


def test_audited_error_bounds_the_unaudited_rows(trained):
    # the audit is a random sample of the network's answers: the largest of
    # about 400 audited errors bounds all but the top 2% of the unaudited ones
    # (it falls below that quantile with probability 0.98^400, about 3e-4)
    eng, sur, P, Y, loss, rng = trained
    Pq = sg.sample(8192, rng)
    r = sur.query(Pq, audit=0.05, seed=7)
    net = r["source"] == sg.SOURCE_NET
    err = np.max(np.abs(r["Y"][net] - sg.solve(eng, Pq[net], sur.nh, chunk=4096)), axis=1)
    assert len(r["audit_err"]) > 200
    assert np.quantile(err, 0.98) <= np.max(r["audit_err"])
