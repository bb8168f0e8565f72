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
    Ys = sg.solve(eng, Pq[fell], sur.nh)
    assert np.max(np.abs(Yq[fell] - Ys)) < 1e-12
    net_lossless = (src == sg.SOURCE_NET) & (Pq[:, 4] == 0.0)
    assert np.all(np.abs(Yq[net_lossless, 50] + Yq[net_lossless, 51] - 1.0) <= 1e-3)
    assert np.any(src == sg.SOURCE_AUDIT) and len(r["audit_err"]) == int(np.sum(src == sg.SOURCE_AUDIT))
