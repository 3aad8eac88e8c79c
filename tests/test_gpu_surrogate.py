"""Learned taper proposal end to end on the GPU, at a reduced size.

The network is trained on runs of the batched engine, ranks candidate tapers
for a beam it has not seen, and its proposals are compared, in full
simulations, with a plain random scan of the same number of runs: the test
shows what the trained network gains over the method without it.  The plain
FP64 method re-runs the best proposals over several shot-noise realisations
and judges the network's error against their mean.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TRAIN_RUNS = 2048
TOP = 16


@pytest.fixture(scope="module")
def trained():
    from felis_b200 import surrogate as sg

    X, Y, _ = sg.dataset(TRAIN_RUNS, seed=21)
    model = sg.Surrogate(seed=2)
    hist = model.fit(X, Y, schedule=((100, 1.0), (50, 0.3)), batch=256, lr=1e-3)
    yield sg, model, hist
    model.close()


def test_training_converges(trained):
    sg, model, hist = trained
    assert hist[-1] < 0.2 * hist[0], hist[[0, -1]]


def test_network_beats_random_scan(trained):
    sg, model, _ = trained
    rng = np.random.default_rng(99)
    wins = 0
    for _ in range(2):
        beam = sg.random_beam(rng)
        r = sg.compare_with_scan(model, beam, n_candidates=20000, top=TOP, scan_runs=TOP)
        wins += r["surrogate_best"] >= r["scan_best"]
    assert wins == 2


def test_plain_verification_and_fallback(trained):
    sg, model, _ = trained
    beam = sg.random_beam(np.random.default_rng(7))
    r = sg.search(model, beam, n_candidates=20000, top=4, tol=0.05, fallback_runs=4, verify=2, seeds=2)
    assert r["best_power"] > 0 and r["shot_noise_rel_std"] >= 0
    # the fallback scan runs exactly when the error against the verified mean exceeds 5 %
    assert r["fallback"] == (r["surrogate_error_best"] > 0.05)
    assert r["runs"] == 2 * 2 + (4 if r["fallback"] else 0)
