"""Learned taper proposal.

A network (`felis_b200.MLP`: 4 linear layers of width 256, GELU, BF16 tensor
cores) learns, from runs that the batched engine itself generates, how the
per-segment power of a FELIS run depends on the undulator taper and on six beam
parameters.  It then ranks many candidate tapers for a given beam; the best
ones are re-run by the plain FP64 method, which judges the network's error and
takes over as a plain scan where that error exceeds 5 %.

Runs (the ensemble of the workload table's surrogate case): time-dependent
FELIS runs of 256 slices with 2048 particles each (512 beamlets x 4, shot
noise), grid key nx = 65, a 1 GeV class flat-top beam and a long Gaussian
seed; each slice spans 4 resonant wavelengths and each step 4 undulator
periods (slices_in_bucket = lambdaUs_in_iteration = 4), so the 640-slice
slippage of the 16.6 m undulator (32 segments of 20 periods, lambda_u 2.6 cm,
no gaps, 160 iterations) stays inside the 1024-wavelength bunch.  Taper: per
segment K_i = K0 (1 - a max(0, z_i - z0)^2) + N(0, 1e-4), z_i the segment's
start, a in [0, 2e-4], z0 in [5, 30] m.  Beam parameters: peak current,
relative energy spread, normalised emittance, matched beta, beam energy (the
undulator stays resonant at the segment-0 K), seed power.

Features (38): the 32 K_i / K0 - 1 and the 6 beam parameters (seed power as
log10).  Targets (33): log10 of the field energy at the end of each segment
(the per-iteration power sums of updateTotalEnergy.cpp:25-36, unscaled) and
the rms spectral bandwidth of the final field over the slices (from its
first-lag moments, felis_b200.analysis.lag_moments, in units of the slice
frequency).
"""
from __future__ import annotations

import os
import tempfile
import time

import numpy as np

SEGMENTS = 32
PERIODS = 20
BUCKET = 4          # wavelengths per slice = undulator periods per step
SLICES = 256
BEAMLETS = 512      # x 4 particles: 2048 per slice
LAMBDA_U_CM = 2.6
SEG_LEN = PERIODS * LAMBDA_U_CM / 100.0
K0 = 2.6
STEPS = SEGMENTS * PERIODS // BUCKET
SEG_STEPS = PERIODS // BUCKET
N_FEATURES = SEGMENTS + 6
N_TARGETS = SEGMENTS + 1

BEAM_RANGES = {
    "current": (2000.0, 4000.0),       # A
    "spread": (0.5e-4, 2.0e-4),        # relative rms energy spread
    "emit_um": (0.3, 0.6),             # normalised emittance
    "beta": (10.0, 30.0),              # m
    "energy_mev": (950.0, 1050.0),
    "log_seed_w": (4.0, 6.0),          # log10 seed power [W]
}
BEAM_KEYS = list(BEAM_RANGES)


def random_beam(rng) -> dict:
    return {k: float(rng.uniform(*BEAM_RANGES[k])) for k in BEAM_KEYS}


def random_taper(rng) -> np.ndarray:
    """K of the 32 segments for a in [0, 2e-4], z0 in [5, 30] m, jitter 1e-4."""
    a = rng.uniform(0.0, 2e-4)
    z0 = rng.uniform(5.0, 30.0)
    z = np.arange(SEGMENTS) * SEG_LEN
    return K0 * (1.0 - a * np.maximum(0.0, z - z0) ** 2) + rng.normal(0.0, 1e-4, SEGMENTS)


def random_tapers(rng, n: int) -> np.ndarray:
    """n tapers at once, [n, 32] (same distribution as random_taper)."""
    a = rng.uniform(0.0, 2e-4, (n, 1))
    z0 = rng.uniform(5.0, 30.0, (n, 1))
    z = np.arange(SEGMENTS)[None, :] * SEG_LEN
    return K0 * (1.0 - a * np.maximum(0.0, z - z0) ** 2) + rng.normal(0.0, 1e-4, (n, SEGMENTS))


def features(beam: dict, k: np.ndarray) -> np.ndarray:
    return np.concatenate([np.asarray(k) / K0 - 1.0, [beam[key] for key in BEAM_KEYS]]).astype(np.float32)


def _input(beam: dict, k: np.ndarray, path: str) -> str:
    from felis_b200 import workloads

    return workloads.write_input(
        path, kind="sase", slices=SLICES, bucket=BUCKET, beamlets=BEAMLETS, per_beamlet=4, nx=65,
        total_length=(STEPS + 0.5) * BUCKET * LAMBDA_U_CM / 100.0, energy_mev=beam["energy_mev"],
        spread_pct=beam["spread"] * 100.0, emit_um=beam["emit_um"], beta=beam["beta"], current=beam["current"],
        K0=K0, lambda_u_cm=LAMBDA_U_CM, units=SEGMENTS, unit_len=SEG_LEN, und_len=SEG_LEN,
        seed_power=10.0 ** beam["log_seed_w"], in_air=False, k_list=k)


def _targets(energy: np.ndarray, moments) -> np.ndarray:
    """energy[it, 2] (Ux, Uy sums) and the final field's first-lag moments ->
    the 33 targets."""
    from felis_b200 import analysis

    p = energy[:, 0] + energy[:, 1]
    seg = p[np.arange(1, SEGMENTS + 1) * SEG_STEPS]
    return np.concatenate([np.log10(np.maximum(seg, 1e-300)), [analysis.lag_moments(moments)[1]]])


def _moments(ux: np.ndarray, uy: np.ndarray) -> tuple[float, float, float]:
    """First-lag moments of downloaded fields (physical slices [S, ny, nx])."""
    r0 = float(np.sum(np.abs(ux) ** 2) + np.sum(np.abs(uy) ** 2))
    r1 = complex(np.sum(np.conj(ux[:-1]) * ux[1:]) + np.sum(np.conj(uy[:-1]) * uy[1:]))
    return r0, r1.real, r1.imag


def _prepare(cases: list, d: str, first: int):
    """Configs and seed fields of a chunk of cases, parsed on host threads."""
    from concurrent.futures import ThreadPoolExecutor

    import felis_b200 as fb

    def one(i):
        b, k = cases[i]
        c = fb.Config(_input(b, k, os.path.join(d, f"c{first + i}.inp")))
        return c, c.load_seed(0)

    with ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as ex:
        return list(ex.map(one, range(len(cases))))


def simulate(cases: list, chunk: int = 512, workdir: str | None = None, seed0: int = 1) -> np.ndarray:
    """Full simulations of (beam, taper) cases on the batched mixed-precision
    engine, `chunk` instances per ensemble (beams from the device loader, shot
    noise seeded seed0 + case index); returns targets [n, 33]."""
    import felis_b200 as fb

    d = workdir or tempfile.mkdtemp(prefix="felis_taper_")
    out = np.zeros((len(cases), N_TARGETS))
    for c0 in range(0, len(cases), chunk):
        part = cases[c0:c0 + chunk]
        prep = _prepare(part, d, c0)
        ens = fb.Batch([c.params for c, _ in prep])
        for i, (c, (ux, uy)) in enumerate(prep):
            beam = c.load_beam_device(0, seed=seed0 + c0 + i)
            ens.upload_particles(i, beam["x"], beam["y"], beam["px"], beam["py"], beam["theta"], beam["gamma"],
                                 beam["offsets"], beam["weights"])
            del beam
            ens.upload_field(i, 0, 0, ux)
            ens.upload_field(i, 0, 1, uy)
        ens.run(0, STEPS)
        mom = ens.spectral_moments(0)
        for i in range(len(part)):
            e, _, _ = ens.diagnostics(i, 0, STEPS + 1)
            out[c0 + i] = _targets(e, mom[i])
        ens.close()
        for c, _ in prep:
            c.close()
    return out


def simulate_plain(beam: dict, k: np.ndarray, workdir: str | None = None, seed: int = 1) -> np.ndarray:
    """The plain FP64 method (felis_create / felis_run) on one case."""
    import felis_b200 as fb

    d = workdir or tempfile.mkdtemp(prefix="felis_taper_")
    c = fb.Config(_input(beam, k, os.path.join(d, "plain.inp")))
    h = fb.Handle(c.params)
    b = c.load_beam_device(0, seed=seed)
    ux, uy = c.load_seed(0)
    h.upload_particles(0, b["x"], b["y"], b["px"], b["py"], b["theta"], b["gamma"], b["offsets"], b["weights"])
    del b
    h.upload_field(0, 0, ux)
    h.upload_field(0, 1, uy)
    h.run(0, STEPS)
    e, _, _ = h.diagnostics(0, STEPS + 1)
    mom = _moments(h.download_field(0, 0)[1:-1], h.download_field(0, 1)[1:-1])
    h.close()
    c.close()
    return _targets(e, mom)


class Surrogate:
    """The network with its input / output normalisation."""

    def __init__(self, width: int = 256, seed: int = 1):
        import felis_b200 as fb

        self.net = fb.MLP(N_FEATURES, width, N_TARGETS, seed=seed)
        self.xm = self.xs = self.ym = self.ys = None

    # epochs and learning-rate factors of the default schedule: the decay
    # matters most at the top of a ranking, where the proposals are chosen
    SCHEDULE = ((300, 1.0), (200, 0.3), (200, 0.1))

    def fit(self, X: np.ndarray, Y: np.ndarray, schedule=SCHEDULE, batch: int = 512, lr: float = 1e-3,
            weight_decay: float = 1e-4, seed: int = 1) -> np.ndarray:
        """AdamW on the normalised data, in stages of (epochs, lr factor);
        returns the mean loss of every epoch."""
        self.xm, self.xs = X.mean(0), X.std(0) + 1e-12
        self.ym, self.ys = Y.mean(0), Y.std(0) + 1e-12
        self.net.set_data((X - self.xm) / self.xs, (Y - self.ym) / self.ys)
        hist = [self.net.train(ep, batch=batch, lr=lr * f, weight_decay=weight_decay, seed=seed + i)
                for i, (ep, f) in enumerate(schedule)]
        return np.concatenate(hist)

    def predict(self, X: np.ndarray) -> np.ndarray:
        y = self.net.forward((np.asarray(X) - self.xm) / self.xs)
        return y * self.ys + self.ym

    def close(self):
        self.net.close()


def dataset(n: int, seed: int = 1, chunk: int = 512) -> tuple[np.ndarray, np.ndarray, list]:
    rng = np.random.default_rng(seed)
    cases = [(random_beam(rng), random_taper(rng)) for _ in range(n)]
    X = np.stack([features(b, k) for b, k in cases])
    Y = simulate(cases, chunk=chunk, seed0=seed * 1_000_000 + 1)
    return X, Y, cases


def propose(model: Surrogate, beam: dict, n_candidates: int, top: int, seed: int = 7):
    """Rank n_candidates random tapers for `beam` by predicted final power;
    returns the `top` tapers and their predicted targets."""
    rng = np.random.default_rng(seed)
    ks = random_tapers(rng, n_candidates)
    X = np.concatenate([ks / K0 - 1.0, np.tile([beam[k] for k in BEAM_KEYS], (n_candidates, 1))], axis=1)
    pred = model.predict(X.astype(np.float32))
    order = np.argsort(-pred[:, SEGMENTS - 1])[:top]
    return ks[order], pred[order]


def search(model: Surrogate, beam: dict, n_candidates: int = 1_000_000, top: int = 64, tol: float = 0.05,
           fallback_runs: int = 64, seed: int = 7, verify: int = 8, seeds: int = 8) -> dict:
    """Surrogate-guided taper search for one beam.  The runs start from shot
    noise, so one run of a taper is one draw of its final power; the network,
    trained on single draws, predicts their mean.  The plain FP64 method
    therefore verifies the `verify` best of the network's `top` proposals
    with `seeds` noise realisations each (verify x seeds runs) and judges the
    network by its error against the verified mean; where that error exceeds
    `tol`, a plain random scan of `fallback_runs` tapers (one FP64 run each)
    takes over.  Returns the best verified taper and the bookkeeping."""
    t0 = time.perf_counter()
    ks, pred = propose(model, beam, n_candidates, top, seed)
    t_rank = time.perf_counter() - t0
    ks, pred = ks[:verify], pred[:verify]
    draws = np.array([[10.0 ** simulate_plain(beam, k, seed=1 + j)[SEGMENTS - 1] for j in range(seeds)] for k in ks])
    p_true = draws.mean(axis=1)
    p_pred = 10.0 ** pred[:, SEGMENTS - 1]
    err = np.abs(p_pred - p_true) / p_true
    best = int(np.argmax(p_true))
    spread = draws.std(axis=1, ddof=1) / p_true if seeds > 1 else np.zeros(len(ks))
    res = {"best_power": float(p_true[best]), "best_taper": ks[best], "runs": verify * seeds, "rank_seconds": t_rank,
           "surrogate_error_max": float(err.max()), "surrogate_error_best": float(err[best]),
           "shot_noise_rel_std": float(spread[best]), "fallback": False}
    if err[best] > tol:
        rng = np.random.default_rng(seed + 1)
        scan = list(random_tapers(rng, fallback_runs))
        ps = np.array([10.0 ** simulate_plain(beam, k)[SEGMENTS - 1] for k in scan])
        res["fallback"] = True
        res["runs"] += fallback_runs
        if ps.max() > res["best_power"]:
            res["best_power"] = float(ps.max())
            res["best_taper"] = scan[int(np.argmax(ps))]
    return res


def compare_with_scan(model: Surrogate, beam: dict, n_candidates: int, top: int, scan_runs: int,
                      seed: int = 7, noise_runs: int = 0) -> dict:
    """What the network gains over the method without it, for one beam, in
    full simulations of one simulator (the batched engine): the best final
    power of the network's `top` proposals against the running best of a
    plain random scan of `scan_runs` tapers, and how many scan runs it takes
    to reach the network's best (None: not within the scan).  With
    noise_runs > 1, the best taper of each side is re-run with that many
    noise realisations: their mean final power (the quantity the network
    predicts) and relative spread."""
    ks, pred = propose(model, beam, n_candidates, top, seed)
    rng = np.random.default_rng(seed + 2)
    scan = random_tapers(rng, scan_runs)
    Y = simulate([(beam, k) for k in list(ks) + list(scan)])
    p_sur = 10.0 ** Y[:top, SEGMENTS - 1]
    p_scan = 10.0 ** Y[top:, SEGMENTS - 1]
    running = np.maximum.accumulate(p_scan)
    best = float(p_sur.max())
    reach = np.flatnonzero(running >= best)
    ib = int(np.argmax(p_sur))
    pred_best = 10.0 ** pred[ib, SEGMENTS - 1]
    out = {"surrogate_best": best, "surrogate_runs": top, "scan_best": float(p_scan.max()),
           "scan_best_at_equal_runs": float(running[min(top, scan_runs) - 1]),
           "scan_runs_to_reach": int(reach[0]) + 1 if reach.size else None, "scan_runs": scan_runs,
           "surrogate_error_at_best": float(abs(pred_best - best) / best)}
    if noise_runs > 1:
        # the shot-noise spread of the network's best taper and of the scan's,
        # and the network's error against the mean over noise realisations
        for name, k in (("surrogate", ks[ib]), ("scan", scan[int(np.argmax(p_scan))])):
            Yn = simulate([(beam, k)] * noise_runs, seed0=7_000_001)
            pn = 10.0 ** Yn[:, SEGMENTS - 1]
            out[f"{name}_best_mean_over_noise"] = float(pn.mean())
            out[f"{name}_best_noise_rel_std"] = float(pn.std(ddof=1) / pn.mean())
            out[f"{name}_best_bandwidth_mean"] = float(Yn[:, SEGMENTS].mean())
        mean = out["surrogate_best_mean_over_noise"]
        out["surrogate_error_vs_noise_mean"] = float(abs(pred_best - mean) / mean)
    return out


def main():
    """The taper study: training runs, training, held-out error, and for a few
    unseen beams the network's proposals against a random scan and the plain
    FP64 verification.  Prints one JSON document."""
    import argparse
    import json

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--runs", type=int, default=20000, help="training runs of the batched engine")
    ap.add_argument("--data", default=None, help="npz cache of the training set (X, Y)")
    ap.add_argument("--candidates", type=int, default=1_000_000)
    ap.add_argument("--top", type=int, default=64)
    ap.add_argument("--scan", type=int, default=1280, help="random-scan runs per beam")
    ap.add_argument("--beams", type=int, default=4)
    ap.add_argument("--noise-runs", type=int, default=32, help="noise realisations of each side's best taper")
    args = ap.parse_args()
    out = {}
    t0 = time.perf_counter()
    if args.data and os.path.exists(args.data):
        d = np.load(args.data)
        X, Y = d["X"], d["Y"]
        out["data"] = f"{len(X)} runs from {args.data}"
    else:
        X, Y, _ = dataset(args.runs, seed=1)
        out["data"] = f"{len(X)} runs generated in {time.perf_counter() - t0:.1f} s"
        if args.data:
            np.savez_compressed(args.data, X=X, Y=Y)
    t1 = time.perf_counter()
    model = Surrogate(seed=1)
    hist = model.fit(X, Y)
    out["train"] = {"seconds": time.perf_counter() - t1, "epochs": len(hist), "loss_first": float(hist[0]),
                    "loss_last": float(hist[-1])}
    Xv, Yv, _ = dataset(512, seed=2)
    Pv = model.predict(Xv)
    e = np.abs(10.0 ** Pv[:, SEGMENTS - 1] - 10.0 ** Yv[:, SEGMENTS - 1]) / 10.0 ** Yv[:, SEGMENTS - 1]
    out["held_out_final_power_error"] = {"median": float(np.median(e)), "p90": float(np.percentile(e, 90))}
    rng = np.random.default_rng(1234)
    out["beams"] = []
    for _ in range(args.beams):
        beam = random_beam(rng)
        r = compare_with_scan(model, beam, args.candidates, args.top, args.scan, noise_runs=args.noise_runs)
        s = search(model, beam, args.candidates, args.top)
        r.update({"beam": beam, "plain_best_power": s["best_power"], "plain_runs": s["runs"],
                  "plain_fallback": s["fallback"], "plain_error_at_best": s["surrogate_error_best"],
                  "plain_error_max": s["surrogate_error_max"], "plain_shot_noise_rel_std": s["shot_noise_rel_std"],
                  "rank_seconds": s["rank_seconds"]})
        out["beams"].append(r)
    model.close()
    print(json.dumps(out, indent=1), flush=True)


if __name__ == "__main__":
    main()
