"""Learned initial guess for the relaxation: an MLP maps the 13 puncture
parameters to the coefficients of a POD basis of uu built from solutions the
relaxation itself generates; vv is guessed as eta * uu (the steady state of
uu_rhs = vv - eta uu).  The guess is used only when its residual L2 is below
the zero guess's (else the zero guess is the fallback), and the FP64
relaxation from either start decides the final error.

    python -m nrpyelliptic_b200.learned [--train 4096] [--test 256] [--modes 256] [--epochs 400] [--mixed-training]
    python -m nrpyelliptic_b200.learned --mlp-only [--epochs 5]   (network training throughput)

Pipeline (one GPU):
  1. training solves: `--train` configurations drawn from the seeded sweep
     distribution (sample_sweep) on the 128x128x16 grid, relaxed from the
     zero guess to log10 L2 <= -10 in batches (nrpyell_relax_batch, or with
     --mixed-training the batched FP32 correction form);
  2. POD by the method of snapshots on the host (float32 Gram matrix of the
     centred uu snapshots, float64 eigendecomposition), `--modes` modes;
  3. MLP 13 -> 4 x 512 (tanh) -> modes, trained with the library's BF16
     tensor-core kernels (nrpyell_mlp_train: Adam, minibatch 256) on
     standardised inputs and the coefficients divided by their overall
     standard deviation;
  4. held-out evaluation on `--test` configurations from another seed: RK4
     steps and wall time to log10 L2 <= -10 from the zero guess and from the
     learned guess (FP64, and FP32-then-FP64), the fallback rate, the guess's
     own error and the difference of the converged solutions.
"""
import argparse
import ctypes as C
import time

import numpy as np

from . import _lib
from .batch import relax_batch, relax_batch_mixed
from .problem import DeviceState, Problem, sample_sweep, with_grid

GRID = (128, 128, 16)
N_FEATURES = 13


def features(cfg):
    """(m0, m1, z0, z1, bScale, P0x, P0y, S0xyz, S1xyz) of a configuration."""
    pu = cfg.punctures
    return [pu.m0, pu.m1, pu.pos0[2], pu.pos1[2], cfg.bScale, pu.P0[0], pu.P0[1], *pu.S0, *pu.S1]


def configs(n, seed):
    return [with_grid(c, GRID) for c in sample_sweep(n, seed)]


def solve_snapshots(cfgs, lib, chunk=64, tol=-10.0, max_steps=40000, log=print, dist=None, mixed=False):
    """Relax every configuration from the zero guess in batches; returns the
    converged uu arrays (float32, ghost zones included) and step counts.
    mixed: the batched FP32 correction form (every step FP32, folded into the
    FP64 state every 256 steps, the FP64 norm as the stop test) instead of
    the FP64 batch; the snapshots then differ from the FP64 ones by ~1e-8 of
    max|uu|, far below what a POD basis resolves.
    With `dist` (replicas.Replicas, one process per GPU) the configurations
    are dealt round-robin over the ranks, each rank solves its share, and the
    snapshots are gathered on the host of every rank."""
    if dist is not None and dist.world > 1:
        from .replicas import shard
        mine = shard(list(range(len(cfgs))), dist.rank, dist.world)
        part = (solve_snapshots([cfgs[i] for i in mine], lib, chunk, tol, max_steps, log, mixed=mixed) if mine
                else (None, []))
        parts = dist.all_gather((mine, part[0], list(part[1])))
        ntot = next(p[1].shape[1] for p in parts if p[1] is not None)
        snaps = np.empty((len(cfgs), ntot), np.float32)
        steps = np.zeros(len(cfgs), np.int64)
        for idx, sn, st in parts:
            for k, i in enumerate(idx):
                snaps[i] = sn[k]
                steps[i] = st[k]
        return snaps, steps
    snaps, steps = None, []
    for c0 in range(0, len(cfgs), chunk):
        probs = [Problem(c, lib=lib, host_aux=False, device_tables=True) for c in cfgs[c0:c0 + chunk]]
        if mixed:
            rc, s32, s64, _, states = relax_batch_mixed(probs, tol=tol, switch=tol, fold_every=256,
                                                        max_steps=max_steps, lib=lib)
            st = s32 + s64
        else:
            rc, st, _, states = relax_batch(probs, tol=tol, max_steps=max_steps, lib=lib)
        if snaps is None:
            snaps = np.empty((len(cfgs), probs[0].Ntot), np.float32)
        for i, (p, s) in enumerate(zip(probs, states)):
            snaps[c0 + i] = s.download("y_n", p.Ntot).astype(np.float32)
            s.free()
        steps.extend(int(x) for x in st)
        del probs, states
        lib.nrpyell_release_tables()
        if (c0 // chunk) % 8 == 7 or c0 + chunk >= len(cfgs):
            log("  solved %d / %d (not converged in the last batch: %d)" % (min(c0 + chunk, len(cfgs)), len(cfgs), rc))
    return snaps, np.array(steps)


def pod(snaps, modes):
    """Mean, basis [modes x Ntot] (float32, orthonormal), coefficients
    [n x modes] and the captured fraction of the variance."""
    mean = snaps.mean(axis=0, dtype=np.float64).astype(np.float32)
    X = snaps - mean
    G = (X @ X.T).astype(np.float64)
    lam, V = np.linalg.eigh(G)
    order = np.argsort(lam)[::-1]
    lam, V = np.maximum(lam[order], 0.0), V[:, order]
    k = min(modes, int(np.sum(lam > lam[0] * 1e-14)))
    basis = ((V[:, :k] / np.sqrt(lam[:k])).T.astype(np.float32) @ X).astype(np.float32)
    coeffs = V[:, :k] * np.sqrt(lam[:k])
    return mean, basis, coeffs, float(lam[:k].sum() / lam.sum())


class Guess:
    """Trained surrogate: feature / coefficient standardisation, the MLP and
    the POD basis on the device."""

    def __init__(self, lib, mean, basis, coeffs, feats, width=512, depth=4, seed=1):
        self.lib = lib
        self.K, self.ntot = basis.shape
        self.fmu, self.fsd = feats.mean(0), feats.std(0) + 1e-12
        # one scale for all coefficients, so that the training loss is the
        # squared L2 error of the reconstructed uu (standardising each mode
        # would weight the barely-excited high modes like the leading ones)
        self.csd = float(coeffs.std()) + 1e-30
        self.mlp = lib.nrpyell_mlp_create(N_FEATURES, width, depth, self.K, 256, seed)
        _lib.check(lib)
        self.d_mean = self._upload(mean)
        self.d_basis = self._upload(basis)

    def _upload(self, a):
        a = np.ascontiguousarray(a, dtype=np.float32)
        p = self.lib.nrpyell_device_malloc(a.nbytes)
        self.lib.nrpyell_memcpy(p, a.ctypes.data, a.nbytes, 0)
        _lib.check(self.lib)
        return p

    def train(self, feats, coeffs, epochs, lr=1e-3, batch=256, seed=2):
        x = self._upload((feats - self.fmu) / self.fsd)
        t = self._upload(coeffs / self.csd)
        hist = np.zeros(epochs)
        batch = min(batch, len(feats))
        last = self.lib.nrpyell_mlp_train(self.mlp, x, t, len(feats), batch, epochs, lr, seed, hist.ctypes.data)
        _lib.check(self.lib)
        self.lib.nrpyell_device_free(x)
        self.lib.nrpyell_device_free(t)
        return last, hist

    def predict(self, feats):
        """POD coefficients [n x K] for feature rows."""
        x = self._upload((np.asarray(feats) - self.fmu) / self.fsd)
        n = len(feats)
        y = self.lib.nrpyell_device_malloc(4 * n * self.K)
        self.lib.nrpyell_mlp_predict(self.mlp, x, n, y)
        out = np.empty((n, self.K), np.float32)
        self.lib.nrpyell_memcpy(out.ctypes.data, y, out.nbytes, 1)
        _lib.check(self.lib)
        self.lib.nrpyell_device_free(x)
        self.lib.nrpyell_device_free(y)
        return out.astype(np.float64) * self.csd

    def write_guess(self, coeffs, eta, y_n_ptr):
        """y_n (device) = the POD reconstruction of one configuration."""
        c = self._upload(np.asarray(coeffs, np.float32))
        self.lib.nrpyell_pod_guess(self.d_mean, self.d_basis, self.K, self.ntot, c, eta, y_n_ptr)
        self.lib.nrpyell_device_free(c)
        _lib.check(self.lib)

    def free(self):
        self.lib.nrpyell_device_free(self.d_mean)
        self.lib.nrpyell_device_free(self.d_basis)
        self.lib.nrpyell_mlp_destroy(self.mlp)


def initial_log10_l2(lib, prob, ds):
    """log10 L2 of the residual of the state in ds (no step is taken)."""
    steps, fin = C.c_int(0), C.c_double(0)
    lib.nrpyell_relax(C.byref(ds.g), prob.dt, -1e300, 0, prob.cfg.R_L2, C.byref(steps), C.byref(fin), None)
    _lib.check(lib)
    return fin.value


def start_state(lib, prob, ds, guess, coeffs, r0=None):
    """Puts the learned guess for one configuration into ds's y_n and keeps it
    only if its residual L2 is below the zero guess's (r0, evaluated here
    when None); otherwise ds gets the zero guess (the fallback).  Returns
    (learned guess used, log10 L2 of the zero guess, of the learned guess)."""
    if r0 is None:
        ds.set_state(prob.zero_state())
        r0 = initial_log10_l2(lib, prob, ds)
    guess.write_guess(coeffs, prob.cfg.eta, C.c_void_p(ds.ptr["y_n"]))
    rl = initial_log10_l2(lib, prob, ds)
    use = bool(rl < r0)
    if not use:
        ds.set_state(prob.zero_state())
    return use, r0, rl


def timed_relax(lib, prob, ds, mixed, max_steps=40000):
    """(RK4 steps, seconds, final log10 L2) of one relaxation from ds's state."""
    fin = C.c_double(0)
    lib.nrpyell_synchronize()
    t0 = time.perf_counter()
    if mixed:
        n32, n64 = C.c_int(0), C.c_int(0)
        lib.nrpyell_relax_mixed(C.byref(ds.g), prob.dt, -10.0, -10.0, 256, max_steps, prob.cfg.R_L2,
                                C.byref(n32), C.byref(n64), C.byref(fin), None)
        steps = n32.value + n64.value
    else:
        st = C.c_int(0)
        lib.nrpyell_relax(C.byref(ds.g), prob.dt, -10.0, max_steps, prob.cfg.R_L2, C.byref(st), C.byref(fin), None)
        steps = st.value
    lib.nrpyell_synchronize()
    sec = time.perf_counter() - t0
    _lib.check(lib)
    return steps, sec, fin.value


KEYS = ["res0", "res_learned", "fallback", "steps_zero", "sec_zero", "fin_zero", "steps_learned", "sec_learned",
        "fin_learned", "steps_mixed", "sec_mixed", "fin_mixed", "err_learned", "err_mixed", "guess_rel_l2"]


def evaluate(lib, guess, cfgs, log=print):
    """Per held-out configuration: zero-guess FP64, learned FP64 and learned
    FP32-then-FP64 relaxations (the learned ones fall back to the zero guess
    where the learned guess's residual is not below the zero guess's)."""
    rows, zeros = [], []
    coeffs = guess.predict([features(c) for c in cfgs])
    for i, cfg in enumerate(cfgs):
        prob = Problem(cfg, lib=lib, host_aux=False, device_tables=True)
        ds = DeviceState(prob, lib=lib)
        r0 = initial_log10_l2(lib, prob, ds)
        s0, t0, f0 = timed_relax(lib, prob, ds, False)
        u_zero = ds.download("y_n", prob.Ntot)
        guess.write_guess(coeffs[i], cfg.eta, C.c_void_p(ds.ptr["y_n"]))
        u_guess = ds.download("y_n", prob.Ntot)
        use, _, rl = start_state(lib, prob, ds, guess, coeffs[i], r0)
        fallback = not use
        s1, t1, f1 = timed_relax(lib, prob, ds, False)
        u_learned = ds.download("y_n", prob.Ntot)
        if fallback:
            ds.set_state(prob.zero_state())
        else:
            guess.write_guess(coeffs[i], cfg.eta, C.c_void_p(ds.ptr["y_n"]))
        s2, t2, f2 = timed_relax(lib, prob, ds, True)
        u_mixed = ds.download("y_n", prob.Ntot)
        umax = np.max(np.abs(u_zero))
        zeros.append(u_zero.astype(np.float32))
        rows.append((r0, rl, fallback, s0, t0, f0, s1, t1, f1, s2, t2, f2,
                     np.max(np.abs(u_learned - u_zero)) / umax, np.max(np.abs(u_mixed - u_zero)) / umax,
                     np.linalg.norm(u_guess - u_zero) / np.linalg.norm(u_zero)))
        ds.free()
        del prob
        if (i + 1) % 32 == 0:
            lib.nrpyell_release_tables()
            log("  evaluated %d / %d" % (i + 1, len(cfgs)))
    a = np.array(rows, dtype=np.float64)
    out = {k: a[:, j] for j, k in enumerate(KEYS)}
    out["u_zero"] = zeros  # converged solutions from the zero guess
    return out


def compare_solvers(lib, guess, cfgs, log=print):
    """Wall time of the held-out configurations solved (a) one by one in FP64
    from the zero guess -- the plain form -- and from the learned guess with
    the fallback rule (b) one by one in FP64, (c) one by one with the FP32
    correction form of the mixed-precision driver, (d) all together in one
    batched FP64 relaxation, (e) all together with the batched correction
    form (every step FP32, folded every 256 steps).  Set-up (grids, tables,
    auxevol) is outside the timings; the learned guess's network evaluation,
    guess writing and fallback test are inside (b)-(e).  Returns a dict of
    solves/s, RK4 steps and the speed-up of each form over (a)."""
    from .batch import relax_batch, relax_batch_mixed
    probs = [Problem(c, lib=lib, host_aux=False, device_tables=True) for c in cfgs]
    states = [DeviceState(p, lib=lib) for p in probs]
    n = len(cfgs)
    out = {"configurations": n}

    def clock(fn):
        lib.nrpyell_synchronize()
        t0 = time.perf_counter()
        r = fn()
        lib.nrpyell_synchronize()
        return time.perf_counter() - t0, r

    # warm-up: tile tuning, and the graph capture of both drivers for every
    # configuration's buffers (graphs are cached per buffers)
    for p, ds in zip(probs, states):
        initial_log10_l2(lib, p, ds)
        timed_relax(lib, p, ds, False, max_steps=32)
        timed_relax(lib, p, ds, True, max_steps=600)
    relax_batch(probs, states, max_steps=32, lib=lib)
    relax_batch_mixed(probs, states, fold_every=256, max_steps=32, lib=lib)
    for p, ds in zip(probs, states):
        ds.set_state(p.zero_state())
    t, steps = clock(lambda: [timed_relax(lib, p, ds, False)[0] for p, ds in zip(probs, states)])
    out["fp64_zero_guess"] = {"solves_per_s": n / t, "steps_median": float(np.median(steps))}

    def learned_starts():
        coeffs = guess.predict([features(c) for c in cfgs])
        return [start_state(lib, p, ds, guess, coeffs[i])[0] for i, (p, ds) in enumerate(zip(probs, states))]

    def single(mixed):
        used = learned_starts()
        return used, [timed_relax(lib, p, ds, mixed)[0] for p, ds in zip(probs, states)]

    for key, mixed in (("fp64_learned", False), ("mixed_learned", True)):
        t, (used, steps) = clock(lambda: single(mixed))
        out[key] = {"solves_per_s": n / t, "steps_median": float(np.median(steps)), "fallbacks": n - int(sum(used))}

    def batched():
        used = learned_starts()
        rc, steps, _, _ = relax_batch(probs, states, lib=lib)
        return used, steps, rc
    t, (used, steps, rc) = clock(batched)
    out["batched_fp64_learned"] = {"solves_per_s": n / t, "steps_median": float(np.median(steps)),
                                   "fallbacks": n - int(sum(used)), "not_converged": int(rc)}

    def batched_mixed():
        used = learned_starts()
        rc, s32, s64, _, _ = relax_batch_mixed(probs, states, switch=-10.0, fold_every=256, max_steps=40000,
                                               lib=lib)
        return used, s32 + s64, rc
    t, (used, steps, rc) = clock(batched_mixed)
    out["batched_mixed_learned"] = {"solves_per_s": n / t, "steps_median": float(np.median(steps)),
                                    "fallbacks": n - int(sum(used)), "not_converged": int(rc)}
    base = out["fp64_zero_guess"]["solves_per_s"]
    for k in ("fp64_learned", "mixed_learned", "batched_fp64_learned", "batched_mixed_learned"):
        out[k]["speedup_vs_fp64_zero_guess"] = out[k]["solves_per_s"] / base
    for ds in states:
        ds.free()
    lib.nrpyell_release_tables()
    return out


def report(ev, print=print):
    fb = ev["fallback"].astype(bool)
    n = len(fb)
    print("held-out: %d configurations, fallback to the zero guess: %d (%.1f %%)" % (n, fb.sum(), 100.0 * fb.mean()))
    print("initial log10 L2: zero guess median %.2f, learned guess median %.2f"
          % (np.median(ev["res0"]), np.median(ev["res_learned"])))
    print("learned guess vs the converged uu: relative L2 error median %.2e, max %.2e"
          % (np.median(ev["guess_rel_l2"]), ev["guess_rel_l2"].max()))
    for name, s, sec, fin in (("zero guess, FP64", "steps_zero", "sec_zero", "fin_zero"),
                              ("learned guess, FP64", "steps_learned", "sec_learned", "fin_learned"),
                              ("learned guess, FP32 then FP64", "steps_mixed", "sec_mixed", "fin_mixed")):
        print("%-30s RK4 steps median %6d mean %8.1f | %.3f s total, %.2f solves/s | worst final log10 L2 %.2f"
              % (name, np.median(ev[s]), ev[s].mean(), ev[sec].sum(), n / ev[sec].sum(), ev[fin].max()))
    if (~fb).any():
        print("where the learned guess is used (%d): RK4 steps median %d vs %d from the zero guess"
              % ((~fb).sum(), np.median(ev["steps_learned"][~fb]), np.median(ev["steps_zero"][~fb])))
    print("steps saved: median %.1f %%; wall time saved: %.1f %% (FP64), %.1f %% (learned + FP32 then FP64)"
          % (100 * np.median(1 - ev["steps_learned"] / ev["steps_zero"]),
             100 * (1 - ev["sec_learned"].sum() / ev["sec_zero"].sum()),
             100 * (1 - ev["sec_mixed"].sum() / ev["sec_zero"].sum())))
    print("max |uu - uu from the zero guess| / max|uu|: learned FP64 %.2e, learned mixed %.2e"
          % (ev["err_learned"].max(), ev["err_mixed"].max()))


def mlp_throughput(lib, n=4096, epochs=5, width=512, depth=4, n_out=256, batch=256):
    """Training throughput of the network alone (the learned guess's shape,
    13 -> depth x width -> n_out, minibatch `batch`) on seeded synthetic
    data: seconds per epoch and the matrix-product TFLOP/s (forward and both
    backward products: 6 flops per weight per row)."""
    rng = np.random.default_rng(3)
    x = rng.normal(size=(n, N_FEATURES)).astype(np.float32)
    t = rng.normal(size=(n, n_out)).astype(np.float32)
    mlp = lib.nrpyell_mlp_create(N_FEATURES, width, depth, n_out, batch, 1)
    dx = lib.nrpyell_device_malloc(x.nbytes)
    dt = lib.nrpyell_device_malloc(t.nbytes)
    lib.nrpyell_memcpy(dx, x.ctypes.data, x.nbytes, 0)
    lib.nrpyell_memcpy(dt, t.ctypes.data, t.nbytes, 0)
    lib.nrpyell_mlp_train(mlp, dx, dt, n, batch, 1, 1e-3, 1, None)  # warm-up
    lib.nrpyell_synchronize()
    t0 = time.perf_counter()
    lib.nrpyell_mlp_train(mlp, dx, dt, n, batch, epochs, 1e-3, 1, None)
    lib.nrpyell_synchronize()
    sec = (time.perf_counter() - t0) / epochs
    _lib.check(lib)
    weights = N_FEATURES * width + (depth - 1) * width * width + width * n_out
    flops = 6.0 * weights * (n // batch) * batch
    lib.nrpyell_device_free(dx)
    lib.nrpyell_device_free(dt)
    lib.nrpyell_mlp_destroy(mlp)
    return sec, flops / sec / 1e12


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=4096)
    ap.add_argument("--test", type=int, default=256)
    ap.add_argument("--modes", type=int, default=256)
    ap.add_argument("--epochs", type=int, default=400)
    ap.add_argument("--seed", type=int, default=20261203)
    ap.add_argument("--test-seed", type=int, default=20261204)
    ap.add_argument("--mixed-training", action="store_true",
                    help="training solves with the batched FP32 correction form (nrpyell_relax_batch_mixed)")
    ap.add_argument("--dump", default=None, help="write the regression data (features, POD coefficients) to this .npz")
    ap.add_argument("--mlp-only", action="store_true",
                    help="time the network's training on synthetic data only (no solves)")
    args = ap.parse_args()
    lib = _lib.load()
    if args.mlp_only:
        sec, tflops = mlp_throughput(lib, epochs=args.epochs)
        print("MLP 13 -> 4 x 512 -> 256, minibatch 256, 4096 rows: %.2f ms per epoch, %.2f TFLOP/s in the matrix "
              "products" % (sec * 1e3, tflops))
        return
    T = {}
    t = time.perf_counter()
    train_cfgs = configs(args.train, args.seed)
    snaps, steps = solve_snapshots(train_cfgs, lib, mixed=args.mixed_training)
    T["training solves"] = time.perf_counter() - t
    print("training solves: %d, RK4 steps median %d" % (len(steps), int(np.median(steps))))
    t = time.perf_counter()
    mean, basis, coeffs, energy = pod(snaps, args.modes)
    T["POD"] = time.perf_counter() - t
    del snaps
    lam = (coeffs ** 2).sum(0)
    print("POD: %d modes, captured variance fraction %.10f" % (basis.shape[0], energy))
    feats = np.array([features(c) for c in train_cfgs])
    guess = Guess(lib, mean, basis, coeffs, feats)
    t = time.perf_counter()
    last, hist = guess.train(feats, coeffs, args.epochs)
    T["MLP training"] = time.perf_counter() - t
    print("MLP training: %d epochs, loss (scaled coefficients) %.3e -> %.3e" % (args.epochs, hist[0], last))
    test_cfgs = configs(args.test, args.test_seed)
    t = time.perf_counter()
    ev = evaluate(lib, guess, test_cfgs)
    T["evaluation"] = time.perf_counter() - t
    if args.dump:
        test_coeffs = np.array([basis @ (u - mean) for u in ev.pop("u_zero")])
        np.savez_compressed(args.dump, feats=feats, coeffs=coeffs, lam=lam, test_feats=np.array(
            [features(c) for c in test_cfgs]), test_coeffs=test_coeffs, pred=guess.predict(
            [features(c) for c in test_cfgs]))
    else:
        ev.pop("u_zero")
    print()
    report(ev)
    t = time.perf_counter()
    cmp = compare_solvers(lib, guess, test_cfgs)
    T["solver comparison"] = time.perf_counter() - t
    print("\nheld-out solves, one form each (set-up outside the timings):")
    for k in ("fp64_zero_guess", "fp64_learned", "mixed_learned", "batched_fp64_learned", "batched_mixed_learned"):
        v = cmp[k]
        print("  %-22s %6.2f solves/s  RK4 steps median %6d  speed-up vs FP64 zero guess %.3f  fallbacks %s"
              % (k, v["solves_per_s"], v["steps_median"], v.get("speedup_vs_fp64_zero_guess", 1.0),
                 v.get("fallbacks", "-")))
    print("phase times: " + ", ".join("%s %.1f s" % kv for kv in T.items()))
    guess.free()


if __name__ == "__main__":
    main()
