"""Trains the flux-correction network on the GPU and evaluates it on held-out seeds.

  python vexelray-sim-fluid_b200/train_learned.py --out DIR [--fine 2048] [--seeds 128] [--pairs 20]
         [--spacing 100 | --sample-every 10] [--interval-steps 16] [--steps-per-pair 3] [--ring 256]
         [--eval-seeds 8]

The learned configuration's data (512 runs, pairs every 10 fine steps to 2000) is
  --seeds 512 --pairs 200 --sample-every 10

Fine runs at --fine^2 (the shallow-water configuration's bump distribution halved in sigma and centres) give the
samples; the network (coarse grid --fine/2) is trained by the library's own forward and backward kernels with Adam.
Writes DIR/learned_<fine>_k<interval>.npy (the fp32 parameters) and .json (the settings, the loss curve's
summary and the held-out evaluation against the plain coarse solver).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent


def package():
    if "vexfluid" in sys.modules:
        return sys.modules["vexfluid"]
    spec = importlib.util.spec_from_file_location("vexfluid", HERE / "__init__.py", submodule_search_locations=[str(HERE)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["vexfluid"] = mod
    spec.loader.exec_module(mod)
    return mod


def initial_params(vf, seed: int = 0) -> np.ndarray:
    """He-normal convolution weights, the last layer's scaled by 0.01 (the network starts near no correction), zero
    biases; the parameter order of vf_cnn_params."""
    rng = np.random.default_rng(seed)
    sizes = [("w1", (32, 25, 3)), ("b1", (32,)), ("w2", (32, 25, 32)), ("b2", (32,)), ("w3", (6, 25, 32)), ("b3", (6,))]
    parts = []
    for name, shape in sizes:
        if name.startswith("w"):
            w = rng.normal(0, np.sqrt(2.0 / (shape[1] * shape[2])), shape)
            parts.append((w * (0.01 if name == "w3" else 1.0)).ravel())
        else:
            parts.append(np.zeros(int(np.prod(shape))))
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == vf.FluxNet.count()
    return p


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--fine", type=int, default=2048)
    ap.add_argument("--seeds", type=int, default=128)
    ap.add_argument("--pairs", type=int, default=20)
    ap.add_argument("--spacing", type=int, default=100)
    ap.add_argument("--interval-steps", type=int, default=16)
    ap.add_argument("--sample-every", type=int, default=None,
                    help="sample every N fine steps of one run, each target from a copy of the run's state")
    ap.add_argument("--steps-per-pair", type=float, default=3)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--ring", type=int, default=256)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--lr-end", type=float, default=2e-4)
    ap.add_argument("--s-flux", type=float, default=1e-3)
    ap.add_argument("--s-res", type=float, default=1e-3)
    ap.add_argument("--eval-seeds", type=int, default=8)
    ap.add_argument("--eval-steps", type=int, default=2000)
    args = ap.parse_args(argv)
    vf = package()
    from vexfluid import learned as L

    out = pathlib.Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    n = args.fine
    interval = args.interval_steps * L.coarse_step_ticks(n)
    net = vf.FluxNet(n // 2, n // 2, batch=args.batch, samples=args.ring, s_flux=args.s_flux, s_res=args.s_res)
    net.params(initial_params(vf))
    train_seeds = list(range(1000, 1000 + args.seeds))   # held-out seeds are 1 .. eval-seeds
    r = L.generate_and_train(net, n, train_seeds, pairs=args.pairs, spacing=args.spacing, interval=interval,
                             batch=args.batch, lr=args.lr, lr_end=args.lr_end, steps_per_pair=args.steps_per_pair,
                             sample_every=args.sample_every, log=lambda s: print(s, flush=True))
    params = net.params()
    stem = f"learned_{n}_k{args.interval_steps}"
    np.save(out / f"{stem}.npy", params)
    evals = []
    for seed in range(1, 1 + args.eval_seeds):
        plain = L.evaluate(None, n, seed, args.eval_steps, interval)
        learned = L.evaluate(net, n, seed, args.eval_steps, interval)
        evals.append({"seed": seed, "plain": plain, "learned": learned})
        print(f"seed {seed}: h RMS error plain {plain['h_rms_error']:.3e} learned {learned['h_rms_error']:.3e} "
              f"speedup {learned['speedup']:.2f}", flush=True)
    losses = r["losses"]
    k = max(1, len(losses) // 20)
    report = {
        "fine": n, "coarse": n // 2, "interval_ticks": interval, "interval_coarse_steps": args.interval_steps,
        "s_flux": args.s_flux, "s_res": args.s_res, "train_seeds": [train_seeds[0], train_seeds[-1]],
        "pairs_per_seed": args.pairs, "spacing_fine_steps": args.spacing, "sample_every_fine_steps": args.sample_every,
        "steps_per_pair": args.steps_per_pair, "ring": args.ring, "adam_steps": len(losses),
        "batch": args.batch, "lr": [args.lr, args.lr_end], "train_seconds": r["seconds"],
        "loss_curve": [float(np.mean(losses[i:i + k])) for i in range(0, len(losses), k)],
        "eval": evals,
        "eval_mean": {"plain_h_rms": float(np.mean([e["plain"]["h_rms_error"] for e in evals])),
                      "learned_h_rms": float(np.mean([e["learned"]["h_rms_error"] for e in evals])),
                      "learned_speedup": float(np.mean([e["learned"]["speedup"] for e in evals]))},
        "command": " ".join(["python", "vexelray-sim-fluid_b200/train_learned.py"] + (argv or sys.argv[1:])),
    }
    (out / f"{stem}.json").write_text(json.dumps(report, indent=1, default=float))
    print(json.dumps(report["eval_mean"]), flush=True)
    net.close()


if __name__ == "__main__":
    main()
