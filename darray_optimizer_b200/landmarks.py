"""Leverage-score model for learned Nystrom landmarks: training data, training, the committed model, and the
learned-versus-uniform comparison.

Training data (all on the GPU, through the library's own kernels):
  * seeded instances of one workload family at n = 16384: the C5 mixture (datagen.mixture, d = 64; the default
    model, landmark_model.npz) or the C2 uniform-hyperplane points (datagen.uniform_hyperplane, d = 128;
    landmark_model_c2.npz);
  * inputs: [x, ||x||, distance to the 8th nearest neighbour] (db200_knn_distance over all points,
    db200_leverage_features);
  * targets: log ridge leverage scores of the instance's kernel matrix, centred per instance.  The scores come
    from the FP64 method: the FP64 low-rank factor Z (db200_lowrank with precision FP64) and
    db200_ridge_leverage(Z, lambda), with lambda set by bisection so that the effective dimension
    sum_k s_k^2 / (s_k^2 + lambda) over Z's singular values equals n / 64.
Training: the MLP of db200_mlp (3 hidden ReLU layers of 256, bf16 weights and activations) by Adam on minibatches
(db200_mlp_adam_step).  The model file holds the fp32 parameters, the input standardisation and the settings.

    python -m darray_optimizer_b200.landmarks train [--config c5|c2] [--out <file.npz>] [--instances 200]
    python -m darray_optimizer_b200.landmarks evaluate [--config c5|c2] [--model <file.npz>]
"""
from __future__ import annotations

import argparse
import json
import math
import time
from pathlib import Path

import numpy as np

from . import datagen
from ._lib import Context, Mlp

PKG = Path(__file__).resolve().parent
MODEL_PATH = PKG / "landmark_model.npz"
WIDTH, HIDDEN, KNN_K = 256, 3, 8
TRAIN_N, TRAIN_D, TRAIN_L = 16384, 64, 528
DEFF_FRACTION = 1.0 / 64
# workload families a model is trained on: generator of one seeded training instance, feature count, model file
CONFIGS = {
    "c5": (lambda seed: datagen.mixture(n=TRAIN_N, d=64, seed=seed), 64, MODEL_PATH),
    "c2": (lambda seed: datagen.uniform_hyperplane(n=TRAIN_N, d=128, seed=seed), 128, PKG / "landmark_model_c2.npz"),
}


def _ptr(t):
    return t.data_ptr()


def lambda_for_deff(sigma2: np.ndarray, deff: float) -> float:
    """lambda with sum sigma2 / (sigma2 + lambda) = deff (bisection on log lambda)."""
    s = np.maximum(np.asarray(sigma2, np.float64), 0.0)
    deff = min(deff, float(np.sum(s > 0)) - 1e-9)
    lo, hi = 1e-12 * max(s.max(), 1e-300), 1e12 * max(s.max(), 1e-300)
    for _ in range(200):
        mid = math.sqrt(lo * hi)
        if np.sum(s / (s + mid)) > deff:
            lo = mid
        else:
            hi = mid
    return math.sqrt(lo * hi)


def instance_inputs(ctx: Context, X, n: int, d: int, s_knn: int | None = None, seed: int = 0):
    """Device tensor F (n x (d + 2)) of model inputs for device points X (n x d)."""
    import torch
    s = n if s_knn is None else min(s_knn, n)
    if s >= n:
        ref = torch.arange(n, dtype=torch.int32, device="cuda")
    else:
        g = np.random.default_rng(seed)
        ref = torch.from_numpy(np.sort(g.choice(n, size=s, replace=False)).astype(np.int32)).cuda()
    knn = torch.empty(n, dtype=torch.float32, device="cuda")
    ctx.knn_distance(n, d, _ptr(X), d, s, _ptr(ref), KNN_K, _ptr(knn))
    F = torch.empty((n, d + 2), dtype=torch.float32, device="cuda")
    ctx.leverage_features(n, d, _ptr(X), d, _ptr(knn), _ptr(F))
    return F


def instance_targets(ctx: Context, w: datagen.Workload, l: int = TRAIN_L, q: int = 1):
    """(F, t, lambda): model inputs and centred log ridge leverage scores of one instance (device tensors)."""
    import torch
    n, d = w.n, w.d
    X = torch.from_numpy(w.X).cuda()
    y = torch.from_numpy(w.y).cuda()
    F = instance_inputs(ctx, X, n, d)
    Om_h = datagen.rng(w.seed + 7919).standard_normal((n, l), dtype=np.float32)
    Om = torch.from_numpy(np.ascontiguousarray(Om_h.T)).cuda()  # n x l column major
    Z = torch.empty((l, n), dtype=torch.float64, device="cuda")
    ctx.lowrank(n, d, l, q, _ptr(X), d, _ptr(y), _ptr(Om), n, w.gamma, _ptr(Z), n, precision=1)
    G = torch.empty((l, l), dtype=torch.float64, device="cuda")
    ctx.gemm_tn(n, l, l, 1.0, _ptr(Z), n, _ptr(Z), n, 0.0, _ptr(G), l)
    ctx.sync()
    sigma2 = np.linalg.eigvalsh(G.cpu().numpy())
    lam = lambda_for_deff(sigma2, DEFF_FRACTION * n)
    lev = torch.empty(n, dtype=torch.float64, device="cuda")
    ctx.ridge_leverage(n, l, _ptr(Z), n, lam, _ptr(lev))
    t = torch.log(torch.clamp(lev, min=1e-30))
    t = (t - t.mean()).to(torch.float32)
    return F, t, lam


def train(ctx: Context, instances: int = 200, epochs: int = 8, batch: int = 8192, lr: float = 1e-3,
          seed: int = 1, holdout: int = 10, log=print, config: str = "c5"):
    """Train the leverage model on `config`'s workload family; returns (net, mean, scale, info)."""
    import torch
    make, dim, _ = CONFIGS[config]
    t0 = time.perf_counter()
    Fs, ts, lams = [], [], []
    for k in range(instances + holdout):
        w = make(10_000 + k)
        F, t, lam = instance_targets(ctx, w)
        Fs.append(F)
        ts.append(t)
        lams.append(lam)
    F_all = torch.cat(Fs[:instances])
    t_all = torch.cat(ts[:instances])
    F_val = torch.cat(Fs[instances:]) if holdout else None
    t_val = torch.cat(ts[instances:]) if holdout else None
    t_data = time.perf_counter() - t0
    mean = F_all.mean(0).cpu().numpy().astype(np.float32)
    scale = (1.0 / torch.clamp(F_all.std(0), min=1e-6)).cpu().numpy().astype(np.float32)
    net = Mlp(ctx, dim + 2, WIDTH, HIDDEN, seed=seed)
    net.set_input_scaling(mean, scale)
    m = F_all.shape[0]
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    steps_per_epoch = m // batch
    total = epochs * steps_per_epoch
    losses, val = [], []
    step = 0
    for ep in range(epochs):
        perm = torch.randperm(m, device="cuda", generator=gen)
        for b in range(steps_per_epoch):
            sel = perm[b * batch:(b + 1) * batch]
            Fb = F_all.index_select(0, sel).contiguous()
            tb = t_all.index_select(0, sel).contiguous()
            cur = lr * 0.5 * (1.0 + math.cos(math.pi * step / total))  # cosine decay
            losses.append(net.adam_step(batch, _ptr(Fb), _ptr(tb), max(cur, 1e-6)))
            step += 1
        if holdout:
            vl = []
            for v0 in range(0, F_val.shape[0], 65536):
                Fv = F_val[v0:v0 + 65536].contiguous()
                tv = t_val[v0:v0 + 65536].contiguous()
                g = torch.empty(net.nparams, dtype=torch.float32, device="cuda")
                vl.append(net.gradients(Fv.shape[0], _ptr(Fv), _ptr(tv), _ptr(g)) * Fv.shape[0])
            val.append(float(sum(vl) / F_val.shape[0]))
        log(f"epoch {ep + 1}/{epochs}: train loss {np.mean(losses[-steps_per_epoch:]):.4f}"
            + (f", held-out loss {val[-1]:.4f}" if val else ""))
    info = {"config": config, "instances": instances, "holdout": holdout, "n": TRAIN_N, "d": dim, "l": TRAIN_L,
            "deff_fraction": DEFF_FRACTION, "lambda_median": float(np.median(lams)), "epochs": epochs,
            "batch": batch, "lr": lr, "seconds_data": t_data, "seconds_total": time.perf_counter() - t0,
            "loss_first": float(losses[0]), "loss_last_epoch": float(np.mean(losses[-steps_per_epoch:])),
            "heldout_loss": val, "target_variance_heldout": float(t_val.var().item()) if holdout else None}
    return net, mean, scale, info


def save_model(path, net: Mlp, mean, scale, info):
    np.savez_compressed(path, params=net.get_params(), mean=mean, scale=scale, width=WIDTH, hidden=HIDDEN,
                        in_dim=net.in_dim, info=json.dumps(info))


def load_model(ctx: Context, path=MODEL_PATH) -> Mlp:
    z = np.load(path, allow_pickle=False)
    net = Mlp(ctx, int(z["in_dim"]), int(z["width"]), int(z["hidden"]), seed=0)
    net.set_params(z["params"])
    net.set_input_scaling(z["mean"], z["scale"])
    return net


def landmark_residual(ctx: Context, w: datagen.Workload, r: int, net: Mlp | None, seed: int, s_res: int = 512,
                      s_knn: int = 16384):
    """Sampled residual of the Nystrom factor on r landmarks drawn by the model (net) or uniformly (net=None:
    all logits 0, the same Gumbel top-k without the network)."""
    import torch
    n, d = w.n, w.d
    X = torch.from_numpy(w.X).cuda()
    y = torch.from_numpy(w.y).cuda()
    logits = torch.zeros(n, dtype=torch.float32, device="cuda")
    if net is not None:
        F = instance_inputs(ctx, X, n, d, s_knn=s_knn, seed=seed)
        net.forward(n, _ptr(F), _ptr(logits))
    keys = torch.empty(n, dtype=torch.float32, device="cuda")
    ctx.gumbel_keys(n, _ptr(logits), seed, _ptr(keys))
    idx = torch.empty(r, dtype=torch.int32, device="cuda")
    ctx.select_topk(n, _ptr(keys), r, _ptr(idx))
    Z = torch.empty((r, n), dtype=torch.float64, device="cuda")
    ctx.landmark_factor(n, d, _ptr(X), d, _ptr(y), w.gamma, r, _ptr(idx), _ptr(Z), n)
    g = np.random.default_rng(seed + 17)
    S = torch.from_numpy(np.sort(g.choice(n, size=min(s_res, n), replace=False)).astype(np.int32)).cuda()
    return ctx.residual_estimate(n, d, _ptr(X), d, _ptr(y), w.gamma, r, _ptr(Z), n, S.numel(), _ptr(S))


def evaluate(ctx: Context, net: Mlp, seeds=(90_001, 90_002, 90_003), r: int = 512, config: str = "c5"):
    make = CONFIGS[config][0]
    out = []
    for s in seeds:
        w = make(s)
        out.append({"seed": s, "learned": landmark_residual(ctx, w, r, net, s),
                    "uniform": landmark_residual(ctx, w, r, None, s)})
    return out


def main(argv=None):
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["train", "evaluate"])
    ap.add_argument("--config", choices=sorted(CONFIGS), default="c5")
    ap.add_argument("--out", default=None)
    ap.add_argument("--model", default=None)
    ap.add_argument("--instances", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=8)
    args = ap.parse_args(argv)
    torch.cuda.init()
    ctx = Context(0, torch.cuda.current_stream().cuda_stream)
    default_path = str(CONFIGS[args.config][2])
    if args.cmd == "train":
        net, mean, scale, info = train(ctx, instances=args.instances, epochs=args.epochs, config=args.config)
        info["evaluation"] = evaluate(ctx, net, config=args.config)
        save_model(args.out or default_path, net, mean, scale, info)
        print(json.dumps(info))
    else:
        net = load_model(ctx, args.model or default_path)
        print(json.dumps(evaluate(ctx, net, config=args.config)))


if __name__ == "__main__":
    main()
