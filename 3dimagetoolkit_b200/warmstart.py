"""Training and evaluation of the learned warm start of the Poisson step.

The network (csrc/unet.cu, im3d_unet_*) maps four fields of an outer iteration -- the
forcing term rhs, the previous solve's u, div(d - b) and phi -- to the correction the
solve will make to phi. Training pairs come from the plain solver: a segmentation run
with IM3D_WS_TRAIN takes one Adam step on every outer iteration's fields and the
correction its red-black Gauss-Seidel solve made (to relative residual 1e-6). With
IM3D_WS_PREDICT the correction starts each solve, which still runs to the same
residual; the previous iterate is kept when the network's start has the larger
residual.

Volumes come from the two-ellipsoid generator of the 64^3 workload (semi-axes 8-16,
intensity 0.8, bias 0.8 -> 1.2 along k, noise 0.05, a radius-20 sphere as the initial
level set): 128^3 volumes of seeds 0-199 for training, 256^3 volumes of seeds 1000-1015
held out for evaluation.

    python -m 3dimagetoolkit_b200.warmstart train --seeds 0-199
    python -m 3dimagetoolkit_b200.warmstart evaluate --seeds 1000-1015
"""
from __future__ import annotations

import os
import time

import numpy as np

from . import _abi, synth

HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS = os.path.join(HERE, "data", "warmstart_unet.npz")

# the segmentation parameters of the solver-generated pairs (the 256^3 workload's)
PARAMS = dict(sigma=3.0, lamda1=1.0, lamda2=1.0, epsilon=1e-3, lamda=0.5, dt=1.0, bc=2,
              tol=0.0, gs_rel_res_tol=1e-6, gs_max_sweeps=1000, omega=1.0, maxiter=100)


def volume(shape, seed, dtype=np.float32):
    """(u0, phi0) from the two-ellipsoid generator."""
    u0 = synth.ellipsoids(shape, seed, n=2, semi_axes=(8, 16), fg_mean=0.8, bias=(0.8, 1.2),
                          noise=0.05, dtype=dtype)
    return u0, synth.sphere_phi0(shape, 20.0, dtype=dtype)


def train(ctx: _abi.Context, net: _abi.UNet, seeds, shape=(128, 128, 128), lr=1e-3, maxiter=100,
          log=None, every=None, budget_s=None) -> dict:
    """One segmentation per seed with a training step on each of its solves; returns the
    per-seed mean losses, the number of pairs and the wall time. every(q) is called
    after each seed (e.g. to save the weights); budget_s stops after that many seconds."""
    params = _abi.default_params(**{**PARAMS, "maxiter": maxiter})
    losses = []
    pairs = 0
    t0 = time.time()
    ctx.set_warm_start(net, _abi.WS_TRAIN, lr)
    try:
        for q, s in enumerate(seeds):
            u0, phi0 = volume(shape, s)
            st = ctx.rsfe_apply(u0, phi0, params)["stats"]
            losses.append(st["ws_loss"])
            pairs += st["iterations"]
            if log and (q % 10 == 0 or q == len(seeds) - 1):
                log(f"seed {s}: mean loss {st['ws_loss']:.3e} ({pairs} pairs, {time.time() - t0:.0f} s)")
            if every:
                every(q)
            if budget_s and time.time() - t0 > budget_s:
                if log:
                    log(f"stopped after seed {s}: time budget of {budget_s:.0f} s")
                break
    finally:
        ctx.set_warm_start(None, _abi.WS_OFF)
    return {"losses": losses, "pairs": pairs, "seconds": time.time() - t0}


def save(net: _abi.UNet, path: str = WEIGHTS, **meta):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez_compressed(path, params=net.get_params(), **{k: np.asarray(v) for k, v in meta.items()})


def load(net: _abi.UNet, path: str = WEIGHTS) -> dict:
    d = np.load(path)
    net.set_params(d["params"])
    return {k: d[k] for k in d.files if k != "params"}


def _solve_ms(prof: dict) -> float:
    """Device time of the Poisson solves in a profiled run (the loop's "poisson_solve"
    stage: the half-sweeps, the residual evaluations and, with the warm start, the
    network, its residual checks and its fallback)."""
    return prof["poisson_solve"][0] if "poisson_solve" in prof else 0.0


def evaluate(ctx: _abi.Context, net: _abi.UNet, seeds, shape=(256, 256, 256), maxiter=100) -> dict:
    """Plain (previous-iterate start) against learned warm start on the same volumes:
    device time of the solves to relative residual 1e-6 per outer iteration, sweeps,
    the solves the network started, and the Dice overlap of the two segmentations."""
    import torch

    params = _abi.default_params(**{**PARAMS, "maxiter": maxiter})
    rows = []
    for s in seeds:
        u0, phi0 = volume(shape, s)
        u0_d = torch.from_numpy(u0).cuda()
        phi0_d = torch.from_numpy(phi0).cuda()
        out = {}
        # one untimed run first: buffers, filters and the network's activations allocated
        ctx.set_warm_start(net, _abi.WS_PREDICT)
        ctx.rsfe_apply(u0_d, phi0_d, _abi.default_params(**{**PARAMS, "maxiter": 2}))
        for mode in ("plain", "learned"):
            ctx.set_warm_start(net if mode == "learned" else None,
                               _abi.WS_PREDICT if mode == "learned" else _abi.WS_OFF)
            ctx.set_profiling(2)  # the solves as a whole: the launches inside keep their overlap
            ctx.profile(reset=True)
            r = ctx.rsfe_apply(u0_d, phi0_d, params)
            prof = ctx.profile(reset=True)
            ctx.set_profiling(0)
            st = r["stats"]
            out[mode] = dict(solve_ms=_solve_ms(prof), loop_ms=st["loop_ms"], sweeps=st["total_sweeps"],
                             iterations=st["iterations"], not_converged=st["not_converged"],
                             last_rel_res=st["last_rel_res"], ws_used=st["ws_used"],
                             ws_rejected=st["ws_rejected"], phi=r["phi"].cpu().numpy())
        ctx.set_warm_start(None, _abi.WS_OFF)
        it = max(out["plain"]["iterations"], 1)
        rows.append({
            "seed": s,
            "plain_solve_ms_per_iteration": out["plain"]["solve_ms"] / it,
            "learned_solve_ms_per_iteration": out["learned"]["solve_ms"] / it,
            "plain_sweeps_per_iteration": out["plain"]["sweeps"] / it,
            "learned_sweeps_per_iteration": out["learned"]["sweeps"] / it,
            "plain_loop_ms": out["plain"]["loop_ms"], "learned_loop_ms": out["learned"]["loop_ms"],
            "network_started": out["learned"]["ws_used"], "previous_iterate_kept": out["learned"]["ws_rejected"],
            "not_converged": out["plain"]["not_converged"] + out["learned"]["not_converged"],
            "last_rel_res": max(out["plain"]["last_rel_res"], out["learned"]["last_rel_res"]),
            "dice_learned_vs_plain": synth.dice(out["learned"]["phi"], out["plain"]["phi"]),
        })
    agg = {k: float(np.mean([r[k] for r in rows])) for k in rows[0] if k != "seed"}
    agg["speedup_time_to_tolerance"] = agg["plain_solve_ms_per_iteration"] / agg["learned_solve_ms_per_iteration"]
    return {"per_volume": rows, "mean": agg}


def main(argv=None):
    import argparse
    import json

    ap = argparse.ArgumentParser(description="train or evaluate the learned Poisson warm start")
    ap.add_argument("what", choices=["train", "evaluate", "forward"])
    ap.add_argument("--seeds", default="0-199", help="first-last (inclusive)")
    ap.add_argument("--size", type=int, default=0, help="cube side (train 128, evaluate 256)")
    ap.add_argument("--maxiter", type=int, default=100)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--weights", default=WEIGHTS)
    ap.add_argument("--init-seed", type=int, default=0)
    ap.add_argument("--budget", type=float, default=0, help="training: stop after this many seconds")
    a = ap.parse_args(argv)
    lo, hi = (int(v) for v in a.seeds.split("-"))
    seeds = list(range(lo, hi + 1))
    with _abi.Context(0) as ctx, _abi.UNet(ctx, seed=a.init_seed) as net:
        if a.what == "train":
            side = a.size or 128
            done = []

            def keep(q):
                done.append(seeds[q])
                if q % 20 == 19:
                    save(net, a.weights, seeds=np.array([lo, seeds[q]]), shape=np.array([side] * 3), lr=a.lr)

            res = train(ctx, net, seeds, shape=(side,) * 3, lr=a.lr, maxiter=a.maxiter,
                        log=lambda m: print(m, flush=True), every=keep, budget_s=a.budget or None)
            save(net, a.weights, seeds=np.array([lo, done[-1]]), shape=np.array([side] * 3), lr=a.lr,
                 pairs=res["pairs"], losses=np.array(res["losses"]), seconds=res["seconds"])
            print(json.dumps({"pairs": res["pairs"], "seconds": res["seconds"],
                              "first_loss": res["losses"][0], "last_loss": res["losses"][-1]}))
        elif a.what == "forward":
            # device time of one inference on random fields (CUDA events, median of 5)
            import torch

            side = a.size or 256
            x = torch.randn((1, 4, side, side, side), device="cuda", dtype=torch.float32)
            ts = []
            for q in range(7):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record()
                net.forward(x)
                e1.record()
                e1.synchronize()
                if q >= 2:
                    ts.append(e0.elapsed_time(e1))
            print(json.dumps({"size": side, "forward_ms": sorted(ts)[len(ts) // 2]}))
        else:
            load(net, a.weights)
            side = a.size or 256
            res = evaluate(ctx, net, seeds, shape=(side,) * 3, maxiter=a.maxiter)
            print(json.dumps(res))


if __name__ == "__main__":
    main()
