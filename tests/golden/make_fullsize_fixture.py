"""Writes the 256^3 reference fixture of this directory by running the REFERENCE's own
code (oracle/_ref/libim3d_ref.so: the reference headers compiled in place by
oracle/Makefile with the headless, GetPot and FFTW-API shims) on the full 256^3
segmentation workload:

* input: the seeded 8-ellipsoid 256^3 volume (seed 0; semi-axes 10-40, intensities
  0.6-0.9, bias 0.7->1.3 along k, noise 0.05) and the radius-20 sphere level set,
  both rounded to float32 and widened back to float64, so that the FP32 and FP64 GPU
  paths and the reference all start from the same numbers;
* parameters: sigma 3, lamda1 = lamda2 = 1, epsilon 1e-3, lamda 0.5, Dirichlet
  boundary, 100 outer iterations, the Poisson step of each iteration solved by
  red-black Gauss-Seidel (plugged in through set_onestep_poisson) to relative
  residual 1e-6 on the residual-check schedule the GPU path uses;
* T = double.

The whole fields (256^3 doubles) are too large to commit, so the fixture keeps:
* the iteration, sweep and residual-check counts;
* per field (phi, u, f1, f2): sum, L2 norm, max-abs;
* sign(phi - 0.5) of every voxel, bit-packed (segmentation agreement and Dice are
  then exact over the whole volume), its count and its SHA-256;
* u, f1 and f2 on the lattice (1::4, 2::4, 3::4) -- 64^3 samples each -- in float32
  (rounding 6e-8, far below the 1e-5 comparison bars), for relative-L2 comparisons.

It takes about 45 minutes on 8 host cores (8 FFTs of 274^3 per outer iteration in the
in-tree FFT, and ~40 red-black sweeps).

    python tests/golden/make_fullsize_fixture.py [--full-out PATH]

--full-out also saves the complete FP64 fields (about 512 MB, not committed).
"""
import argparse
import hashlib
import importlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle_py as O  # noqa: E402

synth = importlib.import_module("3dimagetoolkit_b200.synth")

SEED = 0
PARAMS = dict(sigma=3.0, lamda1=1.0, lamda2=1.0, epsilon=1e-3, lamda=0.5, dt=1.0, a0=0.0,
              b0=1.0, bc=2, maxiter=100, tol=0.0, gs_rel_res_tol=1e-6, gs_check_every=0,
              gs_max_sweeps=1000, omega=1.0)
LATTICE = (slice(1, None, 4), slice(2, None, 4), slice(3, None, 4))
OUT = os.path.join(HERE, "rsfe_c2_256_ref.npz")


def inputs():
    u0, phi0 = synth.config_volume("c2", seed=SEED, dtype=np.float32)
    return u0.astype(np.float64), phi0.astype(np.float64)


def summarise(r, alpha=0.5):
    out = {}
    for f in ("phi", "u", "f1", "f2"):
        x = r[f]
        out[f"{f}_sum"] = np.array(float(x.sum()))
        out[f"{f}_l2"] = np.array(float(np.linalg.norm(x)))
        out[f"{f}_linf"] = np.array(float(np.abs(x).max()))
    for f in ("u", "f1", "f2"):
        out[f"{f}_lattice"] = np.ascontiguousarray(r[f][LATTICE], dtype=np.float32)
    inside = r["phi"] > alpha
    bits = np.packbits(inside.ravel())
    out["inside_bits"] = bits
    out["inside_count"] = np.array(int(inside.sum()))
    out["inside_sha256"] = np.array(hashlib.sha256(bits.tobytes()).hexdigest())
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--full-out", default="")
    ap.add_argument("--maxiter", type=int, default=PARAMS["maxiter"])
    args = ap.parse_args()
    if not O.ref_available():
        sys.exit("oracle/_ref/libim3d_ref.so is missing: run `make -C oracle ref` first")
    u0, phi0 = inputs()
    kw = dict(PARAMS, maxiter=args.maxiter)
    t0 = time.time()
    r = O.rsfe_apply(u0, phi0, O.default_params(**kw), use_reference=True)
    secs = time.time() - t0
    st = r["stats"]
    out = summarise(r)
    out["iterations"] = np.array(st["iterations"])
    out["total_sweeps"] = np.array(st["total_sweeps"])
    out["residual_checks"] = np.array(st["residual_checks"])
    out["last_rel_res"] = np.array(st["last_rel_res"])
    out["last_tol"] = np.array(st["last_tol"])
    out["params"] = np.array(json.dumps(kw))
    out["timeline"] = O.ref_last_timeline()
    out["threads"] = np.array(int(os.environ.get("OMP_NUM_THREADS", os.cpu_count())))
    out["seconds"] = np.array(secs)
    path = OUT if args.maxiter == PARAMS["maxiter"] else OUT.replace(".npz", f"_it{args.maxiter}.npz")
    np.savez_compressed(path, **out)
    if args.full_out:
        np.savez(args.full_out, **{f: r[f] for f in ("phi", "u", "f1", "f2")})
    print(json.dumps({k: (v.item() if v.ndim == 0 and k not in ("timeline",) else None)
                      for k, v in out.items() if v.ndim == 0}), flush=True)
    print(path, os.path.getsize(path), "bytes", f"{secs:.0f} s")


if __name__ == "__main__":
    main()
