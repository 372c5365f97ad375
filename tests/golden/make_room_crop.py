"""Generate the FP64 oracle reference of the hidden-light room's central crop.

The convergence measurement (guided vs plain time to relMSE 1e-3) judges
both GPU arms against this image: the FP64 restatement of the reference's
integrator (oracle/pt_oracle.cpp, precision 64) rendered at many samples per
pixel over a 128 x 128 crop of the 1024 x 1024 hidden-light room (depth 16,
Sobol), on sample indices far from any the GPU renders use (frames from
2^20 on), so the reference's noise is independent of theirs.

The render runs in chunks; after every chunk the per-pixel mean, the
variance of that mean (sample variance / n) and the metadata are written to
the fixture (float32), and the running sums to a state file beside it (not
committed), so an interrupted run leaves a usable, self-describing fixture
and a rerun resumes from the state.

    python tests/golden/make_room_crop.py --spp 65536 --chunk 512
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from pathtracingtutorial_b200 import scenes  # noqa: E402
from oracle.pyoracle import Oracle  # noqa: E402

CROP = (448, 448, 576, 576)          # x0, y0, x1, y1 of the 1024 x 1024 image
FIRST_FRAME = 1 << 20                # sample indices 4 * 2^20 and up
EPS_REL = 1e-2
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "room_crop_fp64.npz")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--spp", type=int, default=65536)
    ap.add_argument("--chunk", type=int, default=512)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--out", default=OUT)
    a = ap.parse_args()
    sa = scenes.hidden_light_room()
    O = Oracle()
    prep = O.prepare(sa)
    x0, y0, x1, y1 = CROP
    shape = (y1 - y0, x1 - x0, 3)
    S = np.zeros(shape, np.float64)
    Q = np.zeros(shape, np.float64)
    n = 0
    secs = 0.0
    state = a.out[:-4] + ".state.npz"
    if os.path.exists(state):
        z = np.load(state)
        if int(z["first_frame"]) == FIRST_FRAME and tuple(z["crop"]) == CROP:
            S, Q, n, secs = z["sum"], z["sumsq"], int(z["spp"]), float(z["seconds"])
            print(f"resuming at {n} spp", flush=True)
    spf = sa.sample_per_frame
    while n < a.spp:
        k = min(a.chunk, a.spp - n)
        frames = k // spf
        (m, v), cnt = O.render(prep, spf, sa.max_depth, sa.sampler, frames=frames,
                               first_frame=FIRST_FRAME + n // spf, precision=64, rtl=0, threads=a.threads,
                               crop=CROP)
        m, v = m[y0:y1, x0:x1], v[y0:y1, x0:x1]
        k = frames * spf
        S += m * k
        Q += v * (k - 1) + m * m * k
        n += k
        secs += cnt["seconds"]
        mean = S / n
        var = np.maximum(Q - n * mean * mean, 0.0) / max(n - 1, 1)
        var_of_mean = var / n
        noise = float(np.mean(var_of_mean / (mean * mean + EPS_REL)))
        np.savez(state + ".tmp.npz", sum=S, sumsq=Q, spp=n, seconds=secs, first_frame=FIRST_FRAME,
                 crop=np.array(CROP))
        os.replace(state + ".tmp.npz", state)
        np.savez_compressed(a.out + ".tmp.npz", mean=mean.astype(np.float32),
                            var_of_mean=var_of_mean.astype(np.float32), spp=n,
                            first_frame=FIRST_FRAME, crop=np.array(CROP), seconds=secs, noise_relmse=noise,
                            eps_rel=EPS_REL, scene=sa.name, width=1024, height=1024, max_depth=sa.max_depth,
                            sampler="sobol")
        os.replace(a.out + ".tmp.npz", a.out)
        print(f"{n} spp  {secs:.0f} s  mean {mean.mean():.5f}  noise relMSE {noise:.3e}", flush=True)


if __name__ == "__main__":
    main()
