"""Generate FP64 oracle references of a 128 x 128 crop: the hidden-light
room's central crop (--scene room, the default) or the 20M-triangle combined
scene's camera-0 central crop (--scene large).

The convergence measurement (guided vs plain time to relMSE 1e-3) judges
both GPU arms against this image: the FP64 restatement of the reference's
integrator (oracle/pt_oracle.cpp, precision 64) rendered at many samples per
pixel over a 128 x 128 crop of the 1024 x 1024 hidden-light room (depth 16,
Sobol), on sample indices far from any the GPU renders use (frames from
2^20 on), so the reference's noise is independent of theirs.

For the 20M-triangle scene the BVH, face order and light tables come from
the library's host prep (node for node the reference's, as the parity tests
check), so the oracle does not rebuild the tree single-threaded; its scene
uses disjoint sample indices likewise (frames from 2^20 on).

The render runs in chunks; after every chunk the per-pixel mean, the
variance of that mean (sample variance / n) and the metadata are written to
the fixture (float32), and the running sums to a state file beside it (not
committed), so an interrupted run leaves a usable, self-describing fixture
and a rerun resumes from the state.

    python tests/golden/make_room_crop.py --spp 65536 --chunk 512
    python tests/golden/make_room_crop.py --scene large --spp 4096 --chunk 128
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from pathtracingtutorial_b200 import scenes  # noqa: E402
from oracle.pyoracle import Oracle, Prepared  # noqa: E402

CROP = (448, 448, 576, 576)          # x0, y0, x1, y1 of the 1024 x 1024 image
LARGE_CROP = (896, 476, 1024, 604)   # x0, y0, x1, y1 of camera 0's 1920 x 1080 image
FIRST_FRAME = 1 << 20                # sample indices 4 * 2^20 and up
EPS_REL = 1e-2
HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "room_crop_fp64.npz")
LARGE_OUT = os.path.join(HERE, "large_crop_fp64.npz")


def large_prepared(O):
    """The 20M-triangle scene prepared by the library's host prep."""
    sa, _ = scenes.large_scene()
    s = sa.scene()
    s.build_accel()
    faces = s.faces()
    refs, pmf, alias = s.emissive_tables()
    env_pmf, env_alias = s.env_tables()
    prep = Prepared(np.ascontiguousarray(sa.vertices), faces, np.ascontiguousarray(sa.materials), s.bvh_nodes(),
                    s.info()["bvh_max_depth"], refs, pmf, alias, np.ascontiguousarray(sa.env, np.float32), env_pmf,
                    env_alias, O.camera_frame(sa.camera), int(sa.camera["width"]), int(sa.camera["height"]))
    return sa, prep


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--spp", type=int, default=65536)
    ap.add_argument("--chunk", type=int, default=512)
    ap.add_argument("--threads", type=int, default=0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--scene", choices=["room", "large"], default="room")
    a = ap.parse_args()
    O = Oracle()
    if a.scene == "room":
        sa = scenes.hidden_light_room()
        prep = O.prepare(sa)
        crop = CROP
        a.out = a.out or OUT
    else:
        sa, prep = large_prepared(O)
        crop = LARGE_CROP
        a.out = a.out or LARGE_OUT
    x0, y0, x1, y1 = crop
    shape = (y1 - y0, x1 - x0, 3)
    S = np.zeros(shape, np.float64)
    Q = np.zeros(shape, np.float64)
    n = 0
    secs = 0.0
    state = a.out[:-4] + ".state.npz"
    if os.path.exists(state):
        z = np.load(state)
        if int(z["first_frame"]) == FIRST_FRAME and tuple(z["crop"]) == crop:
            S, Q, n, secs = z["sum"], z["sumsq"], int(z["spp"]), float(z["seconds"])
            print(f"resuming at {n} spp", flush=True)
    spf = sa.sample_per_frame
    while n < a.spp:
        k = min(a.chunk, a.spp - n)
        frames = k // spf
        (m, v), cnt = O.render(prep, spf, sa.max_depth, sa.sampler, frames=frames,
                               first_frame=FIRST_FRAME + n // spf, precision=64, rtl=0, threads=a.threads,
                               crop=crop)
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
                 crop=np.array(crop))
        os.replace(state + ".tmp.npz", state)
        np.savez_compressed(a.out + ".tmp.npz", mean=mean.astype(np.float32),
                            var_of_mean=var_of_mean.astype(np.float32), spp=n,
                            first_frame=FIRST_FRAME, crop=np.array(crop), seconds=secs, noise_relmse=noise,
                            eps_rel=EPS_REL, scene=sa.name, width=int(sa.camera["width"]),
                            height=int(sa.camera["height"]), max_depth=sa.max_depth, sampler="sobol")
        os.replace(a.out + ".tmp.npz", a.out)
        print(f"{n} spp  {secs:.0f} s  mean {mean.mean():.5f}  noise relMSE {noise:.3e}", flush=True)


if __name__ == "__main__":
    main()
