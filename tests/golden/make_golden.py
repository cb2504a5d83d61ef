"""Generate the golden vectors in tests/golden/ from the REFERENCE's own CPU tracer.

Run where the reference sources are available (they are read only at build time):
    make -C oracle            # builds oracle/_ref/libftref.so from the reference headers
    python tests/golden/make_golden.py [case ...]   # all cases when none is named

For every case in tests/cases.py (the small cases and the benchmark configurations at their
own scene and film size) it stores, from Renderer::tracePhoton run single-threaded
with the reference's per-photon seeding (hero-wavelength cases through tracePhotonHero):
the energy report, the film (XYZ sums and hits), and per photon the number of ray queries,
the termination and the final beta (the last two meaningful for one wavelength per photon).  It also
stores the PCG32 streams of a few photon indices, a baked camera and an emission CDF.
The scene's content hash is stored so that drift in the scene generator is detected.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from goodphotons_b200 import lib, scenes  # noqa: E402
from oracle_bind import Reference  # noqa: E402
import cases  # noqa: E402


def main():
    L = lib.load()
    R = Reference()
    only = set(sys.argv[1:])
    for name, (mk, res, n, mb, seed, hero) in {**cases.CASES, **cases.CONFIG_CASES}.items():
        if only and name not in only:
            continue
        d = mk(L)
        cam = cases.camera(L, res)
        # film and energy accumulated like renderForward; per-photon ray counts (and, for one
        # wavelength per photon, the termination and final beta) from a photon-by-photon run
        r = R.trace(d, cam, n, seed_base=seed, max_bounce=mb, hero_c=hero)
        r.update({k: v for k, v in R.trace(d, cam, n, seed_base=seed, max_bounce=mb, per_photon=True,
                                           hero_c=hero).items() if k in ("rays", "fate", "beta")})
        np.savez_compressed(
            os.path.join(HERE, f"trace_{name}.npz"), scene_hash=np.array(cases.scene_hash(d)),
            energy=r["energy"], xyz=r["xyz"], hits=r["hits"], rays=r["rays"].astype(np.int32),
            fate=r["fate"].astype(np.int8), beta=r["beta"], res=res, n=n, max_bounce=mb, seed_base=seed,
            hero_c=hero)
        print(name, r["energy"])
    if only and "streams" not in only:
        return
    ks = np.array([0, 1, 2, 3, 1000, 123456789, 2**40 + 5, 2**63 - 1], dtype=np.uint64)
    uni = np.stack([R.uniforms(int(k), 16) for k in ks])
    cam = R.look_at((1.0, 1.0, 5.4), (1.0, 1.0, 1.0), (0.0, 1.0, 0.0), 40.0, 256, 192)
    camv = np.array(list(cam.eye) + list(cam.u) + list(cam.v) + list(cam.w) + [cam.tan_half_x, cam.tan_half_y])
    d = scenes.make_cornell(L)
    power, integral, cdf = R.emitter(d, 0)
    np.savez_compressed(os.path.join(HERE, "streams.npz"), photon=ks, uniforms=uni, camera=camv,
                        bb_power=power, bb_integral=integral, bb_cdf=cdf)
    print("streams", uni[0, :4], power)


if __name__ == "__main__":
    main()
