"""Generate the golden vectors under tests/golden/ from the reference itself.

Runs the reference renderer compiled from its own sources (oracle/_ref, built
by oracle/Makefile from the reference tree) on the cases of cases.py and
stores per-sample trace/shade results (class, steps, final state, g, sky
direction, XYZ, jet emission) and one whole frame of pixels.  Usage, where the reference
tree exists:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import oracle  # noqa: E402
from cases import CASES, RENDER_CASE  # noqa: E402


def main():
    ref = oracle.reference()
    if ref is None:
        raise SystemExit("oracle/_ref was not built (needs the reference sources)")
    for name, (make, (x0, y0, w, h)) in CASES.items():
        cfg = make()
        arr, st = ref.trace_rays(cfg, x0, y0, w, h)
        np.savez_compressed(
            os.path.join(HERE, f"{name}.npz"),
            window=np.array([x0, y0, w, h]), what=arr["what"].astype(np.int8),
            steps=arr["steps"], y=arr["y"], g=arr["g"], dir=arr["dir"], xyz=arr["xyz"], jet=arr["jet"],
            stats=np.array([st.rays, st.steps, st.captured, st.disc_hits, st.sun_hits, st.star_hits,
                            st.escaped, st.exhausted]),
            drift=np.array([st.max_norm_error, st.max_carter_drift]),
        )
        print(name, len(arr), "rays", np.bincount(arr["what"], minlength=6))
    # Digests of the reference star catalogue and blackbody table.
    import hashlib
    import json

    cat = ref.star_catalogue(250000, 20240921)
    table = np.array([ref.blackbody_xyz(T) for T in (50.0, 300.0, 5772.0, 1.0e5, 3.0e7, 3.0e9)])
    with open(os.path.join(HERE, "catalogue.json"), "w") as f:
        json.dump({
            "count": 250000, "seed": 20240921,
            "sha256_float64_le": hashlib.sha256(cat.astype("<f8").tobytes()).hexdigest(),
            "first_star": cat[0].tolist(), "last_star": cat[-1].tolist(),
            "blackbody_T": [50.0, 300.0, 5772.0, 1.0e5, 3.0e7, 3.0e9],
            "blackbody_xyz": table.tolist(),
        }, f, indent=1)
    name, make = RENDER_CASE
    cfg = make()
    px, st = ref.render(cfg)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), pixels=px,
                        stats=np.array([st.rays, st.steps, st.captured, st.disc_hits, st.sun_hits,
                                        st.star_hits, st.escaped, st.exhausted]),
                        drift=np.array([st.max_norm_error, st.max_carter_drift]),
                        total_flux=np.array([st.total_flux]))
    print(name, px.shape)


if __name__ == "__main__":
    main()
