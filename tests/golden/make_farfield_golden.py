"""Generate the far-field golden fixtures from the REFERENCE's own CPU path.

Runs the reference's celeris::propagate_pillars (src/celeris/analysis/focal.cpp:
205-238, built from its sources into oracle/_ref/ by oracle/Makefile) on small
seeded inputs and stores inputs and |E|^2 in farfield_ref.npz. The complex
field E is stored from the plain-C restatement, after checking that its |E|^2
agrees with the reference's to 1e-13. Run from the repo root:
    make -C oracle && python tests/golden/make_farfield_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import farfield as F  # noqa: E402

CASES = [
    # name, npil, seed, spread, wavelength, z, cx, cy, n, half_window
    ("ragged_257", 257, 1, 8.0, 0.55, 30.0, 0.0, 0.0, 17, 3.0),
    ("offaxis_1000", 1000, 2, 20.0, 0.633, 100.0, 1.25, -0.75, 24, 5.0),
    ("single_pillar", 1, 3, 1.0, 0.532, 50.0, 0.0, 0.0, 9, 2.0),
    ("two_by_two", 7, 4, 4.0, 0.45, 10.0, 0.5, 0.5, 2, 1.0),
]


def main():
    out = {}
    for name, npil, seed, spread, wl, z, cx, cy, n, W in CASES:
        rng = np.random.default_rng(seed)
        px = rng.uniform(-spread, spread, npil)
        py = rng.uniform(-spread, spread, npil)
        t = rng.uniform(0.5, 1.0, npil) * np.exp(1j * rng.uniform(0, 2 * np.pi, npil))
        I_ref = F.ref_propagate_pillars(px, py, t, cx, cy, z, wl, n, W)
        k = 2.0 * np.pi / wl
        E = F.rs_field(px, py, t, cx, cy, z, k, n, W)
        rel = np.max(np.abs(np.abs(E) ** 2 - I_ref)) / np.max(I_ref)
        assert rel < 1e-13, (name, rel)
        for key, val in dict(px=px, py=py, t=t, I_ref=I_ref, E=E,
                             params=np.array([wl, z, cx, cy, n, W, k])).items():
            out[f"{name}/{key}"] = val
    np.savez_compressed(os.path.join(HERE, "farfield_ref.npz"), **out)
    print("wrote", os.path.join(HERE, "farfield_ref.npz"))


if __name__ == "__main__":
    main()
