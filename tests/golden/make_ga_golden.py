"""Golden vectors for the restated ga2d morphology score.

Reads LangmuirPython/ga2d/score.cache (score, image path) in the reference
tree (REFERENCE, default /root/reference), decodes every listed PNG the way
ga.py:104-105 does (PIL, converted to 8-bit greyscale "L"), scores it with
oracle/ga_score.py and reports how many restated scores equal the cached ones
to the cache's printed precision (3 decimals).  Every sixth binary image is
written, bit-packed, to ga_score.npz with its cached score, so the tests need
no reference tree.

Usage:  python tests/golden/make_ga_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np
from PIL import Image

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REFERENCE = os.environ.get("REFERENCE", "/root/reference")
sys.path.insert(0, ROOT)

from oracle import ga_score as G  # noqa: E402


def main():
    base = os.path.join(REFERENCE, "LangmuirPython", "ga2d")
    rows = [line.split() for line in open(os.path.join(base, "score.cache")) if line.strip()]
    images, cached, names, restated = [], [], [], []
    exact = 0
    worst = (0.0, "")
    for k, (s, path) in enumerate(rows):
        im = np.asarray(Image.open(os.path.join(base, path)).convert("L"))
        sc = G.score(im)
        err = abs(sc - float(s))
        exact += err <= 5e-4
        if err > worst[0]:
            worst = (err, path)
        binary = set(np.unique(im).tolist()) <= {0, 255}
        if binary and k % 6 == 0:
            images.append(np.packbits(im == 255, axis=None))
            cached.append(float(s))
            names.append(path)
            restated.append(sc)
    print(f"{exact} of {len(rows)} restated scores equal score.cache to 3 decimals; "
          f"largest difference {worst[0]:.4f} ({worst[1]})")
    out = os.path.join(HERE, "ga_score.npz")
    np.savez_compressed(out, images=np.stack(images), cached=np.array(cached),
                        restated=np.array(restated), names=np.array(names),
                        shape=np.array([256, 256]))
    print(f"wrote {len(images)} images to {out}")


if __name__ == "__main__":
    main()
