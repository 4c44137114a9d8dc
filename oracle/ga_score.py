"""The reference's morphology score, restated (numpy + scipy.ndimage).

TEST INFRASTRUCTURE ONLY: the "method without the network" that the trained
surrogate is compared against, and its CPU timing.  Only tests/ and bench.py
import it.

Follows LangmuirPython/ga2d/ga.py:83-141 (``score``) and the descriptors it
calls in ga2d/ga_analyze.py: ``average_domain_size`` (ga_analyze.py:166-201)
and ``transfer_distance`` (ga_analyze.py:277-380).  Pinned against the 176
cached scores of ga2d/score.cache through tests/golden/ga_score.npz.

The image is an 8-bit greyscale array (0 / 255) as the reference reads it
(PIL "L"), indexed [row][column].
"""
from __future__ import annotations

import math

import numpy as np
from scipy import ndimage


def average_domain_size(image):
    """Mean and std over connected regions of the image's nonzero phase of
    each region's largest distance to the other phase (ga_analyze.py:166-201)."""
    labels, nb = ndimage.label(image)
    dists = ndimage.distance_transform_edt(image)
    imax = ndimage.maximum(dists, labels, index=np.arange(1, nb + 1))
    imax = np.asarray(imax, np.float64)
    if imax.size == 0:
        return float("nan"), float("nan")
    return float(np.mean(imax)), float(np.std(imax))


def _bfs(passable, seeds):
    """Lattice (4-neighbour) distance from the seed pixels through
    ``passable`` pixels; -1 where unreached.  Seeds are at distance 0 whether
    or not they are passable, as in the reference's work queue."""
    dist = np.full(passable.shape, -1.0)
    frontier = seeds.copy()
    dist[frontier] = 0.0
    visited = frontier.copy()
    d = 0
    while frontier.any():
        d += 1
        nb = np.zeros_like(frontier)
        nb[1:, :] |= frontier[:-1, :]
        nb[:-1, :] |= frontier[1:, :]
        nb[:, 1:] |= frontier[:, :-1]
        nb[:, :-1] |= frontier[:, 1:]
        frontier = nb & passable & ~visited
        visited |= frontier
        dist[frontier] = d
    return dist


def transfer_distance(original):
    """(avg1, con1, avg2, con2): breadth-first distances of the nonzero phase
    from one electrode and of the zero phase from the other, along axis 0 of
    the image rotated by 90 degrees (ga_analyze.py:277-380 with axis=0,
    rot90=1).  Left seeds are nonzero pixels of the first row and spread
    through pixels equal to 255; right seeds are zero pixels of the last row
    and spread through zeros."""
    image = np.rot90(np.asarray(original), 1)
    left = np.zeros(image.shape, bool)
    left[0, :] = image[0, :] != 0
    right = np.zeros(image.shape, bool)
    right[-1, :] = image[-1, :] == 0
    d1 = _bfs(image == 255, left)
    d2 = _bfs(image == 0, right)
    dist = np.where(d1 >= 0, d1, d2)
    nz, z = image != 0, image == 0
    # a phase that reaches its electrode nowhere has transfer distance 0: the
    # cached score of images-256x256/rough/TriStripe-32.png (-717.900) is
    # reproduced with td1 = 0, not with the NaN of an empty average
    r1, r2 = nz & (dist >= 0), z & (dist >= 0)
    avg1 = float(np.average(dist[r1])) if r1.any() else 0.0
    avg2 = float(np.average(dist[r2])) if r2.any() else 0.0
    con1 = float(np.average(dist[nz] >= 0)) if nz.any() else 0.0
    con2 = float(np.average(dist[z] >= 0)) if z.any() else 0.0
    return avg1, con1, avg2, con2


def descriptors(image):
    image = np.asarray(image)
    ads1, _ = average_domain_size(image)
    inverted = image < image.mean()
    ads2, _ = average_domain_size(inverted)
    td1, connect1, td2, connect2 = transfer_distance(image)
    s22 = np.ones((2, 2))
    erosion = int(np.count_nonzero(np.logical_xor(image, ndimage.binary_erosion(image, structure=s22))))
    dilation = int(np.count_nonzero(np.logical_xor(image, ndimage.binary_dilation(image, structure=s22))))
    fraction = float(np.count_nonzero(image)) / float(image.size)
    return dict(ads=(ads1 + ads2) / 2.0, td1=td1, connect1=connect1, td2=td2, connect2=connect2,
                erosion=erosion, dilation=dilation, fraction=fraction)


def score(image):
    """Estimated maximum power of a morphology (ga.py:83-141)."""
    d = descriptors(image)
    ads, c1, c2 = d["ads"], d["connect1"], d["connect2"]
    ps = d["fraction"] * (1.0 - d["fraction"])
    return ((-1.98566e8) + (-1650.14) / ads + (-680.92) * math.pow(ads, 0.25)
            + 1.56236e7 * math.tanh(14.5 * (c1 + 0.4)) + 1.82945e8 * math.tanh(14.5 * (c2 + 0.4))
            + 2231.32 * c1 * c2
            + (-4.72813) * d["td1"] + (-4.86025) * d["td2"]
            + 3.79109e7 * ps ** 8
            + 0.0540293 * d["dilation"] + 0.0700451 * d["erosion"])


def phases_to_image(phase):
    """Surrogate phase (0 donor, 1 acceptor) -> 0/255 image.  White (255) is
    the phase the reference collects at the right electrode of the unrotated
    image (x = X - 1), as the acceptor's electrons are here."""
    return (np.asarray(phase, np.uint8) * 255).astype(np.uint8)
