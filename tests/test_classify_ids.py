"""The classification of primary-ray ID disagreements between the reference's
triangle test and the watertight one (bench.classify_ids), on hand-made hit
records: cracks, leaks and depth ties are explained, anything else is not."""
import numpy as np

from aviatorengine2_b200 import _lib
from bench import classify_ids

MISS = _lib.MISS


def hits(rows):
    h = np.zeros(len(rows), _lib.HIT)
    for i, (obj, prim, t, a, b) in enumerate(rows):
        h[i] = (t, a, b, obj, prim)
    return h


def test_categories():
    ref = hits([(1, 5, 10.0, 0.3, 0.3),      # agree
                (1, 6, 12.0, 0.3, 0.3),      # crack: wt nearer, at an edge
                (2, 7, 9.0, 0.004, 0.5),     # leak: ref nearer, at an edge
                (3, 8, 20.0, 0.3, 0.3),      # depth tie
                (4, 9, 30.0, 0.3, 0.3),      # unexplained: wt nearer, far from edges
                (MISS, MISS, 0.0, 0.0, 0.0)])  # crack: the reference missed
    wt = hits([(1, 5, 10.0, 0.3, 0.3),
               (1, 7, 11.0, 0.005, 0.4),
               (2, 8, 9.5, 0.3, 0.3),
               (5, 1, 20.0000019, 0.3, 0.3),
               (6, 2, 29.0, 0.3, 0.3),
               (7, 3, 40.0, 0.5, 0.001)])
    c = classify_ids(ref, wt)
    assert c["disagree"] == 5
    assert (c["crack"], c["leak"], c["depth_tie"], c["unexplained"]) == (2, 1, 1, 1)
    assert c["unexplained_examples"][0]["ray"] == 4
    assert c["agreement_excluding_explained"] == 1.0 - 1 / 2
