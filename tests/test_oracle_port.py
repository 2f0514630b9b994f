"""The oracle's plain-C restatement, pinned against the reference's own
known-answer tests and against golden fixtures produced by the reference
itself (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

from oracle import port
from tests import parity
from tests.golden import make_golden

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
INF = float("inf")


# Known answers of the reference's BBox::intersect_ray tests (basics/bbox_test.cpp:103-203):
# (origin, direction, box min, box max) -> (hit, t0, t1 range)
BBOX_CASES = [
    ((0.125, -8.0, 0.25), (0.0, 1.0, 0.0), (-1.0, -2.5, -0.5), (8.0, 7.25, 2.0), True, 5.5, (15.25, 15.25001)),
    ((0.125, -8.0, 0.25), (0.0, 2.0, 0.0), (-1.0, -2.5, -0.5), (8.0, 7.25, 2.0), True, 2.75, (7.625, 7.62501)),
    ((20.0, -8.0, 0.25), (0.0, 1.0, 0.0), (-1.0, -2.5, -0.5), (8.0, 7.25, 2.0), False, None, None),
    ((0.0, 0.0, 0.0), (0.0, 1.0, 0.0), (-1.0, -2.5, -0.5), (8.0, 7.25, 2.0), True, 0.0, (7.25, 7.25001)),
    ((-1.0001, -8.0, 0.25), (0.0, 1.0, 0.0), (-1.0, -2.5, -0.5), (8.0, 7.25, 2.0), False, None, None),
    ((-4.0, 0.0, 0.0), (1.0, 0.0, 0.0), (1.0, -1.0, -1.0), (1.0, 1.0, 1.0), True, 5.0, (5.0, 5.00001)),
    ((-4.0, 0.0, 0.0), (0.5, 0.5, 0.5), (1.0, -20.0, -20.0), (1.0, 20.0, 20.0), True, 10.0, (10.0, 10.00001)),
]


@pytest.mark.parametrize("case", range(len(BBOX_CASES)))
def test_bbox_known_answers(case):
    o, d, lo, hi, hit, t0, t1r = BBOX_CASES[case]
    h, a, b = port.box_hit(lo, hi, o, d, INF)
    assert h == hit
    if hit:
        assert a == t0
        assert t1r[0] <= b <= t1r[1]


def test_instance_id_packing():
    # reference basics/instance_id_test.cpp:12-42
    v = 0
    for sub, bits in ((1, 1), (3, 2), (63, 10), (7, 5)):
        v = port.id_push(v, sub, bits)
    assert v & 0x1F == 7
    assert (v >> 5) & 0x3FF == 63
    assert (v >> 15) & 0x3 == 3
    assert (v >> 17) & 0x1 == 1


@pytest.mark.parametrize("name", ["plain", "heightfield", "instanced", "motion"])
def test_port_trace_matches_reference_golden(name):
    g = np.load(os.path.join(GOLDEN, "trace_%s.npz" % name))
    rays = {k[4:]: g[k] for k in g.files if k.startswith("ray_")}
    sc = make_golden.make_scene(name)
    mine = port.trace(sc, rays)
    ref = {"hit": g["hit"], "id": g["id"], "t": g["t"], "uv": g["uv"]}
    # the restatement produces uv for patch leaves only (cell centres, never 0);
    # sphere uv comes from acos and is checked on the GPU side
    patch = (mine["uv"][:, 0] != 0) & (g["closure"] == 1)
    rep = parity.compare_trace(ref, mine, rays["type"], uv_mask=patch)
    parity.assert_parity(rep)
    assert rep["closest_hits"] > 200
