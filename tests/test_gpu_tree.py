"""Device tree / sort / lists against the CPU oracle: bit-exact integer
results (box numbering, parents, children, levels, point permutations, box
ranges, lists 1-4) and identical box centres.

Reference behaviour pinned: pts_tree2d.f / tree_routs2d.f (2D),
pts_tree3d.f / tree_routs3d.f (3D), through the oracle, which itself matches
the reference logs (test_oracle_golden.py)."""
import os

import numpy as np
import pytest

import oracle_lib as O
from zfmm_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def compare(D, ndiv, z, zt=None, isep=1):
    import zfmm_b200
    g = zfmm_b200.tree_dump(D, ndiv, z, zt, isep=isep)
    o = O.tree_dump(D, ndiv, z, zt, isep=isep)
    assert g["nboxes"] == o["nboxes"]
    assert g["nlevels"] == o["nlevels"]
    assert np.array_equal(g["laddr"], o["laddr"])
    for k in ["ilevel", "iparent", "nchild", "ichild", "isrc", "isrcse", "itarg", "itargse",
              "nlist", "lists_flat"]:
        assert np.array_equal(g[k], o[k]), k
    assert g["mnlist"] == o["mnlist"]
    assert np.array_equal(g["centers"], o["centers"])
    return g


def test_tree2d_fixture_matches_oracle_and_log():
    z = np.load(os.path.join(GOLD, "fixture2d.npz"))["zsrc"]
    g = compare(2, 25, z)
    assert g["nboxes"] == 5453 and g["nlevels"] == 10
    assert g["mnlist"] == [12, 27, 15, 5]


def test_tree3d_fixture_matches_oracle_and_log():
    z = np.load(os.path.join(GOLD, "fixture3d.npz"))["zsrc"]
    g = compare(3, 1000, z)
    assert g["nboxes"] == 201 and g["nlevels"] == 3
    assert g["mnlist"] == [34, 56, 56, 14]


@pytest.mark.parametrize("seed", [0, 1])
def test_tree2d_clustered(seed):
    w = W.clustered2d(30000, seed=seed)
    z = w["zsrc"].T
    compare(2, 20, z)


def test_tree2d_separate_targets_and_isep2():
    w = W.clustered2d(8000, seed=3)
    t = W.lap2d_uniform(5000, seed=4)
    compare(2, 15, w["zsrc"].T, t["zsrc"].T)
    compare(2, 20, w["zsrc"].T, t["zsrc"].T, isep=2)


def test_tree2d_curve():
    w = W.curve2d(60000, seed=2)
    compare(2, 20, w["zsrc"].T)


def test_tree3d_random():
    rng = np.random.default_rng(5)
    x = rng.standard_normal((40000, 3)) * np.array([1.0, 0.3, 0.05])
    z = x + 0.05j * np.sin(x)
    compare(3, 50, z)
