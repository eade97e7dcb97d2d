"""The device pair list is sized without reading the pair count back: each q0 has at most
Nq/2 + 8 momentum-conserving pairs (q1 and its partner fold into one pair; at most 8 q1 are
their own partner).  Checked here with the oracle's enumeration for every q0 of odd, even and
mixed meshes."""
import numpy as np
import pytest

from oracle import driver as D
from spring_b200 import synthetic as S


@pytest.mark.parametrize("mesh", [(4, 4, 4), (5, 5, 5), (6, 6, 6), (4, 5, 6), (7, 7, 7)])
def test_pairs_per_q0_within_bound(mesh):
    cr = S.build("rocksalt2")
    q_int, _, _ = D.make_tetrahedron(np.array(mesh, np.int32), cr.G)
    nq = int(np.prod(mesh))
    worst = 0
    for g in range(nq):
        _, _, cnt = D.momentum3(np.array(mesh, np.int32), q_int, q_int[g])
        worst = max(worst, cnt[0])
        assert cnt[0] <= nq // 2 + 8, (mesh, g, cnt[0])
    assert worst >= nq // 2  # the bound is tight to within the self-partner points
