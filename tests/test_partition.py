"""Host logic of the x2 / x3 domain split (canoe_b200.partition): block
configurations, neighbour maps of walled and periodic domains, and the
scatter / gather of states.  No GPU."""
import numpy as np
import pytest

from canoe_b200 import partition, problems
from canoe_b200._abi import BC_BLOCK, BC_PERIODIC, BC_REFLECT


def _c2(nx2=12, nx3=8):
    return problems.moist3d(nx1=16, nx2=nx2, nx3=nx3, x1max=2000.0, x2max=3000.0,
                            x3max=2000.0)


def test_periodic_domain_wraps_neighbours():
    p = _c2()
    assert p.cfg.bc[2] == BC_PERIODIC and p.cfg.bc[4] == BC_PERIODIC
    sp = partition.split(p, 3, 2)
    assert len(sp.blocks) == 6
    for idx, (b, nbr) in enumerate(zip(sp.blocks, sp.neighbors)):
        b2, b3 = idx % 3, idx // 3
        assert (b.cfg.nx2, b.cfg.nx3) == (4, 4)
        assert all(b.cfg.bc[q] == BC_BLOCK for q in range(2, 6))
        assert nbr == {2: b3 * 3 + (b2 - 1) % 3, 3: b3 * 3 + (b2 + 1) % 3,
                       4: ((b3 - 1) % 2) * 3 + b2, 5: ((b3 + 1) % 2) * 3 + b2}
        # x1 is never cut
        assert (b.cfg.bc[0], b.cfg.bc[1]) == (p.cfg.bc[0], p.cfg.bc[1])
        assert b.cfg.x2min == pytest.approx(p.cfg.x2min + b2 * 4 * p.cfg.dx2)


def test_walled_domain_keeps_its_walls():
    p = problems.bubble2d(nx1=20, nx2=12, x1max=200.0, x2max=120.0)
    assert p.cfg.bc[2] == BC_REFLECT
    sp = partition.split(p, 3)
    assert [sorted(n) for n in sp.neighbors] == [[3], [2, 3], [2]]
    assert sp.blocks[0].cfg.bc[2] == BC_REFLECT and sp.blocks[2].cfg.bc[3] == BC_REFLECT
    assert sp.blocks[1].cfg.bc[2] == BC_BLOCK and sp.blocks[1].cfg.bc[3] == BC_BLOCK


def test_single_block_per_direction_keeps_periodic():
    sp = partition.split(_c2(), 2, 1)
    assert all(b.cfg.bc[4] == BC_PERIODIC and b.cfg.bc[5] == BC_PERIODIC for b in sp.blocks)


def test_scatter_gather_round_trip():
    p = _c2()
    sp = partition.split(p, 4, 2)
    got = partition.gather(sp, p.u.shape, [b.u for b in sp.blocks], p.cfg.nx2, p.cfg.nx3)
    np.testing.assert_array_equal(p.interior(got), p.interior(p.u))


@pytest.mark.parametrize("nb2,nb3", [(5, 1), (1, 3), (12, 1)])
def test_rejects_uneven_or_thin_blocks(nb2, nb3):
    with pytest.raises(ValueError):
        partition.split(_c2(), nb2, nb3)
