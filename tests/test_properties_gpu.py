"""Size-independent properties of the CUDA step at the benchmark's full size
(2048x2048 cells, 8x8 ppc, 268M particles) and of the sort's repack path."""
import numpy as np
import pytest

from em2d_oracle import OracleSim
import zpic_b200 as zb
from helpers import same_multisets

pytestmark = pytest.mark.gpu


def continuity_residual(rho0, rho1, J, sim, dt):
    """max |(rho1-rho0)/dt + div J| with the deposit's staggering (backward differences)."""
    ntx, nty = sim.ntiles
    nxx, nxy = sim.nx
    ex, ey = sim.ext
    dense = np.zeros((nty * nxy, ntx * nxx, 2))
    for ty in range(nty):
        for tx in range(ntx):
            blk = J[ty * ntx + tx][:ex * ey].reshape(ey, ex, 3)
            dense[ty * nxy:(ty + 1) * nxy, tx * nxx:(tx + 1) * nxx] = blk[1:1 + nxy, 1:1 + nxx, :2]
    dx = sim.box[0] / (ntx * nxx)
    dy = sim.box[1] / (nty * nxy)
    div = (dense[..., 0] - np.roll(dense[..., 0], 1, axis=1)) / dx + \
          (dense[..., 1] - np.roll(dense[..., 1], 1, axis=0)) / dy
    drho = (rho1.astype(np.float64) - rho0.astype(np.float64)) / dt
    return np.abs(drho + div).max(), np.abs(drho).max()


@pytest.fixture(scope='module')
def big():
    s = zb.Simulation((128, 128), (16, 16), (204.8, 204.8), 0.07)
    s.add_species(-1.0, (8, 8), udist=('thermal', (0.05, 0.05, 0.05), (0, 0, 0)))
    s.advance(3)
    return s


def test_full_size_charge_conservation(big):
    rho0 = big.charge(0)
    big.advance(1)
    rho1 = big.charge(0)
    res, scale = continuity_residual(rho0, rho1, big.grid('J'), big, 0.07)
    # FP32 sums of ~64 particles x 3 contributions per cell
    assert res <= 1e-4 * scale + 1e-4


def test_full_size_invariants(big):
    """Particles::validate (particles.cpp:961-1045): counts conserved (periodic),
    cells inside the tile, positions in [-0.5, 0.5), finite momenta."""
    assert big.np_total(0) == 2048 * 2048 * 64
    npt, ix, x, u = big.particles(0)
    assert npt.sum() == 2048 * 2048 * 64
    assert ix.min() >= 0 and ix.max() < 16
    assert x.min() >= -0.5 and x.max() < 0.5
    assert np.isfinite(u).all()
    assert big.np_max_tile(0) == npt.max()


@pytest.mark.parametrize('capacity', [None, 0.3])
def test_relocation_and_repack_free_streaming(capacity):
    """A drifting slab fills empty tiles beyond their spare room: such tiles
    move into the free pool at the end of the buffer (relocation), and with
    little capacity the pool runs out and the whole layout is rebuilt
    (repack).  Free streaming keeps every particle bit-exact, so tile counts
    and multisets must match the oracle exactly."""
    geom = ((8, 4), (16, 16), (12.8, 6.4), 0.07)

    def setup(s):
        s.add_species(-1.0, (4, 4), density=('slab', 1.0, 0.5, 3.0, 0),
                      udist=('thermal', (0.05, 0.05, 0.05), (0.9, 0.0, 0.0)))
        return s
    o = setup(OracleSim(*geom))
    g = zb.Simulation(*geom)
    if capacity is not None:
        g.set_option('capacity_factor', capacity)
    setup(g)
    occupied0 = set(np.nonzero(o.tiles(0)[0])[0])
    for n in range(1, 121):
        o.species_advance_free(0)
        g.species_advance(0, zb.ADVANCE_FREE)
        if n % 20 == 0:
            assert same_multisets(o.particles(0), g.particles(0)), 'step %d' % n
    # the slab moved into tiles that were empty at the start
    assert set(np.nonzero(o.tiles(0)[0])[0]) - occupied0
    assert g.relocations(0) > 0
    if capacity is not None:
        assert g.repacks(0) > 0


@pytest.mark.parametrize('ntiles,bc', [
    ((1, 1), (1, 1, 1, 1)), ((2, 1), (1, 1, 1, 1)), ((1, 2), (1, 1, 1, 1)), ((3, 5), (1, 1, 1, 1)),
    ((3, 5), (0, 0, 1, 1)), ((4, 3), (0, 0, 0, 0)), ((4, 3), (1, 1, 0, 0)),
])
def test_sort_geometries_free_streaming(ntiles, bc):
    """The tile sort on a hot plasma (many leavers, diagonal ones included)
    for tilings where a tile is its own neighbour (1 tile along an axis) or
    two directions lead to the same neighbour (2 tiles), with periodic and
    open edges: free streaming keeps every particle bit-exact, so the
    per-tile multisets must match the oracle's at every step."""
    geom = (ntiles, (8, 8), (ntiles[0] * 0.8, ntiles[1] * 0.8), 0.05)

    def setup(s):
        s.add_species(-1.0, (3, 2), udist=('thermal', (0.4, 0.3, 0.1), (0.2, -0.1, 0.0)), bc=bc)
        return s
    o, g = setup(OracleSim(*geom)), setup(zb.Simulation(*geom))
    for n in range(1, 31):
        o.species_advance_free(0)
        g.species_advance(0, zb.ADVANCE_FREE)
        assert same_multisets(o.particles(0), g.particles(0)), 'step %d' % n
    if bc[0] == 0:
        assert o.tiles(0)[0].sum() < 64 * ntiles[0] * ntiles[1] * 6   # particles left through open edges
