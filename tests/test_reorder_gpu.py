"""In-tile reorder (option "reorder"): it changes only the order of the
particles inside each tile.  A reorder keeps every tile's particle multiset
bit for bit, and right after it each tile lists its particles in cell
round-robin order.  Later steps stay on the same trajectory up to the FP32
order of the per-CTA additions into the global current (CTAs per tile and
species add their tile currents in any order), as with any other change of
particle order."""
import numpy as np
import pytest

import zpic_b200 as zb
from helpers import same_multisets, rel_err

pytestmark = pytest.mark.gpu

GEOM = ((4, 4), (16, 16), (6.4, 6.4), 0.07)


def weibel(s):
    s.add_species(-1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, 0.6)))
    s.add_species(1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -0.6)))
    return s


def energies(s):
    e, b = s.emf_energy()
    return np.array([s.species_energy(0), s.species_energy(1), e.sum(), b.sum()])


def test_reorder_keeps_particles():
    a, b = weibel(zb.Simulation(*GEOM)), weibel(zb.Simulation(*GEOM))
    b.set_option('reorder', 1)
    a.advance(1)
    b.advance(1)                       # step 1, then a reorder
    for sp in range(2):
        assert same_multisets(a.particles(sp), b.particles(sp))
    a.advance(30)
    b.advance(30)
    assert rel_err(energies(b), energies(a)) <= 1e-4
    for sp in range(2):
        assert b.np_total(sp) == a.np_total(sp) == 64 * 64 * 16
    with pytest.raises(zb.ZpicError):
        a.set_option('reorder', -1)


@pytest.mark.parametrize('nx, ppc', [((16, 16), (4, 4)), ((16, 16), (9, 9)), ((32, 32), (2, 2))])
def test_reorder_round_robin_order(nx, ppc):
    """Both launch forms: two 512-thread CTAs per SM for 16x16 tiles that fit
    half of the shared memory, one 1024-thread CTA for larger tiles (16x16
    cells at 81 per cell: 20,736 particles) and for tiles of more cells."""
    geom = ((64 // nx[0], 64 // nx[1]), nx, (6.4, 6.4), 0.07)
    s = zb.Simulation(*geom)
    s.add_species(-1.0, ppc, udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, 0.6)))
    s.add_species(1.0, ppc, udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -0.6)))
    s.set_option('reorder', 5)
    s.advance(5)                       # the last thing step 5 does is a reorder
    for sp in range(2):
        npt, ix, x, u = s.particles(sp)
        assert int(npt.max()) > 64
        o = 0
        for n in npt:
            cell = ix[o:o + n, 0] + nx[0] * ix[o:o + n, 1]
            counts = np.bincount(cell, minlength=nx[0] * nx[1])
            # round r holds one particle of each cell with more than r
            # particles, in ascending cell order
            k = 0
            for r in range(counts.max()):
                cells_r = np.nonzero(counts > r)[0]
                assert np.array_equal(cell[k:k + len(cells_r)], cells_r)
                k += len(cells_r)
            assert k == n
            o += n


def test_reorder_moving_window():
    """Moving-window steps (graph replays and eager steps) reorder too."""
    def lwfa(s):
        s.add_species(-1.0, (4, 2), density=('step', 1.0, 2.0, 0))
        s.add_laser('gaussian', start=5.5, fwhm=1.0, a0=2.0, omega0=10.0, W0=1.5, focus=5.0, axis=3.2, sin_pol=1)
        s.set_moving_window()
        return s
    geom = ((16, 4), (16, 16), (256 * 0.025, 64 * 0.1), 0.022)
    a, b = lwfa(zb.Simulation(*geom)), lwfa(zb.Simulation(*geom))
    b.set_option('reorder', 1)
    a.advance_mov_window(1)
    b.advance_mov_window(1)
    assert same_multisets(a.particles(0), b.particles(0))
    b.set_option('reorder', 4)
    a.advance_mov_window(59)
    b.advance_mov_window(59)
    assert a.np_total(0) == b.np_total(0)
    ea, eb = a.emf_energy(), b.emf_energy()
    assert rel_err(eb[0].sum(), ea[0].sum()) <= 1e-4
    assert rel_err(b.species_energy(0), a.species_energy(0)) <= 1e-4


def test_reorder_skips_tiles_beyond_shared_memory():
    """32x32 tiles holding 65,536 particles each do not fit the reorder's
    shared-memory permutation: they keep their order, and nothing changes."""
    geom = ((2, 2), (32, 32), (6.4, 6.4), 0.07)

    def dense(s):
        s.add_species(-1.0, (8, 8), udist=('thermal', (0.05, 0.05, 0.05), (0, 0, 0)))
        return s
    a, b = dense(zb.Simulation(*geom)), dense(zb.Simulation(*geom))
    b.set_option('reorder', 1)
    a.advance(1)
    b.advance(1)
    assert same_multisets(a.particles(0), b.particles(0))
    assert b.np_total(0) == 64 * 64 * 64
