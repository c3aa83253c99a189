"""Failure paths and particle-buffer growth, through the C-ABI, without
faulting the GPU.

* A particle found outside its tile (only reachable by moving twice without
  the tile sort) is left untouched and reported: ZPIC_E_DEVICE at the next
  synchronising call.  The reference has no such check; its corresponding
  errors print and exit(1) (particles.cpp:991-994).
* A bounded wait on the bulk copies that gives up (a poll limit of 1, far
  below a copy's latency) makes the kernel skip its work for that tile and
  report ZPIC_E_DEVICE; the copies still land before the CTA exits, so the
  context stays usable and the next step runs normally.
* Particle buffers grow instead of failing when the moving window injects
  past the capacity, as the reference's sort grows its buffers
  (particles.cpp:863-888), and when species_set hands over a larger set.
"""
import numpy as np
import pytest

from em2d_oracle import OracleSim
import zpic_b200 as zb
from helpers import same_multisets

pytestmark = pytest.mark.gpu

WEIBEL = ((8, 8), (16, 16), (12.8, 12.8), 0.07)


def weibel(sim):
    sim.add_species(-1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, 0.6)))
    sim.add_species(1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -0.6)))
    return sim


def _outside(ix, nx):
    return (ix[:, 0] < 0) | (ix[:, 0] >= nx[0]) | (ix[:, 1] < 0) | (ix[:, 1] >= nx[1])


def test_second_move_without_sort_is_reported_and_leaves_leavers_untouched():
    g = weibel(zb.Simulation(*WEIBEL))
    g.species_push(0)
    g.species_move(0)
    g.synchronize()
    npt, ix, x, u = g.particles(0)
    out = _outside(ix, WEIBEL[1])
    assert out.any(), 'some particles must have left their tile'
    g.species_move(0)
    with pytest.raises(zb.ZpicError, match='moved more than one tile'):
        g.synchronize()
    npt2, ix2, x2, u2 = g.particles(0)
    assert np.array_equal(npt, npt2)
    # the flagged particles kept their state; the others moved again
    assert np.array_equal(ix[out], ix2[out]) and np.array_equal(x[out], x2[out])
    assert not np.array_equal(x[~out], x2[~out])
    # reported once: the status word starts clean again
    g.synchronize()


def test_expired_bulk_copy_wait_skips_the_work_and_is_reported():
    g = weibel(zb.Simulation(*WEIBEL))
    before = [int(g.np_total(sp)) for sp in range(2)]
    g.set_option('wait_limit', 1)
    g.advance(1)
    with pytest.raises(zb.ZpicError, match='bounded wait expired'):
        g.synchronize()
    # tiles whose copies did not arrive in time kept their particles and
    # fields; the state stays consistent (counts, tile membership, finite)
    for sp in range(2):
        npt, ix, x, u = g.particles(sp)
        assert int(npt.sum()) == before[sp]
        assert not _outside(ix, WEIBEL[1]).any()
        assert np.isfinite(x).all() and np.isfinite(u).all()
    # the limit back to its default: steps run and nothing is reported
    g.set_option('wait_limit', 4194304)
    g.advance(2)
    g.synchronize()
    for w in 'EBJ':
        assert np.isfinite(g.grid(w)).all()


def test_invalid_wait_limit_rejected():
    g = weibel(zb.Simulation(*WEIBEL))
    with pytest.raises(zb.ZpicError, match='wait_limit'):
        g.set_option('wait_limit', 0)


def window_growth(s):
    # a cold column of plasma at the right edge: no current, no fields, every
    # step reproducible bit for bit; the window fills the box column by column
    s.add_species(-1.0, (4, 4), density=('step', 1.0, 5.4, 0))
    s.set_moving_window()
    return s


GROW = ((8, 2), (8, 8), (6.4, 1.6), 0.07)


def test_window_injection_grows_the_buffer_and_matches_the_oracle():
    o = window_growth(OracleSim(*GROW))
    g = zb.Simulation(*GROW)
    g.set_option('capacity_factor', 0.1)
    window_growth(g)
    cap0 = g.max_part(0)
    assert same_multisets(o.particles(0), g.particles(0))
    for n in (1, 10, 40, 90, 140):
        o.advance_mov_window(n - o.iter())
        g.advance_mov_window(n - g.iter())
        assert same_multisets(o.particles(0), g.particles(0)), 'step %d' % n
    # the box is full now: 64 x 16 cells x 16 ppc, more than the initial capacity
    assert g.np_total(0) == 64 * 16 * 16
    assert g.np_total(0) > cap0 and g.max_part(0) >= g.np_total(0)


def test_species_set_larger_than_the_buffer_grows_it():
    geom = ((4, 4), (16, 16), (6.4, 6.4), 0.07)
    g = zb.Simulation(*geom)
    g.set_option('capacity_factor', 0.05)
    g.add_species(-1.0, (2, 2), udist=('thermal', (0.1, 0.1, 0.1), (0, 0, 0)))
    big = OracleSim(*geom)
    big.add_species(-1.0, (6, 6), udist=('thermal', (0.1, 0.1, 0.1), (0, 0, 0)))
    state = big.particles(0)
    assert int(state[0].sum()) > g.max_part(0)
    g.set_particles(0, *state)
    assert g.max_part(0) >= int(state[0].sum())
    assert same_multisets(state, g.particles(0))
    # and it steps like the oracle from there
    big.advance(1)
    g.advance(1)
    assert same_multisets(big.particles(0), g.particles(0))


def test_batch_rebuilds_after_a_run_grows():
    geom = ((4, 4), (16, 16), (6.4, 6.4), 0.07)
    sims = []
    for k in range(2):
        s = zb.Simulation(*geom)
        s.set_option('capacity_factor', 0.05)
        s.add_species(-1.0, (2, 2), udist=('thermal', (0.1, 0.1, 0.1), (0, 0, 0)))
        sims.append(s)
    batch = zb.Batch(sims)
    batch.advance(1)
    batch.synchronize()
    o = OracleSim(*geom)
    o.add_species(-1.0, (6, 6), udist=('thermal', (0.1, 0.1, 0.1), (0, 0, 0)))
    sims[1].set_particles(0, *o.particles(0))
    assert sims[1].max_part(0) >= int(o.tiles(0)[0].sum())
    # the oracle takes the run's fields after the batch's first step, so that
    # the next step's particle update starts from the same state
    for w in 'EB':
        o.set_grid(w, sims[1].grid(w))
    batch.advance(1)
    batch.synchronize()
    o.advance(1)
    assert same_multisets(o.particles(0), sims[1].particles(0))
