"""Pins the oracle (plain-C restatement, oracle/em2d_oracle.c) to the reference.

* against the committed golden fixtures (outputs of the reference's own
  openmp/em2d build, tests/golden/make_golden.py): bit-exact;
* against the reference build itself (oracle/_ref, one OpenMP thread) when it
  is present: bit-exact over many steps on every exercised path.
"""
import os

import numpy as np
import pytest

from em2d_oracle import OracleSim, RefSim, ref_available

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
needs_ref = pytest.mark.skipif(not ref_available('scalar'), reason='reference build oracle/_ref not present')


def weibel(sim, ppc=(4, 4)):
    sim.add_species(-1.0, ppc, udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, 0.6)))
    sim.add_species(1.0, ppc, udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -0.6)))
    return sim


def energies(sim):
    e, b = sim.emf_energy()
    return np.array([sim.species_energy(k) for k in range(sim.nsp)] + list(e) + list(b))


def assert_same_state(a, b, mask_pad=True):
    for sp in range(a.nsp):
        for x, y in zip(a.particles(sp), b.particles(sp)):
            assert np.array_equal(x, y)
    n = a.ext[0] * a.ext[1]
    for w in 'EBJ':
        assert np.array_equal(a.grid(w)[:, :n], b.grid(w)[:, :n]), w


# ---- golden fixtures ----
def test_golden_weibel_small_state_and_history():
    g = np.load(os.path.join(GOLD, 'weibel_small.npz'))
    o = weibel(OracleSim((4, 4), (8, 8), (3.2, 3.2), 0.07), (2, 2))
    n = o.ext[0] * o.ext[1]

    def check(tag):
        for sp in range(2):
            npt, ix, x, u = o.particles(sp)
            assert np.array_equal(npt, g['%s_np%d' % (tag, sp)])
            assert np.array_equal(ix, g['%s_ix%d' % (tag, sp)])
            assert np.array_equal(x, g['%s_x%d' % (tag, sp)])
            assert np.array_equal(u, g['%s_u%d' % (tag, sp)])
        for w in 'EBJ':
            assert np.array_equal(o.grid(w)[:, :n], g['%s_%s' % (tag, w)][:, :n]), w
    check('s0')
    hist = [energies(o)]
    for k in range(1, 41):
        o.advance(1)
        if k == 5:
            check('s5')
        hist.append(energies(o))
    assert np.array_equal(np.array(hist), g['energy'])


def test_golden_weibel_energy_history():
    g = np.load(os.path.join(GOLD, 'weibel_energy.npz'))
    o = weibel(OracleSim((8, 8), (16, 16), (12.8, 12.8), 0.07))
    hist = [energies(o)]
    for _ in range(20):              # first 200 steps of the 500 in the fixture
        o.advance(10)
        hist.append(energies(o))
    assert np.array_equal(np.array(hist), g['energy'][:21])


def lwfa_small(s):
    s.add_species(-1.0, (4, 2), density=('step', 1.0, 2.0, 0))
    s.add_laser('gaussian', start=5.5, fwhm=1.0, a0=2.0, omega0=10.0, W0=1.5, focus=5.0, axis=3.2, sin_pol=1)
    s.set_moving_window()
    s.current_set_filter('compensated', 0, 2)
    return s


def test_golden_lwfa_small():
    g = np.load(os.path.join(GOLD, 'lwfa_small.npz'))
    o = lwfa_small(OracleSim((16, 4), (16, 16), (256 * 0.025, 64 * 0.1), 0.022))
    hist, counts = [energies(o)], [o.tiles(0)[0].sum()]
    for _ in range(12):
        o.advance_mov_window(10)
        hist.append(energies(o))
        counts.append(o.tiles(0)[0].sum())
    assert np.array_equal(np.array(counts), g['np_total'])
    assert np.array_equal(np.array(hist), g['energy'])


def test_golden_diagnostics():
    """Charge density and phase spaces of the oracle against the reference's
    (Species::deposit_charge, Species::dep_phasespace) after 20 steps."""
    import sys
    sys.path.insert(0, GOLD)
    from make_golden import PHASESPACES
    g = np.load(os.path.join(GOLD, 'diagnostics_small.npz'))
    o = weibel(OracleSim((8, 8), (16, 16), (12.8, 12.8), 0.07))
    o.advance(20)
    for sp in range(2):
        assert np.array_equal(o.charge(sp), g['charge%d' % sp])
        for k, c in enumerate(PHASESPACES):
            assert np.array_equal(o.phasespace(sp, *c), g['pha%d_%d' % (sp, k)]), (sp, c)


# ---- live reference build ----
@needs_ref
def test_pin_weibel_live():
    geom = ((8, 8), (16, 16), (12.8, 12.8), 0.07)
    o, r = weibel(OracleSim(*geom)), weibel(RefSim(*geom, threads=1))
    assert_same_state(o, r)
    for n in (1, 24):
        o.advance(n)
        r.advance(n)
        assert_same_state(o, r)
        assert np.array_equal(energies(o), energies(r))


def walls(s):
    s.add_species(-1.0, (2, 3), density=('slab', 1.0, 1.0, 5.0, 1),
                  udist=('thermal', (0.2, 0.1, 0.05), (0.1, 0, 0)), push_type=1, bc=(2, 2, 2, 2))
    s.add_species(2.0, (3, 2), density=('sphere', 0.5, 3.2, 3.2, 2.0),
                  udist=('thermalcorr', (0.05, 0.2, 0.1), (0, 0.2, 0), 3), bc=(2, 2, 2, 2))
    s.emf_set_bc((2, 3, 3, 2))
    s.current_set_bc((2, 2, 2, 2))
    s.current_set_filter('binomial', 1, 2)
    s.add_laser('plane', start=3.0, fwhm=1.0, a0=1.0, omega0=5.0, polarization=0.3)
    return s


@needs_ref
def test_pin_walls_profiles_filters_live():
    geom = ((4, 4), (16, 16), (6.4, 6.4), 0.05)
    o, r = walls(OracleSim(*geom)), walls(RefSim(*geom, threads=1))
    assert_same_state(o, r)
    o.advance(60)
    r.advance(60)
    assert_same_state(o, r)


@needs_ref
def test_pin_moving_window_live():
    geom = ((16, 4), (16, 16), (256 * 0.025, 64 * 0.1), 0.022)
    o, r = lwfa_small(OracleSim(*geom)), lwfa_small(RefSim(*geom, threads=1))
    assert_same_state(o, r)
    o.advance_mov_window(60)
    r.advance_mov_window(60)
    assert_same_state(o, r)


@needs_ref
def test_pin_fine_grained_calls_live():
    """push / move / sort / current / field calls one at a time (simulation.h:90-107)."""
    geom = ((4, 4), (16, 16), (6.4, 6.4), 0.07)
    o, r = weibel(OracleSim(*geom), (2, 2)), weibel(RefSim(*geom, threads=1), (2, 2))
    for s in (o, r):
        s.advance(3)
        s.current_zero()
        for sp in range(2):
            s.species_push(sp)
            s.species_move(sp)
            s.species_process_bc(sp)
            s.species_tile_sort(sp)
        s.current_advance()
        s.emf_advance(True)
    assert_same_state(o, r)


def test_fp64_oracle_tracks_fp32():
    """The FP64 build of the same path, started from the FP32 initial state,
    stays within FP32 round-off growth of the FP32 run over 50 steps."""
    geom = ((4, 4), (16, 16), (6.4, 6.4), 0.07)
    o32 = weibel(OracleSim(*geom), (2, 2))
    o64 = weibel(OracleSim(*geom, real='f64'), (2, 2))
    for sp in range(2):
        npt, ix, x, u = o32.particles(sp)
        o64.set_particles(sp, npt, ix, x.astype(np.float64), u.astype(np.float64))
    o32.advance(50)
    o64.advance(50)
    e32, e64 = energies(o32), energies(o64)
    assert np.all(np.abs(e32[:2] - e64[:2]) <= 1e-4 * np.abs(e64[:2]))


def test_oracle_continues_from_a_taken_state():
    """set_clock (with set_particles / set_grid) restarts the oracle at step k
    exactly where its own uninterrupted run stands: the next steps agree bit
    for bit, across window moves (the check the GPU parity tests rely on
    when they continue the oracle from the library's state)."""
    geom = ((16, 4), (16, 16), (256 * 0.025, 64 * 0.1), 0.022)
    run = lwfa_small(OracleSim(*geom))
    for k in (7, 20, 41):
        run.advance_mov_window(k - run.iter())
        cont = lwfa_small(OracleSim(*geom))
        for sp in range(run.nsp):
            cont.set_particles(sp, *run.particles(sp))
        for w in 'EB':
            cont.set_grid(w, run.grid(w))
        cont.set_clock(k)
        assert cont.iter() == k
        for s in (run, cont):
            s.advance_mov_window(3)
        assert_same_state(run, cont)
    w = weibel(OracleSim((4, 4), (16, 16), (6.4, 6.4), 0.07), (2, 2))
    w.advance(5)
    c = weibel(OracleSim((4, 4), (16, 16), (6.4, 6.4), 0.07), (2, 2))
    for sp in range(2):
        c.set_particles(sp, *w.particles(sp))
    for g in 'EB':
        c.set_grid(g, w.grid(g))
    c.set_clock(5)
    w.advance(2)
    c.advance(2)
    assert_same_state(w, c)
