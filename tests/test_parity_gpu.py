"""Parity of the CUDA em2d step against the oracle (plain-C restatement of the
reference openmp/em2d build), through the library's C-ABI.

Bars (from the reference's arithmetic):
* per-particle push and move, initial states, tile counts and per-tile
  particle multisets: bit-exact;
* the Yee solver and the current guard-cell sums on identical inputs: bit-exact;
* deposited current: FP32 summation order differs (shared atomics vs the
  reference's serial loop) -> max|dJ| <= 1e-6 * max|J|;
* multi-step energy histories: relative agreement 1e-3 (chaotic growth of
  round-off differences in an unstable plasma).
"""
import numpy as np
import pytest

from em2d_oracle import OracleSim
import zpic_b200 as zb
from helpers import same_multisets, interior_mask, rel_err, random_fields

pytestmark = pytest.mark.gpu

WEIBEL = ((8, 8), (16, 16), (12.8, 12.8), 0.07)
J_TOL = 1e-6


def weibel(sim):
    sim.add_species(-1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, 0.6)))
    sim.add_species(1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -0.6)))
    return sim


def pair(setup, geom=WEIBEL):
    return setup(OracleSim(*geom)), setup(zb.Simulation(*geom))


def test_initial_state_bit_exact():
    o, g = pair(weibel)
    for sp in range(2):
        a, b = o.particles(sp), g.particles(sp)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


def test_push_bit_exact():
    o, g = pair(weibel)
    E = random_fields(o, 1)
    B = random_fields(o, 2)
    for s in (o, g):
        s.set_grid('E', E)
        s.set_grid('B', B)
    for sp in range(2):
        o.species_push(sp)
        g.species_push(sp)
        a, b = o.particles(sp), g.particles(sp)
        assert np.array_equal(a[3], b[3]), 'momenta differ'
        assert abs(o.species_energy(sp) - g.species_energy(sp)) <= 1e-12 * abs(o.species_energy(sp))


def test_euler_push_bit_exact():
    geom = ((4, 4), (16, 16), (6.4, 6.4), 0.05)

    def setup(s):
        s.add_species(-1.0, (2, 2), udist=('thermal', (0.2, 0.1, 0.05), (0.1, 0, 0)), push_type=1)
        return s
    o, g = pair(setup, geom)
    E, B = random_fields(o, 3, 2.0), random_fields(o, 4, 5.0)
    for s in (o, g):
        s.set_grid('E', E)
        s.set_grid('B', B)
    o.species_push(0)
    g.species_push(0)
    # sinf/cosf of the exact rotation come from different math libraries: allow 2 ulp
    a, b = o.particles(0)[3], g.particles(0)[3]
    assert np.allclose(a, b, rtol=3e-7, atol=1e-7)


def test_move_deposit():
    o, g = pair(weibel)
    for s in (o, g):
        s.current_zero()
    for sp in range(2):
        o.species_move(sp)
        g.species_move(sp)
        a, b = o.particles(sp), g.particles(sp)
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]), 'positions differ'
    m = interior_mask(o)
    assert rel_err(g.grid('J')[:, m], o.grid('J')[:, m]) <= J_TOL


def test_move_deposit_fp32_tile_current():
    """Option "jacc" 0: FP32 shared atomics (the reference's FP32 sums in
    another order)."""
    o, g = pair(weibel)
    g.set_option('jacc', 0)
    for s in (o, g):
        s.current_zero()
    for sp in range(2):
        o.species_move(sp)
        g.species_move(sp)
    m = interior_mask(o)
    assert rel_err(g.grid('J')[:, m], o.grid('J')[:, m]) <= J_TOL


def test_move_deposit_fp64_tile_current():
    """Option "jacc": the tile current is summed in FP64 and rounded once per
    cell; positions stay bit-exact and the current within the FP32 bar."""
    o, g = pair(weibel)
    g.set_option('jacc', 1)
    for s in (o, g):
        s.current_zero()
    for sp in range(2):
        o.species_move(sp)
        g.species_move(sp)
        a, b = o.particles(sp), g.particles(sp)
        assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]), 'positions differ'
    m = interior_mask(o)
    assert rel_err(g.grid('J')[:, m], o.grid('J')[:, m]) <= J_TOL


def test_move_deposit_fixed_point_tile_current():
    """Option "jacc" 2 (default): fixed-point tile current in two 32-bit words.  Positions bit-exact,
    current within the FP32 bar, and with one CTA per tile and two species
    (two FP32 additions per cell onto zero, which commute) the deposited
    current is the same bit for bit on every run."""
    o = weibel(OracleSim(*WEIBEL))
    o.current_zero()
    for sp in range(2):
        o.species_move(sp)
    runs = []
    for _ in range(2):
        g = weibel(zb.Simulation(*WEIBEL))
        g.set_option('jacc', 2)
        g.set_option('chunks', 1)
        g.current_zero()
        for sp in range(2):
            g.species_move(sp)
            a, b = o.particles(sp), g.particles(sp)
            assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2]), 'positions differ'
        runs.append(g.grid('J'))
    m = interior_mask(o)
    assert rel_err(runs[0][:, m], o.grid('J')[:, m]) <= J_TOL
    assert np.array_equal(runs[0], runs[1])
    with pytest.raises(zb.ZpicError):
        g.set_option('jacc', 3)


def test_fixed_point_flush_dense_tiles():
    """65,536 particles per tile in one CTA: the fixed-point tile current is
    flushed to the raw current between groups of 20,480 particles; the
    deposited current stays within the FP32 bar of the oracle's."""
    geom = ((2, 2), (16, 16), (3.2, 3.2), 0.07)

    def setup(s):
        s.add_species(-1.0, (16, 16), udist=('thermal', (0.2, 0.2, 0.2), (0.05, 0, 0)))
        return s
    o, g = pair(setup, geom)
    g.set_option('chunks', 1)
    for s in (o, g):
        s.current_zero()
        s.species_move(0)
    assert np.array_equal(o.particles(0)[2], g.particles(0)[2])
    m = interior_mask(o)
    assert rel_err(g.grid('J')[:, m], o.grid('J')[:, m]) <= J_TOL


def test_tile_sort_multisets():
    o, g = pair(weibel)
    for s in (o, g):
        s.current_zero()
        for sp in range(2):
            s.species_move(sp)
        for sp in range(2):
            s.species_tile_sort(sp)
    for sp in range(2):
        assert same_multisets(o.particles(sp), g.particles(sp))


def test_current_advance_bit_exact():
    o, g = pair(weibel)
    rng = np.random.default_rng(5)
    raw = rng.normal(size=(64, o.tile_vol, 3)).astype(np.float32)
    for s in (o, g):
        s.current_zero()
        s.set_grid('J', raw)
        s.current_advance()
    m = interior_mask(o)
    assert np.array_equal(o.grid('J')[:, m], g.grid('J')[:, m])


def test_yee_bit_exact():
    o, g = pair(weibel)
    E, B, J = random_fields(o, 6), random_fields(o, 7), random_fields(o, 8)
    for s in (o, g):
        s.current_zero()
        s.set_grid('J', J)
        s.current_advance()
        s.set_grid('E', E)
        s.set_grid('B', B)
        s.emf_advance(True)
    m = interior_mask(o)
    for w in 'EB':
        assert np.array_equal(o.grid(w)[:, m], g.grid(w)[:, m]), w


def test_one_step():
    o, g = pair(weibel)
    o.advance(1)
    g.advance(1)
    for sp in range(2):
        assert same_multisets(o.particles(sp), g.particles(sp))
        assert abs(o.species_energy(sp) - g.species_energy(sp)) <= 1e-12 * abs(o.species_energy(sp))
    m = interior_mask(o)
    assert rel_err(g.grid('J')[:, m], o.grid('J')[:, m]) <= J_TOL
    # The field solve is bit-exact (test_yee_bit_exact), so after one step from
    # E = B = 0 the field differences must be fully explained by the current's
    # rounding differences: E = -dt J, B = -(dt/2) curl E twice.
    dt, dx, dy = WEIBEL[3], WEIBEL[2][0] / 128, WEIBEL[2][1] / 128
    eps = np.finfo(np.float32).eps
    dJ = np.abs(g.grid('J')[:, m] - o.grid('J')[:, m]).max()
    dE = np.abs(g.grid('E')[:, m] - o.grid('E')[:, m]).max()
    dB = np.abs(g.grid('B')[:, m] - o.grid('B')[:, m]).max()
    assert dE <= 1.1 * dt * dJ + 4 * eps * np.abs(o.grid('E')[:, m]).max()
    assert dB <= 1.1 * dt * (1 / dx + 1 / dy) * dE + 4 * eps * np.abs(o.grid('B')[:, m]).max()
    assert g.nmove() == o.nmove()


def test_energy_history_weibel():
    o, g = pair(weibel)
    for _ in range(10):
        o.advance(20)
        g.advance(20)
        for sp in range(2):
            assert rel_err(g.species_energy(sp), o.species_energy(sp)) <= 1e-3
        eo, bo = o.emf_energy()
        eg, bg = g.emf_energy()
        assert rel_err(eg.sum(), eo.sum()) <= 1e-3
        assert rel_err(bg.sum(), bo.sum()) <= 1e-3
    for sp in range(2):
        assert np.array_equal(o.tiles(sp)[0].sum(), g.tiles(sp)[0].sum())


def lwfa_small(s):
    s.add_species(-1.0, (4, 2), density=('step', 1.0, 2.0, 0))
    s.add_laser('gaussian', start=5.5, fwhm=1.0, a0=2.0, omega0=10.0, W0=1.5, focus=5.0, axis=3.2, sin_pol=1)
    s.set_moving_window()
    s.current_set_filter('compensated', 0, 2)
    return s


LWFA = ((16, 4), (16, 16), (256 * 0.025, 64 * 0.1), 0.022)


def test_moving_window_laser():
    o, g = pair(lwfa_small, LWFA)
    m = interior_mask(o)
    for w in 'EB':
        assert np.array_equal(o.grid(w)[:, m], g.grid(w)[:, m]), 'laser fields ' + w
    o.advance_mov_window(1)
    g.advance_mov_window(1)
    assert same_multisets(o.particles(0), g.particles(0))
    for n in (30, 60):
        o.advance_mov_window(n - o.iter())
        g.advance_mov_window(n - g.iter())
        eo, bo = o.emf_energy()
        eg, bg = g.emf_energy()
        assert rel_err(eg.sum(), eo.sum()) <= 1e-3
        assert rel_err(bg.sum(), bo.sum()) <= 1e-3
        # the step after n, from the same state (the oracle continues from the
        # library's particles, fields and clocks): the window's move, the
        # injected column and the sort must agree particle for particle
        c = lwfa_small(OracleSim(*LWFA))
        c.set_particles(0, *g.particles(0))
        for w in 'EB':
            c.set_grid(w, g.grid(w))
        c.set_clock(n)
        c.advance_mov_window(1)
        g.advance_mov_window(1)
        assert np.array_equal(c.tiles(0)[0], g.tiles(0)[0]), 'step %d tile counts' % (n + 1)
        assert same_multisets(c.particles(0), g.particles(0)), 'step %d particles' % (n + 1)
        o.advance_mov_window(1)


def walls(s):
    s.add_species(-1.0, (2, 3), density=('slab', 1.0, 1.0, 5.0, 1),
                  udist=('thermal', (0.2, 0.1, 0.05), (0.1, 0, 0)), bc=(2, 2, 2, 2))
    s.add_species(2.0, (3, 2), density=('sphere', 0.5, 3.2, 3.2, 2.0),
                  udist=('thermalcorr', (0.05, 0.2, 0.1), (0, 0.2, 0), 3), bc=(2, 2, 2, 2))
    s.emf_set_bc((2, 3, 3, 2))
    s.current_set_bc((2, 2, 2, 2))
    s.current_set_filter('binomial', 1, 2)
    s.add_laser('plane', start=3.0, fwhm=1.0, a0=1.0, omega0=5.0, polarization=0.3)
    return s


def test_walls_filters_profiles():
    geom = ((4, 4), (16, 16), (6.4, 6.4), 0.05)
    o, g = pair(walls, geom)
    for sp in range(2):
        assert same_multisets(o.particles(sp), g.particles(sp))
    o.advance(1)
    g.advance(1)
    for sp in range(2):
        assert same_multisets(o.particles(sp), g.particles(sp))
    o.advance(40)
    g.advance(40)
    for sp in range(2):
        assert o.tiles(sp)[0].sum() == g.tiles(sp)[0].sum()
        assert rel_err(g.species_energy(sp), o.species_energy(sp)) <= 1e-3


def test_diagnostics_charge_and_phasespace():
    """Charge density and 1D / 2D phase spaces (Species::deposit_charge,
    Species::dep_phasespace) after 20 steps.  Against the oracle evaluated on
    the same particles: FP32 sums in another order, max|d| <= 1e-5 * max|ref|.
    Against the reference's committed fixtures (its own trajectory, which
    differs by the current's rounding): max|d| <= 1e-3 * max|ref|."""
    import os
    import sys
    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')
    sys.path.insert(0, gold)
    from make_golden import PHASESPACES
    g = np.load(os.path.join(gold, 'diagnostics_small.npz'))
    s = weibel(zb.Simulation(*WEIBEL))
    s.advance(20)
    o = weibel(OracleSim(*WEIBEL))
    for sp in range(2):
        o.set_particles(sp, *s.particles(sp))

    def close(got, ref, tol):
        assert got.shape == ref.shape
        return np.abs(got.astype(np.float64) - ref).max() <= tol * np.abs(ref).max()
    for sp in range(2):
        got = s.charge(sp)
        assert close(got, o.charge(sp), 1e-5) and close(got, g['charge%d' % sp], 1e-3)
        for k, c in enumerate(PHASESPACES):
            got = s.phasespace(sp, *c)
            assert close(got, o.phasespace(sp, *c), 1e-5), (sp, c)
            assert close(got, g['pha%d_%d' % (sp, k)], 1e-3), (sp, c)
    with pytest.raises(zb.ZpicError):
        s.phasespace(0, 'ux', (-1, 1), 10, 'x', (0, 12.8), 10)     # 2D needs quant1 > quant0
    # a large phase space goes through global atomics instead of a shared copy
    big = s.phasespace(0, 'x', (0.0, 12.8), 256, 'uz', (-1.5, 1.5), 256)
    assert close(big, o.phasespace(0, 0, (0.0, 12.8), 256, 4, (-1.5, 1.5), 256), 1e-5)


def test_weibel_growth_rate():
    """Weibel growth rate from the magnetic energy history: the exponential
    rate fitted over the linear phase agrees with the oracle's within 1e-3."""
    o, g = pair(weibel)
    eb_o, eb_g = [], []
    for _ in range(250):
        o.advance(1)
        g.advance(1)
        eb_o.append(o.emf_energy()[1].sum())
        eb_g.append(g.emf_energy()[1].sum())
    eb_o, eb_g = np.log(np.array(eb_o)), np.log(np.array(eb_g))
    # growth phase: steps 30 to 230 (log E_B rises by ~7 e-folds, with the
    # plasma oscillation on top, the same in both histories)
    sel = np.arange(30, 230)
    t = (sel + 1) * WEIBEL[3]
    rate_o = np.polyfit(t, eb_o[sel], 1)[0]
    rate_g = np.polyfit(t, eb_g[sel], 1)[0]
    assert rate_o > 0
    assert abs(rate_g - rate_o) <= 1e-3 * rate_o


def test_moving_window_graph_replay():
    """Moving-window steps replayed from CUDA graphs (one per pattern of window
    moves) against the same steps issued one by one: same particle counts per
    tile, energies equal up to FP32 summation order."""
    a = lwfa_small(zb.Simulation(*LWFA))
    b = lwfa_small(zb.Simulation(*LWFA))
    b.set_option('graph', 0)
    for n in range(1, 81):
        a.advance_mov_window(1 if n < 40 else 2)
        b.advance_mov_window(1 if n < 40 else 2)
        if a.iter() >= 80:
            break
    assert a.iter() == b.iter()
    assert np.array_equal(a.tiles(0)[0], b.tiles(0)[0])
    ea, eb = a.emf_energy(), b.emf_energy()
    assert rel_err(a.species_energy(0), b.species_energy(0)) <= 1e-5
    assert rel_err(ea[0].sum() + ea[1].sum(), eb[0].sum() + eb[1].sum()) <= 1e-5


def test_window_shift_after_field_solve_bit_exact():
    """In a moving-window step the window shift takes over the field solve's
    guard-cell refresh (the Yee kernel keeps B's first interior column for
    it).  Fields, guard cells included, must be bit for bit those of the
    field solve and the shift issued one after the other with their own guard
    refreshes (EMF::advance through emf_advance), over steps with and without
    a move; random E and B, no particles (zero current)."""
    geom = ((8, 4), (16, 16), (128 * 0.025, 64 * 0.1), 0.022)
    a, b = zb.Simulation(*geom), zb.Simulation(*geom)
    E, B = random_fields(a, 11), random_fields(a, 12)
    for s in (a, b):
        s.set_moving_window()
        s.set_grid('E', E)
        s.set_grid('B', B)
    for n in range(8):
        a.advance_mov_window(1)
        b.emf_advance(True)
        for w in 'EB':
            assert np.array_equal(a.grid(w), b.grid(w)), 'step %d, %s' % (n + 1, w)


@pytest.mark.parametrize('nx, chunks', [((8, 8), 0), ((32, 32), 0), ((16, 16), -1), ((24, 8), 3)])
def test_tile_shapes_and_chunking(nx, chunks):
    """Tile shapes other than the compile-time 16x16 one, and the CTA
    chunkings: 10 steps of the Weibel set-up (128x128 cells) against the
    oracle -- per-tile counts and multisets after one step, energies after
    ten."""
    geom = ((128 // nx[0], 128 // nx[1]), nx, (12.8, 12.8), 0.07)
    o, g = pair(weibel, geom)
    g.set_option('chunks', chunks)
    o.advance(1)
    g.advance(1)
    for sp in range(2):
        assert np.array_equal(o.tiles(sp)[0], g.tiles(sp)[0])
        assert same_multisets(o.particles(sp), g.particles(sp))
    m = interior_mask(o)
    assert rel_err(g.grid('J')[:, m], o.grid('J')[:, m]) <= J_TOL
    o.advance(9)
    g.advance(9)
    for sp in range(2):
        assert rel_err(g.species_energy(sp), o.species_energy(sp)) <= 1e-5
    eo, bo = o.emf_energy()
    eg, bg = g.emf_energy()
    assert rel_err(eg.sum(), eo.sum()) <= 1e-5
