"""Parity at the benchmark configurations' own sizes, through the C-ABI.

* Uniform warm plasma (2048^2 cells, 16x16 tiles, 8x8 ppc, Thermal uth 0.05):
  the initial state at the full size, bit for bit; the same workload on a
  512^2 box (16.8 M particles) stepped against the oracle.
* Laser wakefield with a moving window at the full 4096x512 size (13.5 M
  particles): initial particles and Gaussian-laser fields bit for bit, step
  parity at steps 1, 101, 102 and 501, and the free-running run against the
  reference's own openmp/em2d build at steps 100 and 500.
* Members of the 256-run Weibel ensemble, advanced inside a Batch, against
  the oracle (step parity) and the reference build (energies after 100 steps).
* The Weibel set-up with two electron species, as the benchmark states it,
  and the reference driver's electron/positron variant: energy
  histories and the Weibel growth rate over 500 steps.

Step parity after step 1 re-anchors: the oracle takes the library's state at
step k (particles, E, B and every clock, window moves included) and both take
step k+1.  The deposited current differs from the oracle's by FP32 summation
order only, so free-running trajectories drift apart at round-off level; a
re-anchored step compares one step's arithmetic exactly at any point of the
run.  Bars:
* particle multisets per tile after a step: bit-exact;
* J: max|dJ| <= 1e-6 max|J|, E and B differences explained by dJ;
* energy histories and growth rates: 1e-3 relative.
"""
import numpy as np
import pytest

from em2d_oracle import OracleSim, RefSim, ref_available
import zpic_b200 as zb
from helpers import same_multisets, interior_mask, rel_err, multiset_mismatch_tiles

pytestmark = pytest.mark.gpu

J_TOL = 1e-6
EPS = np.finfo(np.float32).eps


def plasma(s):
    """The uniform warm plasma's species: electrons, 8x8 ppc, Thermal uth 0.05, ufl 0."""
    s.add_species(-1.0, (8, 8), udist=('thermal', (0.05, 0.05, 0.05), (0, 0, 0)))
    return s


def plasma_geom(ncell):
    nt = ncell // 16
    return ((nt, nt), (16, 16), (ncell * 0.1, ncell * 0.1), 0.07)


def lwfa(s):
    """Laser wakefield: 4x2 ppc behind a density step at x = 20, cold; Gaussian
    pulse a0 2, omega0 10, W0 4, fwhm 2 (start 17, focus 20, axis 25.6, Ez);
    moving window; no current filter."""
    s.add_species(-1.0, (4, 2), density=('step', 1.0, 20.0, 0))
    s.add_laser('gaussian', start=17.0, fwhm=2.0, a0=2.0, omega0=10.0, W0=4.0, focus=20.0, axis=25.6, sin_pol=1)
    s.set_moving_window()
    return s


LWFA = ((256, 32), (16, 16), (4096 * 0.025, 512 * 0.1), 0.022)


def weibel(literal):
    def setup(s):
        s.add_species(-1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, 0.6)))
        s.add_species(-1.0 if literal else 1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -0.6)))
        return s
    return setup


WEIBEL = ((8, 8), (16, 16), (12.8, 12.8), 0.07)


def ensemble_member(n, p, uz, uth):
    geom = ((n // 16, n // 16), (16, 16), (n * 0.1, n * 0.1), 0.07)

    def setup(s):
        s.add_species(-1.0, (p, p), udist=('thermalcorr', (uth, uth, uth), (0, 0, uz)))
        s.add_species(1.0, (p, p), udist=('thermalcorr', (uth, uth, uth), (0, 0, -uz)))
        return s
    return geom, setup


# ---------------------------------------------------------------------------
def reanchor(o, g, k):
    """The oracle continues from the library's state at step k."""
    for sp in range(o.nsp):
        o.set_particles(sp, *g.particles(sp))
    for w in 'EB':
        o.set_grid(w, g.grid(w))
    o.set_clock(k)


def step_and_compare(o, g, geom, moving_window=False, what=''):
    """One step on both; particles bit-exact per tile, J within the FP32 bar,
    fields explained by the current's rounding differences."""
    if moving_window:
        o.advance_mov_window(1)
        g.advance_mov_window(1)
    else:
        o.advance(1)
        g.advance(1)
    for sp in range(o.nsp):
        a, b = o.particles(sp), g.particles(sp)
        assert same_multisets(a, b), '%s: species %d particles differ (tiles %s)' % (
            what, sp, multiset_mismatch_tiles(a, b)[:8])
        eo, eg = o.species_energy(sp), g.species_energy(sp)
        assert abs(eo - eg) <= 1e-12 * abs(eo) + 1e-300, '%s: kinetic energy' % what
    m = interior_mask(o)
    Jo, Jg = o.grid('J')[:, m], g.grid('J')[:, m]
    assert rel_err(Jg, Jo) <= J_TOL, '%s: current' % what
    (ntx, nty), (nxx, nxy), (bx, by), dt = geom
    dx, dy = bx / (ntx * nxx), by / (nty * nxy)
    dJ = np.abs(Jg - Jo).max()
    Eo, Bo = o.grid('E')[:, m], o.grid('B')[:, m]
    dE = np.abs(g.grid('E')[:, m] - Eo).max()
    dB = np.abs(g.grid('B')[:, m] - Bo).max()
    assert dE <= 1.1 * dt * dJ + 4 * EPS * np.abs(Eo).max(), '%s: E' % what
    assert dB <= 1.1 * dt * (1 / dx + 1 / dy) * dE + 4 * EPS * np.abs(Bo).max(), '%s: B' % what


def same_initial_state(o, g, nsp):
    for sp in range(nsp):
        for a, b in zip(o.particles(sp), g.particles(sp)):
            assert np.array_equal(a, b), 'initial particles of species %d' % sp


def energies(s):
    e, b = s.emf_energy()
    return np.array([s.species_energy(sp) for sp in range(s.nsp)] + [e.sum(), b.sum()])


def _enough_host_memory(gb):
    try:
        import psutil
        return psutil.virtual_memory().available >= gb * 2**30
    except Exception:
        return True


# ---------------------------------------------------------------------------
# Uniform warm plasma
# ---------------------------------------------------------------------------
def test_uniform_plasma_512_initial_state_and_steps():
    geom = plasma_geom(512)
    o, g = plasma(OracleSim(*geom)), plasma(zb.Simulation(*geom))
    same_initial_state(o, g, 1)
    step_and_compare(o, g, geom, what='step 1')
    for k in range(1, 5):
        reanchor(o, g, k)
        step_and_compare(o, g, geom, what='step %d' % (k + 1))
    assert g.nmove() == 5 * g.np_total(0)


def test_uniform_plasma_2048_initial_state_bit_exact():
    """The benchmark's own 268,435,456-particle initial state, every tile."""
    if not _enough_host_memory(48):
        pytest.skip('needs ~48 GB of host memory for the oracle and the two copies')
    geom = plasma_geom(2048)
    g = plasma(zb.Simulation(*geom))
    gs = g.particles(0)
    g.close()
    o = plasma(OracleSim(*geom))
    os_ = o.particles(0)
    o.close()
    assert int(gs[0].sum()) == 2048 * 2048 * 64
    for a, b in zip(os_, gs):
        assert np.array_equal(a, b)


# ---------------------------------------------------------------------------
# Laser wakefield, moving window, full size
# ---------------------------------------------------------------------------
def test_lwfa_full_size_initial_state_and_step_parity():
    o, g = lwfa(OracleSim(*LWFA)), lwfa(zb.Simulation(*LWFA))
    same_initial_state(o, g, 1)
    m = interior_mask(o)
    for w in 'EB':
        assert np.array_equal(o.grid(w)[:, m], g.grid(w)[:, m]), 'laser field ' + w
    step_and_compare(o, g, LWFA, True, 'step 1')
    for k in (100, 101, 500):
        g.advance_mov_window(k - g.iter())
        reanchor(o, g, k)
        step_and_compare(o, g, LWFA, True, 'step %d' % (k + 1))
        # window position and injection bookkeeping continue identically
        assert np.array_equal(o.tiles(0)[0], g.tiles(0)[0]), 'step %d tile counts' % (k + 1)


@pytest.mark.skipif(not ref_available('avx2'), reason='reference build oracle/_ref missing')
def test_lwfa_full_size_free_running_against_reference_build():
    """The wakefield run compared at steps 100 and 500 with the reference's
    own openmp/em2d build (all host threads).  The two runs sum the current
    in different orders, so their trajectories drift apart at round-off
    level: energies agree to 1e-3 and the per-tile counts agree in all but a
    few tiles."""
    r, g = lwfa(RefSim(*LWFA, variant='avx2')), lwfa(zb.Simulation(*LWFA))
    for k in (100, 500):
        r.advance_mov_window(k - r.iter())
        g.advance_mov_window(k - g.iter())
        er, eg = energies(r), energies(g)
        assert np.all(np.abs(eg - er) <= 1e-3 * np.abs(er)), 'step %d energies %s vs %s' % (k, eg, er)
        nr, ng = r.tiles(0)[0], g.tiles(0)[0]
        assert abs(int(nr.sum()) - int(ng.sum())) <= 1e-4 * nr.sum(), 'step %d totals' % k
        differ = int((nr != ng).sum())
        assert differ <= 0.01 * len(nr), 'step %d: %d tiles differ in count' % (k, differ)


# ---------------------------------------------------------------------------
# Ensemble members inside a Batch
# ---------------------------------------------------------------------------
def _drawn_members():
    from bench import ensemble_specs
    specs = ensemble_specs(256)
    pick = []
    for want in ((512, 8), (64, 2)):
        pick.append(next(i for i, s in enumerate(specs) if (s[0], s[1]) == want))
    for i, s in enumerate(specs):
        if len(pick) == 4:
            break
        if i not in pick and s[0] not in (512, 64) and all(specs[j][0] != s[0] for j in pick):
            pick.append(i)
    return [specs[i] for i in pick]


def test_ensemble_members_in_a_batch_against_the_oracle():
    members = _drawn_members()
    assert {(m[0], m[1]) for m in members} >= {(512, 8), (64, 2)}
    runs = []
    for spec in members:
        geom, setup = ensemble_member(*spec)
        runs.append((geom, setup, setup(zb.Simulation(*geom))))
    batch = zb.Batch([g for _, _, g in runs])
    batch.advance(1)
    batch.synchronize()
    for (geom, setup, g), spec in zip(runs, members):
        o = setup(OracleSim(*geom))
        o.advance(1)
        for sp in range(2):
            assert same_multisets(o.particles(sp), g.particles(sp)), 'member %s species %d' % (spec, sp)
        m = interior_mask(o)
        assert rel_err(g.grid('J')[:, m], o.grid('J')[:, m]) <= J_TOL
        o.close()
    batch.advance(99)
    batch.synchronize()
    for (geom, setup, g), spec in zip(runs, members):
        if ref_available('avx2'):
            r = setup(RefSim(*geom, variant='avx2'))
            r.advance(100)
            er, eg = energies(r), energies(g)
            assert np.all(np.abs(eg - er) <= 1e-3 * np.abs(er)), 'member %s energies %s vs %s' % (spec, eg, er)
            r.close()
        o = setup(OracleSim(*geom))
        reanchor(o, g, 100)
        g2 = g  # the member continues alone for the re-anchored step
        step_and_compare(o, g2, geom, what='member %s step 101' % (spec,))
        o.close()
    batch.close()


# ---------------------------------------------------------------------------
# Weibel: two electron species, and the reference driver's electron/positron variant
# ---------------------------------------------------------------------------
def _growth_rate(t, b2, lo, hi):
    sel = (t >= lo) & (t <= hi)
    return np.polyfit(t[sel], np.log(b2[sel]), 1)[0]


@pytest.mark.parametrize('literal', [True, False], ids=['two-electron-species', 'electron-positron'])
def test_weibel_500_steps_energy_history_and_growth_rate(literal):
    o, g = weibel(literal)(OracleSim(*WEIBEL)), weibel(literal)(zb.Simulation(*WEIBEL))
    same_initial_state(o, g, 2)
    hist_o, hist_g = [], []
    for _ in range(500):
        o.advance(1)
        g.advance(1)
        hist_o.append(energies(o))
        hist_g.append(energies(g))
    ho, hg = np.array(hist_o), np.array(hist_g)
    for k in (99, 199, 299, 399, 499):
        assert np.all(np.abs(hg[k] - ho[k]) <= 1e-3 * np.abs(ho[k])), 'step %d: %s vs %s' % (k + 1, hg[k], ho[k])
    # Weibel growth rate: exponential fit of the magnetic energy over its
    # growth phase (between 1e-6 and 1e-2 of its peak, from the oracle's run)
    t = (np.arange(500) + 1) * WEIBEL[3]
    b2o, b2g = ho[:, -1], hg[:, -1]
    peak = b2o.max()
    grow = np.nonzero((b2o > 1e-6 * peak) & (b2o < 1e-2 * peak))[0]
    assert len(grow) > 20, 'no growth phase found'
    lo, hi = t[grow[0]], t[grow[-1]]
    go, gg = _growth_rate(t, b2o, lo, hi), _growth_rate(t, b2g, lo, hi)
    assert go > 0 and abs(gg - go) <= 1e-3 * go, 'growth rate %g vs %g' % (gg, go)
    # and the last step's arithmetic, exactly
    reanchor(o, g, 500)
    step_and_compare(o, g, WEIBEL, what='step 501')
