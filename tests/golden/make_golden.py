"""Generates the golden fixtures in this directory from the reference's own
openmp/em2d build (oracle/_ref/libzpic_ref.so, scalar, one OpenMP thread).

    python tests/golden/make_golden.py

The reference's tests hold no known-answer vectors, so these fixtures are
outputs of the reference itself, run here on seeded inputs:

* weibel_small.npz   -- 32x32 cells (4x4 tiles of 8x8), e-/e+ 2x2 ppc,
                        ThermalCorr uth 0.1, ufl +-0.6: full state at step 0
                        and step 5 (particles, tile counts, E, B, J) and the
                        energy history of 40 steps
* weibel_energy.npz  -- the Weibel test of the reference driver
                        (openmp/em2d/main.cpp:179-259: 128x128 cells, 8x8
                        tiles, e-/e+ 4x4 ppc): energies every 10 steps to 500
* lwfa_small.npz     -- 256x64 cells moving window, step density, Gaussian
                        laser (a0 2, omega0 10), compensated filter: particle
                        count and energies every 10 steps to 120
* diagnostics_small.npz -- the Weibel test set-up after 20 steps: charge
                        density of both species and 1D / 2D phase spaces
                        (Species::dep_phasespace) for the PHASESPACES list
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, '..', '..', 'oracle'))
from em2d_oracle import RefSim  # noqa: E402


def weibel(sim, ppc):
    sim.add_species(-1.0, ppc, udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, 0.6)), name='electrons')
    sim.add_species(1.0, ppc, udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -0.6)), name='positrons')
    return sim


def energies(sim):
    e, b = sim.emf_energy()
    return [sim.species_energy(k) for k in range(sim.nsp)] + list(e) + list(b)


def state(sim, tag):
    out = {}
    for sp in range(sim.nsp):
        npt, ix, x, u = sim.particles(sp)
        out['%s_np%d' % (tag, sp)] = npt
        out['%s_ix%d' % (tag, sp)] = ix
        out['%s_x%d' % (tag, sp)] = x
        out['%s_u%d' % (tag, sp)] = u
    for w in 'EBJ':
        out['%s_%s' % (tag, w)] = sim.grid(w)
    return out


# (quant0, range0, size0, quant1, range1, size1); quant1 < 0 for 1D
PHASESPACES = [
    (0, (0.0, 12.8), 64, -1, (0.0, 1.0), 1),
    (1, (1.0, 11.0), 33, -1, (0.0, 1.0), 1),
    (2, (-0.5, 0.5), 100, -1, (0.0, 1.0), 1),
    (4, (-1.0, 1.0), 77, -1, (0.0, 1.0), 1),
    (0, (0.0, 12.8), 64, 2, (-0.5, 0.5), 50),
    (2, (-0.5, 0.5), 40, 4, (-1.2, 1.2), 60),
    (1, (0.0, 12.8), 32, 3, (-0.4, 0.4), 32),
]


def diagnostics():
    s = weibel(RefSim((8, 8), (16, 16), (12.8, 12.8), 0.07, threads=1), (4, 4))
    s.advance(20)
    d = {}
    for sp in range(2):
        d['charge%d' % sp] = s.charge(sp)
        for k, c in enumerate(PHASESPACES):
            d['pha%d_%d' % (sp, k)] = s.phasespace(sp, *c)
    np.savez_compressed(os.path.join(HERE, 'diagnostics_small.npz'), **d)
    s.close()


def main():
    diagnostics()
    geom = ((4, 4), (8, 8), (3.2, 3.2), 0.07)
    s = weibel(RefSim(*geom, threads=1), (2, 2))
    d = state(s, 's0')
    hist = [energies(s)]
    for n in range(1, 41):
        s.advance(1)
        if n == 5:
            d.update(state(s, 's5'))
        hist.append(energies(s))
    d['energy'] = np.array(hist)
    d['geom'] = np.array([4, 4, 8, 8, 3.2, 3.2, 0.07])
    np.savez_compressed(os.path.join(HERE, 'weibel_small.npz'), **d)
    s.close()

    s = weibel(RefSim((8, 8), (16, 16), (12.8, 12.8), 0.07, threads=1), (4, 4))
    hist = [energies(s)]
    for n in range(50):
        s.advance(10)
        hist.append(energies(s))
    np.savez_compressed(os.path.join(HERE, 'weibel_energy.npz'), energy=np.array(hist), every=10)
    s.close()

    s = RefSim((16, 4), (16, 16), (256 * 0.025, 64 * 0.1), 0.022, threads=1)
    s.add_species(-1.0, (4, 2), density=('step', 1.0, 2.0, 0))
    s.add_laser('gaussian', start=5.5, fwhm=1.0, a0=2.0, omega0=10.0, W0=1.5, focus=5.0, axis=3.2, sin_pol=1)
    s.set_moving_window()
    s.current_set_filter('compensated', 0, 2)
    hist, counts = [energies(s)], [s.tiles(0)[0].sum()]
    for n in range(12):
        s.advance_mov_window(10)
        hist.append(energies(s))
        counts.append(s.tiles(0)[0].sum())
    np.savez_compressed(os.path.join(HERE, 'lwfa_small.npz'), energy=np.array(hist), np_total=np.array(counts),
                        every=10)
    s.close()


if __name__ == '__main__':
    main()
