"""Batched simulations (zpic_b200_batch_*): several independent runs of
different sizes advanced with one launch per phase give the same results as
advancing each run on its own."""
import numpy as np
import pytest

import zpic_b200 as zb
from helpers import same_multisets, rel_err

pytestmark = pytest.mark.gpu

RUNS = [((4, 4), (16, 16), (6.4, 6.4), 0.07, (2, 2), 0.3),
        ((8, 8), (16, 16), (12.8, 12.8), 0.07, (4, 4), 0.6),
        ((6, 4), (16, 16), (9.6, 6.4), 0.07, (8, 8), 0.5)]


def make(r):
    ntiles, nx, box, dt, ppc, uz = r
    s = zb.Simulation(ntiles, nx, box, dt)
    s.add_species(-1.0, ppc, udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, uz)))
    s.add_species(1.0, ppc, udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -uz)))
    return s


def test_batch_matches_individual_runs():
    solo = [make(r) for r in RUNS]
    batched = [make(r) for r in RUNS]
    b = zb.Batch(batched)
    b.advance(1)
    b.synchronize()
    for s in solo:
        s.advance(1)
    for s, t in zip(solo, batched):
        for sp in range(2):
            assert same_multisets(s.particles(sp), t.particles(sp))
    b.advance(30)
    b.synchronize()
    for s in solo:
        s.advance(30)
    for s, t in zip(solo, batched):
        assert t.iter() == s.iter() == 31
        for sp in range(2):
            assert t.np_total(sp) == s.np_total(sp)
            assert rel_err(t.species_energy(sp), s.species_energy(sp)) <= 1e-3
        eb_s, eb_t = s.emf_energy()[1].sum(), t.emf_energy()[1].sum()
        assert rel_err(eb_t, eb_s) <= 1e-3
    b.close()
