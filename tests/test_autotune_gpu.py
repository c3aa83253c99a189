"""The CTA-per-tile autotuner: it picks one of its candidates, its trial steps
are real steps, and the tuned run stays on the same trajectory as an untuned
run advanced to the same iteration (the choice only changes the FP32 order in
which per-CTA partial currents are added)."""
import numpy as np
import pytest

import zpic_b200 as zb
from helpers import rel_err

pytestmark = pytest.mark.gpu

GEOM = ((8, 8), (16, 16), (12.8, 12.8), 0.07)


def weibel(s):
    s.add_species(-1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, 0.6)))
    s.add_species(1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -0.6)))
    return s


def energies(s):
    e, b = s.emf_energy()
    return np.array([s.species_energy(0), s.species_energy(1), e.sum(), b.sum()])


def test_sim_autotune_keeps_trajectory():
    a, b = weibel(zb.Simulation(*GEOM)), weibel(zb.Simulation(*GEOM))
    c = a.autotune(2)
    assert c in (-1, 0, 1, 2, 4, 8, 16, 32, 64)
    n = a.iter()
    assert n >= 3                       # one candidate at least: 1 + 2 steps
    b.advance(n)
    a.advance(20)
    b.advance(20)
    assert rel_err(energies(a), energies(b)) <= 1e-4
    for sp in range(2):
        assert a.np_total(sp) == b.np_total(sp) == 128 * 128 * 16
    with pytest.raises(zb.ZpicError):
        a.autotune(0)


def test_batch_autotune():
    sims = [weibel(zb.Simulation(*GEOM)) for _ in range(3)]
    ref = weibel(zb.Simulation(*GEOM))
    batch = zb.Batch(sims)
    c = batch.autotune(2)
    assert c in (0, 1, 2, 4, 8, 16, 32, 64)
    batch.advance(10)
    batch.synchronize()
    n = sims[0].iter()
    assert all(s.iter() == n for s in sims)
    ref.advance(n)
    for s in sims:
        assert rel_err(energies(s), energies(ref)) <= 1e-4
    batch.close()
