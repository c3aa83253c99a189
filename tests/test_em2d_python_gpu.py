"""The Python em2d interface (zpic_b200.em2d, the reference's
openmp/python/em2d class names and signatures) driving the GPU step: a
Weibel script and a moving-window laser script written as for the
reference's module, checked against the oracle, and their ZDF output."""
import numpy as np
import pytest

from em2d_oracle import OracleSim
from zdf_read import read as zdf_read
from zpic_b200 import em2d
from helpers import rel_err

pytestmark = pytest.mark.gpu


def oracle_energies(o):
    e, b = o.emf_energy()
    return np.array([o.species_energy(k) for k in range(o.nsp)] + [e.sum(), b.sum()])


def facade_energies(sim):
    e, b = sim.emf.get_energy()
    return np.array([sim._s.species_energy(sp._index) for sp in sim.species] + [sum(e), sum(b)])


def test_weibel_script(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    electrons = em2d.Species('electrons', -1.0, [4, 4],
                             udist=em2d.udist.ThermalCorr([0.1, 0.1, 0.1], [0, 0, 0.6]))
    positrons = em2d.Species('positrons', +1.0, [4, 4],
                             udist=em2d.udist.ThermalCorr([0.1, 0.1, 0.1], [0, 0, -0.6]))
    sim = em2d.Simulation([8, 8], [16, 16], [12.8, 12.8], 0.07, species=[electrons, positrons])
    assert abs(em2d.zpic.courant(dims=[128, 128], box=[12.8, 12.8]) - 0.0707107) < 1e-6
    while sim.n < 100:
        sim.advance()
    assert sim.n == 100 and abs(sim.t - 7.0) < 1e-9
    o = OracleSim((8, 8), (16, 16), (12.8, 12.8), 0.07)
    o.add_species(-1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, 0.6)))
    o.add_species(1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -0.6)))
    o.advance(100)
    assert rel_err(facade_energies(sim), oracle_energies(o)) <= 1e-3

    # data accessors
    x = electrons.gather('x')
    assert x.shape == (128 * 128 * 16,) and x.min() >= 0 and x.max() < 12.8
    rho = electrons.get_charge().gather()
    assert rho.shape == (128, 128) and abs(float(rho.astype(np.float64).mean()) + 1.0) < 1e-4
    bz = sim.emf.B.gather('z')
    assert bz.shape == (128, 128)
    assert abs(float((bz.astype(np.float64) ** 2).sum()) - sim.emf.get_energy()[1][2]) <= 1e-3 * sum(sim.emf.get_energy()[1])
    pha = electrons.get_phasespace('x', [0, 12.8], 64, 'uz', [-1.5, 1.5], 48)
    assert pha.shape == (48, 64) and pha.sum() > 0
    assert np.all(electrons.get_phasespace('uz', [-1, 1], 8, 'x', [0, 12.8], 8) == 0)   # reference: no case, zeros
    with pytest.raises(Exception):
        electrons.get_phasespace('x', [0, 1], 8, 'x', [0, 1], 8)

    # diagnostics
    sim.emf.save('B', 'z')
    sim.current.save('x')
    electrons.save()
    electrons.save_charge()
    electrons.save_phasespace('ux', [-1, 1], 128)
    electrons.save_phasespace('x', [0, 12.8], 64, 'uz', [-1.5, 1.5], 48)
    f = zdf_read(tmp_path / 'EMF' / 'Bz-000100.zdf')
    assert f['grid']['count'] == (128, 128) and np.array_equal(f['datasets']['Bz'], bz)
    assert f['iteration']['name'] == 'Iteration' and f['iteration']['n'] == 100
    f = zdf_read(tmp_path / 'CURRENT' / 'Jx-000100.zdf')
    assert f['grid']['count'] == (128, 128)
    f = zdf_read(tmp_path / 'PARTICLES' / 'particles-electrons-000100.zdf')
    assert f['particles']['np'] == 128 * 128 * 16 and np.array_equal(f['datasets']['x'], x)
    # charge and phase-space deposits are FP32 atomic sums: equal up to their order
    f = zdf_read(tmp_path / 'CHARGE' / 'electrons' / 'electrons-charge-000100.zdf')
    assert np.abs(f['datasets']['electrons-charge'] - rho).max() <= 1e-5 * np.abs(rho).max()
    assert f['iteration']['t'] == float(np.float32(100) * np.float32(0.07))
    f = zdf_read(tmp_path / 'PHASESPACE' / 'electrons' / 'electrons-ux-000100.zdf')
    assert f['grid']['count'] == (128,) and f['grid']['axis'][0]['min'] == -1.0
    f = zdf_read(tmp_path / 'PHASESPACE' / 'electrons' / 'electrons-xuz-000100.zdf')
    assert np.abs(f['datasets']['electrons-xuz'] - pha).max() <= 1e-5 * np.abs(pha).max()


def test_moving_window_laser_script(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    electrons = em2d.Species('electrons', -1.0, [4, 2], density=em2d.density.Step('x', 1.0, 2.0))
    sim = em2d.Simulation([16, 4], [16, 16], [256 * 0.025, 64 * 0.1], 0.022,
                          species=electrons, moving_window=True)
    assert sim.add(em2d.laser.Gaussian(start=5.5, fwhm=1.0, a0=2.0, omega0=10.0, W0=1.5,
                                       focus=5.0, axis=3.2, sin_pol=1)) == 0
    sim.current.set_filter(em2d.filter.Compensated('x', 2))
    for _ in range(60):
        sim.advance()
    o = OracleSim((16, 4), (16, 16), (256 * 0.025, 64 * 0.1), 0.022)
    o.add_species(-1.0, (4, 2), density=('step', 1.0, 2.0, 0))
    o.add_laser('gaussian', start=5.5, fwhm=1.0, a0=2.0, omega0=10.0, W0=1.5, focus=5.0, axis=3.2, sin_pol=1)
    o.set_moving_window()
    o.current_set_filter('compensated', 0, 2)
    o.advance_mov_window(60)
    assert rel_err(facade_energies(sim), oracle_energies(o)) <= 1e-3
    # 60 steps of dt 0.022 move a window of dx 0.025 by 52 cells
    sim.emf.save('E', 'z')
    electrons.save_charge()
    f = zdf_read(tmp_path / 'EMF' / 'Ez-000060.zdf')
    assert abs(f['grid']['axis'][0]['min'] - 52 * 0.025) < 1e-6
    f = zdf_read(tmp_path / 'CHARGE' / 'electrons' / 'electrons-charge-000060.zdf')
    assert abs(f['grid']['axis'][0]['min'] - 52 * 0.025) < 1e-6
