"""The reference's own test drivers (Weibel, LWFA), built against the drop-in
C++ headers (zpic-parallel_b200/cpp/) and run on the GPU: their printed
energies agree with the oracle, and their ZDF diagnostics are readable and
consistent with the library's state."""
import os
import re
import subprocess

import numpy as np
import pytest

from em2d_oracle import OracleSim
from zdf_read import read as zdf_read

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, 'zpic-parallel_b200', 'bin')


def run(tmp_path, exe, *args):
    out = subprocess.run([os.path.join(BIN, exe)] + [str(a) for a in args], cwd=tmp_path,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    return out.stdout


def energies(text):
    vals = dict(re.findall(r'\(\*info\*\) (.+?) = (-?[0-9.eE+-]+)', text))
    return {k: float(v) for k, v in vals.items()}


def test_weibel_driver(tmp_path):
    out = run(tmp_path, 'weibel', 100)
    e = energies(out)
    o = OracleSim((8, 8), (16, 16), (12.8, 12.8), 0.07)
    o.add_species(-1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, 0.6)))
    o.add_species(1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -0.6)))
    o.advance(100)
    ee, eb = o.emf_energy()
    assert abs(e['electrons'] - o.species_energy(0)) <= 1e-3 * o.species_energy(0)
    assert abs(e['positrons'] - o.species_energy(1)) <= 1e-3 * o.species_energy(1)
    assert abs(e['Electric field'] - ee.sum()) <= 1e-3 * ee.sum()
    assert abs(e['Magnetic field'] - eb.sum()) <= 1e-3 * eb.sum()
    assert re.search(r'\[benchmark\] [0-9.]+ GPart/s', out)
    bz = zdf_read(tmp_path / 'EMF' / 'Bz-000100.zdf')
    assert bz['TYPE'] == 'grid' and bz['grid']['count'] == (128, 128) and bz['iteration']['n'] == 100
    # the saved Bz squared sums to the printed magnetic energy's z part (EMF::get_energy)
    assert abs(float((bz['datasets']['Bz'].astype(np.float64) ** 2).sum()) - eb[2]) <= 1e-3 * eb.sum() + 1e-6
    p = zdf_read(tmp_path / 'PARTICLES' / 'particles-electrons-000100.zdf')
    assert p['TYPE'] == 'particles' and p['particles']['np'] == 128 * 128 * 16
    x = p['datasets']['x']
    assert x.min() >= 0 and x.max() < 12.8
    rho = zdf_read(tmp_path / 'CHARGE' / 'electrons' / 'electrons-charge-000100.zdf')['datasets']['electrons-charge']
    assert abs(float(rho.astype(np.float64).mean()) + 1.0) < 1e-4     # n0 = 1 electrons
    pux = zdf_read(tmp_path / 'PHASESPACE' / 'electrons' / 'electrons-ux-000100.zdf')
    assert pux['grid']['count'] == (128,) and pux['grid']['axis'][0]['min'] == -1.0
    # density integrates to n0 = 1 over the box (12.8 x 12.8) times the bin width
    # in u (bins below -1, above 1 and the last one are not deposited)
    assert 0.95 < float(pux['datasets']['electrons-ux'].astype(np.float64).sum()) * (2.0 / 128) / (12.8 * 12.8) < 1.0001
    pxz = zdf_read(tmp_path / 'PHASESPACE' / 'electrons' / 'electrons-xuz-000100.zdf')
    assert pxz['grid']['count'] == (128, 96) and pxz['datasets']['electrons-xuz'].shape == (96, 128)


def test_lwfa_driver(tmp_path):
    out = run(tmp_path, 'lwfa', 2.0)
    e = energies(out)
    assert np.isfinite(list(e.values())).all()
    assert e['Electric field'] > 0
    ex = zdf_read(tmp_path / 'EMF' / ('Ez-%06d.zdf' % int(re.search(r'n = (\d+)', out).group(1))))
    assert ex['grid']['count'] == (1024, 128)
