"""The drop-in ZDF writer (zpic-parallel_b200/cpp/zdf.h) writes files byte for
byte like the reference's own writer (zdf.c) for the same data and metadata."""
import os
import subprocess

import numpy as np
import pytest

from em2d_oracle import RefSim, ref_available

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope='module')
def writer(tmp_path_factory):
    out = tmp_path_factory.mktemp('zdfw') / 'zdf_write_grid'
    subprocess.check_call(['/usr/bin/g++', '-O1', '-std=c++17', '-I', os.path.join(ROOT, 'zpic-parallel_b200', 'cpp'),
                           '-o', str(out), os.path.join(ROOT, 'tests', 'tools', 'zdf_write_grid.cpp')])
    return str(out)


@pytest.mark.skipif(not ref_available('scalar'), reason='reference build oracle/_ref not present')
def test_grid_file_bytes_match_reference(writer, tmp_path, monkeypatch):
    geom = ((4, 2), (16, 16), (6.4, 3.2), 0.05)
    r = RefSim(*geom, threads=1)
    r.add_species(-1.0, (2, 2), udist=('thermal', (0.1, 0.1, 0.1), (0, 0, 0)))
    r.add_laser('plane', start=3.0, fwhm=1.0, a0=1.0, omega0=5.0, polarization=0.3)
    r.advance(3)
    monkeypatch.chdir(tmp_path)
    r.emf_save('B', 2)                      # EMF/Bz-000003.zdf, written by the reference
    r.species_save_charge(0)                # CHARGE/species/species-charge-000003.zdf
    ref_b = (tmp_path / 'EMF' / 'Bz-000003.zdf').read_bytes()
    ref_c = (tmp_path / 'CHARGE' / 'species' / 'species-charge-000003.zdf').read_bytes()
    # same data through the drop-in writer
    B = r.grid('B')
    ntx, nty = geom[0]
    nxx, nxy = geom[1]
    ex, ey = r.ext
    dense = np.zeros((nty * nxy, ntx * nxx), np.float32)
    for ty in range(nty):
        for tx in range(ntx):
            blk = B[ty * ntx + tx][:ex * ey].reshape(ey, ex, 3)
            dense[ty * nxy:(ty + 1) * nxy, tx * nxx:(tx + 1) * nxx] = blk[1:1 + nxy, 1:1 + nxx, 2]
    dense.tofile(tmp_path / 'bz.bin')
    subprocess.check_call([writer, str(tmp_path / 'bz.bin'), '64', '32', 'Bz', 'B_z', 'm_e c \\omega_n e^{-1}',
                           '0', '6.4000000953674316', '0', '3.2000000476837158', '3', '0.15000000000000002',
                           str(tmp_path / 'MINE')])
    mine = (tmp_path / 'MINE' / 'Bz-000003.zdf').read_bytes()
    assert mine == ref_b
    rho = r.charge(0).astype(np.float32)
    rho.tofile(tmp_path / 'rho.bin')
    # Species::save_charge stores iter * dt with the species' FP32 time step
    t32 = '%.17g' % float(np.float32(3) * np.float32(0.05))
    subprocess.check_call([writer, str(tmp_path / 'rho.bin'), '64', '32', 'species-charge', 'species \\rho', 'n_e',
                           '0', '6.4000000953674316', '0', '3.2000000476837158', '3', t32,
                           str(tmp_path / 'MINEC'), 'ITERATION'])
    assert (tmp_path / 'MINEC' / 'species-charge-000003.zdf').read_bytes() == ref_c
    # the test reader parses what the reference wrote
    from zdf_read import read
    g = read(tmp_path / 'EMF' / 'Bz-000003.zdf')
    assert g['grid']['count'] == (64, 32) and g['iteration']['n'] == 3
    assert [a['name'] for a in g['grid']['axis']] == ['x', 'y']
    assert abs(g['grid']['axis'][0]['max'] - 6.4) < 1e-6 and abs(g['grid']['axis'][1]['max'] - 3.2) < 1e-6
    assert np.array_equal(g['datasets']['Bz'], dense)
    # the Python writer of the library writes the same bytes
    import zpic_b200.zdf as pz
    fn = pz.save_grid(dense, 'Bz', 'B_z', 'm_e c \\omega_n e^{-1}',
                      [('x', 0.0, float(np.float32(6.4)), 'x', 'c/\\omega_n'),
                       ('y', 0.0, float(np.float32(3.2)), 'y', 'c/\\omega_n')],
                      3, 3 * 0.05, str(tmp_path / 'PY'))
    assert open(fn, 'rb').read() == ref_b
    fn = pz.save_grid(rho, 'species-charge', 'species \\rho', 'n_e',
                      [('x', 0.0, float(np.float32(6.4)), 'x', 'c/\\omega_n'),
                       ('y', 0.0, float(np.float32(3.2)), 'y', 'c/\\omega_n')],
                      3, float(t32), str(tmp_path / 'PYC'), iter_name='ITERATION')
    assert open(fn, 'rb').read() == ref_c


def test_python_particle_file_layout(tmp_path):
    """Particle files of the Python writer read back with the test reader."""
    import zpic_b200.zdf as pz
    from zdf_read import read
    rng = np.random.default_rng(1)
    q = [rng.random(100).astype(np.float32) for _ in range(5)]
    fn = pz.save_particles(q, 'electrons', 'electrons', ['x', 'y', 'ux', 'uy', 'uz'],
                           ['x', 'y', 'u_x', 'u_y', 'u_z'], ['c/\\omega_n'] * 2 + ['c'] * 3, 7, 0.49,
                           str(tmp_path / 'PARTICLES'))
    d = read(fn)
    assert d['TYPE'] == 'particles' and d['particles']['np'] == 100 and d['iteration']['n'] == 7
    for name, a in zip(['x', 'y', 'ux', 'uy', 'uz'], q):
        assert np.array_equal(d['datasets'][name], a)
