"""Per-phase timing (option "profile"): 1 times every phase of eagerly issued
steps, 2 keeps the CUDA graph of the step and times the particle kernel in its
replays through event-record nodes pointed at fresh events before every
replay.  Both count one particle-kernel launch per step and species, report
positive times, and leave the trajectory as it is."""
import numpy as np
import pytest

import zpic_b200 as zb
from helpers import rel_err

pytestmark = pytest.mark.gpu

GEOM = ((8, 8), (16, 16), (12.8, 12.8), 0.07)


def plasma(s):
    s.add_species(-1.0, (4, 4), udist=('thermal', (0.05, 0.05, 0.05), (0, 0, 0)))
    return s


@pytest.mark.parametrize('mode', [1, 2])
def test_profile_modes(mode):
    a, b = plasma(zb.Simulation(*GEOM)), plasma(zb.Simulation(*GEOM))
    b.set_option('profile', mode)
    a.advance(3)
    b.advance(3)
    b.synchronize()
    b.reset_phase_times()
    a.advance(6)
    b.advance(6)
    b.synchronize()
    ph = b.phase_times()
    assert ph['particles'][1] == 6 and ph['particles'][0] > 0
    if mode == 1:
        # eager steps time every phase; graph replays only the particle kernel
        for k in ('sort', 'fields'):
            assert ph[k][1] > 0 and ph[k][0] > 0
    e_a, e_b = a.emf_energy(), b.emf_energy()
    assert rel_err(e_b[0].sum(), e_a[0].sum()) <= 1e-5
    assert rel_err(b.species_energy(0), a.species_energy(0)) <= 1e-6
    # back to untimed graph replays
    b.set_option('profile', 0)
    b.advance(4)
    b.synchronize()
    with pytest.raises(zb.ZpicError):
        b.set_option('profile', 3)


def test_profile_graph_mode_moving_window():
    """Moving-window steps are issued eagerly when profiled (mode 2 included)
    and time every phase."""
    s = zb.Simulation((16, 4), (16, 16), (256 * 0.025, 64 * 0.1), 0.022)
    s.add_species(-1.0, (4, 2), density=('step', 1.0, 2.0, 0))
    s.set_moving_window()
    s.set_option('profile', 2)
    s.advance_mov_window(5)
    s.synchronize()
    ph = s.phase_times()
    assert ph['particles'][1] == 5 and ph['particles'][0] > 0
    assert ph['fields'][1] > 0
