"""zpic_b200_charge_deposit_noalloc: the charge density for callers that cannot
allocate device memory (a framework that owns all device memory through its
own pool, a real-time or in-situ loop that must not stall on the allocator).
The caller allocates the inputs and the output; the entry point itself uses
the library's fixed scratch array and must give the same density as
zpic_b200_species_charge, call after call (the shared scratch is cleared by
each call).

This file is collected last so that a run stopping at the first failure has
run every other test before it.
"""
import numpy as np
import pytest

import zpic_b200 as zb

pytestmark = pytest.mark.gpu

GEOM = ((8, 8), (16, 16), (12.8, 12.8), 0.07)
M_Q = (-1.0, 1.0)
# both paths sum FP32 shared-memory atomics per tile in different orders
RHO_TOL = 1e-6


def _weibel():
    sim = zb.Simulation(*GEOM, device=0)
    for m_q, uz in zip(M_Q, (0.6, -0.6)):
        sim.add_species(m_q, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, uz)))
    sim.advance(3)
    return sim


def _noalloc_charge(sim, sp, parts=None):
    import torch
    npt, ix, x, _ = parts if parts is not None else sim.particles(sp)
    off = np.zeros_like(npt)
    off[1:] = np.cumsum(npt)[:-1]
    d_np = torch.from_numpy(npt).cuda()
    d_off = torch.from_numpy(off).cuda()
    d_ix = torch.from_numpy(ix).cuda()
    d_x = torch.from_numpy(x).cuda()
    ny, nx = GEOM[0][1] * GEOM[1][1], GEOM[0][0] * GEOM[1][0]
    out = torch.full((ny, nx), float('nan'), dtype=torch.float32, device='cuda')
    q = np.float32(np.copysign(1.0, M_Q[sp]) / 16.0)      # n0 / (ppc.x * ppc.y)
    stream = torch.cuda.current_stream()
    zb.charge_deposit_noalloc(GEOM[0], GEOM[1], q, d_np.data_ptr(), d_off.data_ptr(), d_ix.data_ptr(),
                              d_x.data_ptr(), out.data_ptr(), stream.cuda_stream)
    stream.synchronize()
    return out.cpu().numpy()


def test_noalloc_charge_matches_allocating_path_twice():
    sim = _weibel()
    for sp in (0, 1):            # two calls in a row through the shared scratch
        ref = sim.charge(sp)
        got = _noalloc_charge(sim, sp)
        assert np.isfinite(got).all()
        assert np.abs(got - ref).max() <= RHO_TOL * np.abs(ref).max()


def test_noalloc_rejects_grid_beyond_scratch():
    import torch
    dummy = torch.zeros(4, dtype=torch.int32, device='cuda')
    with pytest.raises(zb.ZpicError, match='maximum'):
        zb.charge_deposit_noalloc((512, 512), (16, 16), 1.0, dummy.data_ptr(), dummy.data_ptr(),
                                  dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), 0)


def test_noalloc_rejects_oversized_tiles_before_any_work():
    """Tile sides whose guard-cell block would overflow 32-bit arithmetic
    (65535 + 1 squared wraps to 0) are rejected on the host, like any tile
    block above 12,288 cells."""
    import torch
    dummy = torch.zeros(4, dtype=torch.int32, device='cuda')
    for nx in ((65535, 65535), (12288, 1), (110, 110), (4294967295, 1)):
        with pytest.raises(zb.ZpicError, match='maximum'):
            zb.charge_deposit_noalloc((1, 1), nx, 1.0, dummy.data_ptr(), dummy.data_ptr(),
                                      dummy.data_ptr(), dummy.data_ptr(), dummy.data_ptr(), 0)


def test_noalloc_skips_particles_outside_their_tile():
    """Particles whose cell lies outside their tile (an unsorted set) are
    skipped: the result is the deposit of the others."""
    sim = _weibel()
    npt, ix, x, u = sim.particles(0)
    bad = ix.copy()
    bad[0] = (-1, 0)
    bad[1] = (GEOM[1][0], 3)
    bad[2] = (5, GEOM[1][1] + 7)
    got = _noalloc_charge(sim, 0, (npt, bad, x, u))
    keep = np.ones(len(ix), bool)
    keep[:3] = False
    # the same set with those three particles removed (they sit in tile 0)
    npt2 = npt.copy()
    npt2[0] -= 3
    ref = _noalloc_charge(sim, 0, (npt2, ix[keep], x[keep], u[keep]))
    assert np.isfinite(got).all()
    assert np.abs(got - ref).max() <= RHO_TOL * np.abs(ref).max()
