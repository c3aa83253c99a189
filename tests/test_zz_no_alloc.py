"""zpic_b200_charge_deposit_noalloc: the charge density for callers that cannot
allocate device memory (frameworks owning all device memory, allocation-free
real-time loops, work recorded into CUDA graphs).  The caller allocates the
inputs and the output; the entry point itself uses the library's fixed
scratch array and must give the same density as zpic_b200_species_charge,
call after call (the shared scratch is cleared by each call).

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


def _noalloc_charge(sim, sp):
    import torch
    npt, ix, x, _ = sim.particles(sp)
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
