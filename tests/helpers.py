"""Shared helpers for the parity tests: per-tile multisets, tolerances, set-ups."""
import numpy as np


def tile_multisets(npt, ix, x, u):
    """Per-tile particle multisets as sorted rows of raw 32-bit words."""
    rows = np.concatenate([ix.astype(np.int32).view(np.uint32),
                           np.ascontiguousarray(x, np.float32).view(np.uint32),
                           np.ascontiguousarray(u, np.float32).view(np.uint32)], axis=1)
    out = []
    o = 0
    for n in npt:
        r = rows[o:o + n]
        o += n
        order = np.lexsort(r.T[::-1])
        out.append(r[order])
    return out


def same_multisets(a, b):
    """True when two particle states (np, ix, x, u) hold the same particles per tile, bit for bit."""
    if not np.array_equal(a[0], b[0]):
        return False
    ma, mb = tile_multisets(*a), tile_multisets(*b)
    return all(np.array_equal(p, q) for p, q in zip(ma, mb))


def interior_mask(sim):
    """Mask of the tile cells that hold data (excludes the tile_vol padding)."""
    m = np.zeros(sim.tile_vol, bool)
    m[:sim.ext[0] * sim.ext[1]] = True
    return m


def rel_err(a, b):
    """max|a-b| / max|b| (normwise relative error)."""
    d = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max()
    s = np.abs(np.asarray(b, np.float64)).max()
    return d / s if s > 0 else d


def random_fields(sim_like, seed, scale=0.3):
    """Seeded random E/B tiled buffers with consistent (periodic) guard cells."""
    rng = np.random.default_rng(seed)
    ntx, nty = sim_like.ntiles
    nxx, nxy = sim_like.nx
    dense = rng.uniform(-scale, scale, size=(nty * nxy, ntx * nxx, 3)).astype(np.float32)
    return tile_from_dense(sim_like, dense)


def tile_from_dense(sim_like, dense):
    """Tiled buffer [ntiles, tile_vol, 3] from a dense periodic grid (guards filled by wrap)."""
    ntx, nty = sim_like.ntiles
    nxx, nxy = sim_like.nx
    ex, ey = sim_like.ext
    gy, gx = dense.shape[:2]
    out = np.zeros((ntx * nty, sim_like.tile_vol, 3), np.float32)
    jj = np.arange(ey) - 1
    ii = np.arange(ex) - 1
    for ty in range(nty):
        for tx in range(ntx):
            rows = (ty * nxy + jj) % gy
            cols = (tx * nxx + ii) % gx
            blk = dense[np.ix_(rows, cols)]
            out[ty * ntx + tx, :ex * ey] = blk.reshape(ex * ey, 3)
    return out
