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


def _rows(ix, x, u):
    return np.concatenate([np.ascontiguousarray(ix, np.int32).view(np.uint32),
                           np.ascontiguousarray(x, np.float32).view(np.uint32),
                           np.ascontiguousarray(u, np.float32).view(np.uint32)], axis=1)


def _canonical(npt, ix, x, u):
    """Rows (raw 32-bit words) of a particle state with their tile index as a
    last column, in a canonical order: sorted by a 64-bit mix of the tile and
    the row.  Equal multisets per tile give equal arrays; rows that mix to the
    same key can only be reordered between two states if they differ, which
    makes the comparison fail, never pass."""
    rows = _rows(ix, x, u)
    tile = np.repeat(np.arange(len(npt), dtype=np.uint32), np.asarray(npt, np.int64))
    rows = np.concatenate([rows, tile[:, None]], axis=1)
    w = rows.view(np.uint64) if rows.shape[1] % 2 == 0 else None
    h = np.full(len(rows), 0x243F6A8885A308D3, np.uint64)
    cols = [w[:, k] for k in range(w.shape[1])] if w is not None else \
        [rows[:, k].astype(np.uint64) for k in range(rows.shape[1])]
    for c in cols:
        h ^= c
        h *= np.uint64(0xBF58476D1CE4E5B9)
        h ^= h >> np.uint64(31)
    return np.take(rows, np.argsort(h), axis=0)


def same_multisets(a, b):
    """True when two particle states (np, ix, x, u) hold the same particles per tile, bit for bit."""
    if not np.array_equal(np.asarray(a[0]), np.asarray(b[0])):
        return False
    return np.array_equal(_canonical(*a), _canonical(*b))


def multiset_mismatch_tiles(a, b):
    """Tiles whose particle multisets differ (counts or contents) between two states."""
    na, nb = np.asarray(a[0]), np.asarray(b[0])
    bad = set(np.nonzero(na != nb)[0].tolist())
    same = np.nonzero(na == nb)[0]
    ca, cb = _canonical(*a), _canonical(*b)
    oa = np.concatenate([[0], np.cumsum(na)])
    ob = np.concatenate([[0], np.cumsum(nb)])
    for t in same:
        if not np.array_equal(ca[oa[t]:oa[t + 1]], cb[ob[t]:ob[t + 1]]):
            bad.add(int(t))
    return sorted(bad)


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
