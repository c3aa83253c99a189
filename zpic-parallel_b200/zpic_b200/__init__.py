"""Python binding of libzpic_b200.so (the B200 em2d time step), over its C-ABI.

Mirrors the role of the reference's Cython binding (openmp/python/em2d):
``Simulation`` wraps one simulation with its EMF, Current and species;
``Batch`` steps several simulations together.  Every call goes to the CUDA
library; there is no CPU fallback -- importing works without a GPU, but
creating a simulation then fails with the CUDA error.

Specs (same as the reference's constructors):

* density: ``('none',)``, ``('uniform', n0)``, ``('step', n0, pos, dir)``,
  ``('slab', n0, begin, end, dir)``, ``('sphere', n0, cx, cy, r)``
* udist: ``('none',)``, ``('cold', ufl)``, ``('thermal', uth, ufl)``,
  ``('thermalcorr', uth, ufl, npmin)``
* bc tuples: ``(x.lower, x.upper, y.lower, y.upper)`` with the reference's enum values
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(HERE), 'lib', 'libzpic_b200.so')

ZPIC_OK = 0

_DENS = {'none': 0, 'uniform': 1, 'step': 2, 'slab': 3, 'sphere': 4}
_UDIST = {'none': 0, 'cold': 1, 'thermal': 2, 'thermalcorr': 3}
_FILTER = {'none': 0, 'binomial': 1, 'compensated': 2}
_WHICH = {'E': 0, 'B': 1, 'J': 2}
_QUANT = {'x': 0, 'y': 1, 'ux': 2, 'uy': 3, 'uz': 4}
ADVANCE_FULL, ADVANCE_CURRENT, ADVANCE_FREE = 0, 1, 2

# Names of every entry point declared in include/zpic_b200.h
EXPORTS = [
    'zpic_b200_last_error', 'zpic_b200_version', 'zpic_b200_set_device',
    'zpic_b200_sim_create', 'zpic_b200_sim_destroy', 'zpic_b200_sim_add_species',
    'zpic_b200_sim_set_moving_window', 'zpic_b200_sim_advance', 'zpic_b200_sim_advance_mov_window',
    'zpic_b200_sim_iter', 'zpic_b200_sim_nmove', 'zpic_b200_sim_synchronize', 'zpic_b200_sim_set_option',
    'zpic_b200_sim_phase_times', 'zpic_b200_sim_reset_phase_times', 'zpic_b200_sim_launch_count',
    'zpic_b200_sim_stream',
    'zpic_b200_batch_stream', 'zpic_b200_batch_launch_count',
    'zpic_b200_sim_autotune', 'zpic_b200_batch_autotune', 'zpic_b200_species_repacks',
    'zpic_b200_emf_set_bc', 'zpic_b200_emf_advance', 'zpic_b200_emf_energy', 'zpic_b200_laser_add',
    'zpic_b200_current_set_bc', 'zpic_b200_current_set_filter', 'zpic_b200_current_zero',
    'zpic_b200_current_advance',
    'zpic_b200_species_advance', 'zpic_b200_species_advance_mov_window', 'zpic_b200_species_push',
    'zpic_b200_species_move', 'zpic_b200_species_process_bc', 'zpic_b200_species_tile_sort',
    'zpic_b200_species_set_bc', 'zpic_b200_species_set_push_type', 'zpic_b200_species_energy',
    'zpic_b200_species_nmove', 'zpic_b200_species_np_total', 'zpic_b200_species_np_max_tile',
    'zpic_b200_species_max_part', 'zpic_b200_species_relocations',
    'zpic_b200_species_get_tiles', 'zpic_b200_species_get', 'zpic_b200_species_set',
    'zpic_b200_species_gather', 'zpic_b200_species_charge', 'zpic_b200_species_phasespace',
    'zpic_b200_grid_size', 'zpic_b200_grid_get', 'zpic_b200_grid_set', 'zpic_b200_grid_gather',
    'zpic_b200_batch_create', 'zpic_b200_batch_advance', 'zpic_b200_batch_synchronize',
    'zpic_b200_batch_destroy', 'zpic_b200_charge_deposit_noalloc',
]


class ZpicError(RuntimeError):
    pass


class _Density(ctypes.Structure):
    _fields_ = [('type', ctypes.c_int32), ('n0', ctypes.c_float), ('a', ctypes.c_float),
                ('b', ctypes.c_float), ('c', ctypes.c_float), ('dir', ctypes.c_int32)]


class _Udist(ctypes.Structure):
    _fields_ = [('type', ctypes.c_int32), ('uth', ctypes.c_float * 3), ('ufl', ctypes.c_float * 3),
                ('npmin', ctypes.c_int32)]


class _SpeciesDesc(ctypes.Structure):
    _fields_ = [('name', ctypes.c_char_p), ('m_q', ctypes.c_float), ('ppc', ctypes.c_uint32 * 2),
                ('density', _Density), ('udist', _Udist), ('push_type', ctypes.c_int32),
                ('bc', ctypes.c_int32 * 4)]


class _LaserDesc(ctypes.Structure):
    _fields_ = [('type', ctypes.c_int32), ('start', ctypes.c_float), ('fwhm', ctypes.c_float),
                ('rise', ctypes.c_float), ('flat', ctypes.c_float), ('fall', ctypes.c_float),
                ('a0', ctypes.c_float), ('omega0', ctypes.c_float), ('polarization', ctypes.c_float),
                ('cos_pol', ctypes.c_float), ('sin_pol', ctypes.c_float), ('filter', ctypes.c_uint32),
                ('W0', ctypes.c_float), ('focus', ctypes.c_float), ('axis', ctypes.c_float)]


_lib = None


def lib():
    """Load libzpic_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ZpicError('libzpic_b200.so not built: run `make -C zpic-parallel_b200` '
                            '(or __graft_entry__.build())')
        L = ctypes.CDLL(LIB_PATH)
        P, I, U, D = ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint32, ctypes.c_double
        FP, IP, DP = ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(D)
        U64P = ctypes.POINTER(ctypes.c_uint64)
        sig = {
            'zpic_b200_last_error': (ctypes.c_char_p, []),
            'zpic_b200_version': (I, []),
            'zpic_b200_set_device': (I, [I]),
            'zpic_b200_sim_create': (I, [U, U, U, U, ctypes.c_float, ctypes.c_float, D, ctypes.POINTER(P)]),
            'zpic_b200_sim_destroy': (I, [P]),
            'zpic_b200_sim_add_species': (I, [P, ctypes.POINTER(_SpeciesDesc), IP]),
            'zpic_b200_sim_set_moving_window': (I, [P]),
            'zpic_b200_sim_advance': (I, [P, I]),
            'zpic_b200_sim_advance_mov_window': (I, [P, I]),
            'zpic_b200_sim_iter': (I, [P, ctypes.POINTER(U)]),
            'zpic_b200_sim_nmove': (I, [P, U64P]),
            'zpic_b200_sim_synchronize': (I, [P]),
            'zpic_b200_sim_set_option': (I, [P, ctypes.c_char_p, D]),
            'zpic_b200_sim_phase_times': (I, [P, DP, U64P, I]),
            'zpic_b200_sim_reset_phase_times': (I, [P]),
            'zpic_b200_sim_launch_count': (I, [P, U64P]),
            'zpic_b200_sim_stream': (I, [P, ctypes.POINTER(P)]),
            'zpic_b200_batch_stream': (I, [P, ctypes.POINTER(P)]),
            'zpic_b200_batch_launch_count': (I, [P, ctypes.POINTER(ctypes.c_uint64)]),
            'zpic_b200_sim_autotune': (I, [P, I, IP]),
            'zpic_b200_species_repacks': (I, [P, I, U64P]),
            'zpic_b200_species_relocations': (I, [P, I, U64P]),
            'zpic_b200_batch_autotune': (I, [P, I, IP]),
            'zpic_b200_emf_set_bc': (I, [P, IP]),
            'zpic_b200_emf_advance': (I, [P, I]),
            'zpic_b200_emf_energy': (I, [P, DP, DP]),
            'zpic_b200_laser_add': (I, [P, ctypes.POINTER(_LaserDesc)]),
            'zpic_b200_current_set_bc': (I, [P, IP]),
            'zpic_b200_current_set_filter': (I, [P, I, I, U]),
            'zpic_b200_current_zero': (I, [P]),
            'zpic_b200_current_advance': (I, [P]),
            'zpic_b200_species_advance': (I, [P, I, I]),
            'zpic_b200_species_advance_mov_window': (I, [P, I]),
            'zpic_b200_species_push': (I, [P, I]),
            'zpic_b200_species_move': (I, [P, I]),
            'zpic_b200_species_process_bc': (I, [P, I]),
            'zpic_b200_species_tile_sort': (I, [P, I]),
            'zpic_b200_species_set_bc': (I, [P, I, IP]),
            'zpic_b200_species_set_push_type': (I, [P, I, I]),
            'zpic_b200_species_energy': (I, [P, I, DP]),
            'zpic_b200_species_nmove': (I, [P, I, U64P]),
            'zpic_b200_species_np_total': (I, [P, I, U64P]),
            'zpic_b200_species_np_max_tile': (I, [P, I, ctypes.POINTER(U)]),
            'zpic_b200_species_max_part': (I, [P, I, ctypes.POINTER(U)]),
            'zpic_b200_species_get_tiles': (I, [P, I, IP, IP]),
            'zpic_b200_species_get': (I, [P, I, IP, FP, FP]),
            'zpic_b200_species_set': (I, [P, I, IP, IP, FP, FP]),
            'zpic_b200_species_gather': (I, [P, I, I, FP]),
            'zpic_b200_species_charge': (I, [P, I, FP]),
            'zpic_b200_species_phasespace': (I, [P, I, I, FP, I, I, FP, I, FP]),
            'zpic_b200_grid_size': (I, [P, I, U64P]),
            'zpic_b200_grid_get': (I, [P, I, FP]),
            'zpic_b200_grid_set': (I, [P, I, FP]),
            'zpic_b200_grid_gather': (I, [P, I, I, FP]),
            'zpic_b200_batch_create': (I, [ctypes.POINTER(P), I, ctypes.POINTER(P)]),
            'zpic_b200_batch_advance': (I, [P, I]),
            'zpic_b200_batch_synchronize': (I, [P]),
            'zpic_b200_batch_destroy': (I, [P]),
            'zpic_b200_charge_deposit_noalloc': (I, [U, U, U, U, ctypes.c_float, P, P, P, P, P, P]),
        }
        for name, (r, a) in sig.items():
            f = getattr(L, name)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def _check(rc):
    if rc != ZPIC_OK:
        msg = lib().zpic_b200_last_error()
        raise ZpicError('zpic_b200 error %d: %s' % (rc, msg.decode() if msg else ''))


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def density_desc(spec):
    kind = spec[0]
    d = _Density()
    d.type = _DENS[kind]
    d.n0 = 1.0
    if kind == 'uniform':
        d.n0 = spec[1]
    elif kind == 'step':
        d.n0, d.a = spec[1], spec[2]
        d.dir = spec[3] if len(spec) > 3 else 0
    elif kind == 'slab':
        d.n0, d.a, d.b = spec[1], spec[2], spec[3]
        d.dir = spec[4] if len(spec) > 4 else 0
    elif kind == 'sphere':
        d.n0, d.a, d.b, d.c = spec[1], spec[2], spec[3], spec[4]
    elif kind == 'none':
        d.n0 = 0.0
    return d


def udist_desc(spec):
    kind = spec[0]
    u = _Udist()
    u.type = _UDIST[kind]
    u.npmin = 2
    uth, ufl = (0, 0, 0), (0, 0, 0)
    if kind == 'cold':
        ufl = spec[1]
    elif kind == 'thermal':
        uth, ufl = spec[1], spec[2]
    elif kind == 'thermalcorr':
        uth, ufl = spec[1], spec[2]
        if len(spec) > 3:
            u.npmin = spec[3]
    for k in range(3):
        u.uth[k] = uth[k]
        u.ufl[k] = ufl[k]
    return u


class Simulation:
    """Simulation( ntiles, nx, box, dt ) -- simulation.h:39-180 on one B200."""

    def __init__(self, ntiles, nx, box, dt, device=None):
        L = lib()
        if device is not None:
            _check(L.zpic_b200_set_device(int(device)))
        self.ntiles = tuple(int(v) for v in ntiles)
        self.nx = tuple(int(v) for v in nx)
        self.box = tuple(float(v) for v in box)
        self.dt = float(dt)
        h = ctypes.c_void_p()
        _check(L.zpic_b200_sim_create(self.ntiles[0], self.ntiles[1], self.nx[0], self.nx[1],
                                      self.box[0], self.box[1], self.dt, ctypes.byref(h)))
        self.h = h
        self.nsp = 0
        self.ext = (1 + self.nx[0] + 2, 1 + self.nx[1] + 2)
        self.tile_vol = (self.ext[0] * self.ext[1] + 3) & ~3

    def close(self):
        if getattr(self, 'h', None):
            lib().zpic_b200_sim_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- set-up ----
    def add_species(self, m_q, ppc, density=('uniform', 1.0), udist=('none',), push_type=0,
                    bc=(1, 1, 1, 1), name='species'):
        d = _SpeciesDesc()
        self._name = name.encode()
        d.name = self._name
        d.m_q = m_q
        d.ppc[0], d.ppc[1] = int(ppc[0]), int(ppc[1])
        d.density = density_desc(density)
        d.udist = udist_desc(udist)
        d.push_type = int(push_type)
        for k in range(4):
            d.bc[k] = int(bc[k]) if bc is not None else 1
        sid = ctypes.c_int32()
        _check(lib().zpic_b200_sim_add_species(self.h, ctypes.byref(d), ctypes.byref(sid)))
        self.nsp += 1
        return sid.value

    def set_moving_window(self):
        _check(lib().zpic_b200_sim_set_moving_window(self.h))

    def emf_set_bc(self, bc):
        _check(lib().zpic_b200_emf_set_bc(self.h, (ctypes.c_int32 * 4)(*bc)))

    def current_set_bc(self, bc):
        _check(lib().zpic_b200_current_set_bc(self.h, (ctypes.c_int32 * 4)(*bc)))

    def current_set_filter(self, kind, direction=0, order=1):
        _check(lib().zpic_b200_current_set_filter(self.h, _FILTER[kind], int(direction), int(order)))

    def add_laser(self, kind, **kw):
        d = _LaserDesc()
        d.type = {'plane': 0, 'gaussian': 1}[kind]
        d.filter = 1
        for k, v in kw.items():
            setattr(d, k, v)
        rc = lib().zpic_b200_laser_add(self.h, ctypes.byref(d))
        return 0 if rc == ZPIC_OK else -1

    def set_option(self, key, value):
        _check(lib().zpic_b200_sim_set_option(self.h, key.encode(), float(value)))

    def autotune(self, steps=3):
        """Pick the CTAs per tile by timing real steps; returns the choice."""
        v = ctypes.c_int()
        _check(lib().zpic_b200_sim_autotune(self.h, int(steps), ctypes.byref(v)))
        return v.value

    # ---- stepping ----
    def advance(self, n=1):
        _check(lib().zpic_b200_sim_advance(self.h, int(n)))

    def advance_mov_window(self, n=1):
        _check(lib().zpic_b200_sim_advance_mov_window(self.h, int(n)))

    def current_zero(self):
        _check(lib().zpic_b200_current_zero(self.h))

    def current_advance(self):
        _check(lib().zpic_b200_current_advance(self.h))

    def emf_advance(self, with_current=True):
        _check(lib().zpic_b200_emf_advance(self.h, int(bool(with_current))))

    def species_advance(self, sp, mode=ADVANCE_FULL):
        _check(lib().zpic_b200_species_advance(self.h, sp, mode))

    def species_push(self, sp):
        _check(lib().zpic_b200_species_push(self.h, sp))

    def species_move(self, sp):
        _check(lib().zpic_b200_species_move(self.h, sp))

    def species_process_bc(self, sp):
        _check(lib().zpic_b200_species_process_bc(self.h, sp))

    def species_tile_sort(self, sp):
        _check(lib().zpic_b200_species_tile_sort(self.h, sp))

    def synchronize(self):
        _check(lib().zpic_b200_sim_synchronize(self.h))

    # ---- diagnostics ----
    def iter(self):
        v = ctypes.c_uint32()
        _check(lib().zpic_b200_sim_iter(self.h, ctypes.byref(v)))
        return v.value

    def nmove(self):
        v = ctypes.c_uint64()
        _check(lib().zpic_b200_sim_nmove(self.h, ctypes.byref(v)))
        return v.value

    def species_energy(self, sp):
        v = ctypes.c_double()
        _check(lib().zpic_b200_species_energy(self.h, sp, ctypes.byref(v)))
        return v.value

    def repacks(self, sp):
        """Times the tile sort rebuilt the slot layout of species sp."""
        v = ctypes.c_uint64()
        _check(lib().zpic_b200_species_repacks(self.h, sp, ctypes.byref(v)))
        return v.value

    def relocations(self, sp):
        """Tiles of species sp that outgrew their slot and moved into the pool."""
        v = ctypes.c_uint64()
        _check(lib().zpic_b200_species_relocations(self.h, sp, ctypes.byref(v)))
        return v.value

    def np_total(self, sp):
        v = ctypes.c_uint64()
        _check(lib().zpic_b200_species_np_total(self.h, sp, ctypes.byref(v)))
        return v.value

    def np_max_tile(self, sp):
        v = ctypes.c_uint32()
        _check(lib().zpic_b200_species_np_max_tile(self.h, sp, ctypes.byref(v)))
        return v.value

    def max_part(self, sp):
        """Particle-buffer capacity of species sp (Particles::max_part; grows on demand)."""
        v = ctypes.c_uint32()
        _check(lib().zpic_b200_species_max_part(self.h, sp, ctypes.byref(v)))
        return v.value

    def emf_energy(self):
        e = (ctypes.c_double * 3)()
        b = (ctypes.c_double * 3)()
        _check(lib().zpic_b200_emf_energy(self.h, e, b))
        return np.array(e[:]), np.array(b[:])

    def tiles(self, sp):
        nt = self.ntiles[0] * self.ntiles[1]
        np_ = np.zeros(nt, np.int32)
        off = np.zeros(nt, np.int32)
        _check(lib().zpic_b200_species_get_tiles(self.h, sp, _iptr(np_), _iptr(off)))
        return np_, off

    def particles(self, sp):
        """np[ntiles], ix[N,2] int32, x[N,2] float32, u[N,3] float32 (tile order)."""
        npt, _ = self.tiles(sp)
        n = int(npt.sum())
        ix = np.zeros((n, 2), np.int32)
        x = np.zeros((n, 2), np.float32)
        u = np.zeros((n, 3), np.float32)
        _check(lib().zpic_b200_species_get(self.h, sp, _iptr(ix), _fptr(x), _fptr(u)))
        return npt, ix, x, u

    def set_particles(self, sp, npt, ix, x, u):
        npt = np.ascontiguousarray(npt, np.int32)
        ix = np.ascontiguousarray(ix, np.int32)
        x = np.ascontiguousarray(x, np.float32)
        u = np.ascontiguousarray(u, np.float32)
        _check(lib().zpic_b200_species_set(self.h, sp, _iptr(npt), _iptr(ix), _fptr(x), _fptr(u)))

    def gather(self, sp, quant):
        npt, _ = self.tiles(sp)
        out = np.zeros(int(npt.sum()), np.float32)
        _check(lib().zpic_b200_species_gather(self.h, sp, _QUANT[quant], _fptr(out)))
        return out

    def grid(self, which):
        """Tiled buffer incl. guard cells, shape [ntiles, tile_vol, 3]."""
        n = ctypes.c_uint64()
        _check(lib().zpic_b200_grid_size(self.h, _WHICH[which], ctypes.byref(n)))
        out = np.zeros((n.value, 3), np.float32)
        _check(lib().zpic_b200_grid_get(self.h, _WHICH[which], _fptr(out)))
        return out.reshape(self.ntiles[0] * self.ntiles[1], self.tile_vol, 3)

    def set_grid(self, which, data):
        data = np.ascontiguousarray(data, np.float32)
        _check(lib().zpic_b200_grid_set(self.h, _WHICH[which], _fptr(data)))

    def grid_gather(self, which, fc):
        out = np.zeros((self.ntiles[1] * self.nx[1], self.ntiles[0] * self.nx[0]), np.float32)
        _check(lib().zpic_b200_grid_gather(self.h, _WHICH[which], int(fc), _fptr(out)))
        return out

    def charge(self, sp):
        out = np.zeros((self.ntiles[1] * self.nx[1], self.ntiles[0] * self.nx[0]), np.float32)
        _check(lib().zpic_b200_species_charge(self.h, sp, _fptr(out)))
        return out

    PHASESPACE = {'x': 0, 'y': 1, 'ux': 2, 'uy': 3, 'uz': 4}

    def phasespace(self, sp, q0, range0, size0, q1=-1, range1=(0.0, 1.0), size1=1):
        """Species::dep_phasespace: float32 out[size0], or out[size1, size0]
        for a 2D phase space (q1 > q0).  Quantities by index (0 x, 1 y, 2 ux,
        3 uy, 4 uz) or name."""
        q0 = self.PHASESPACE.get(q0, q0)
        q1 = self.PHASESPACE.get(q1, q1)
        r0 = (ctypes.c_float * 2)(*range0)
        r1 = (ctypes.c_float * 2)(*range1)
        out = np.zeros((size0,) if q1 < 0 else (size1, size0), np.float32)
        _check(lib().zpic_b200_species_phasespace(self.h, sp, int(q0), r0, int(size0), int(q1), r1,
                                                  int(size1), _fptr(out)))
        return out

    # ---- instrumentation ----
    def phase_times(self):
        ms = (ctypes.c_double * 5)()
        nl = (ctypes.c_uint64 * 5)()
        _check(lib().zpic_b200_sim_phase_times(self.h, ms, nl, 5))
        names = ['particles', 'sort', 'current', 'fields', 'other']
        return {k: (ms[i], nl[i]) for i, k in enumerate(names)}

    def reset_phase_times(self):
        _check(lib().zpic_b200_sim_reset_phase_times(self.h))

    def stream_handle(self):
        """cudaStream_t (as an int) that all work of this simulation runs on."""
        v = ctypes.c_void_p()
        _check(lib().zpic_b200_sim_stream(self.h, ctypes.byref(v)))
        return v.value or 0

    def launch_count(self):
        v = ctypes.c_uint64()
        _check(lib().zpic_b200_sim_launch_count(self.h, ctypes.byref(v)))
        return v.value


class Batch:
    """Several independent simulations advanced together, one launch per phase."""

    def __init__(self, sims):
        self.sims = list(sims)
        arr = (ctypes.c_void_p * len(self.sims))(*[s.h for s in self.sims])
        h = ctypes.c_void_p()
        _check(lib().zpic_b200_batch_create(arr, len(self.sims), ctypes.byref(h)))
        self.h = h

    def advance(self, n=1):
        _check(lib().zpic_b200_batch_advance(self.h, int(n)))

    def synchronize(self):
        _check(lib().zpic_b200_batch_synchronize(self.h))

    def launch_count(self):
        v = ctypes.c_uint64()
        _check(lib().zpic_b200_batch_launch_count(self.h, ctypes.byref(v)))
        return v.value

    def autotune(self, steps=3):
        """Pick the CTAs per tile for all runs by timing real batch steps."""
        v = ctypes.c_int()
        _check(lib().zpic_b200_batch_autotune(self.h, int(steps), ctypes.byref(v)))
        return v.value

    def stream_handle(self):
        """The cudaStream_t (as an int) the batch's steps run on."""
        v = ctypes.c_void_p()
        _check(lib().zpic_b200_batch_stream(self.h, ctypes.byref(v)))
        return v.value or 0

    def close(self):
        if getattr(self, 'h', None):
            lib().zpic_b200_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def charge_deposit_noalloc(ntiles, nx, q, d_np, d_offset, d_ix, d_x, d_charge, stream=0):
    """Charge density of a packed particle set already on the device, without
    device allocation (see zpic_b200_charge_deposit_noalloc in include/zpic_b200.h).
    Pointer arguments are device addresses (ints); raises ZpicError on failure."""
    _check(lib().zpic_b200_charge_deposit_noalloc(
        int(ntiles[0]), int(ntiles[1]), int(nx[0]), int(nx[1]), float(q),
        d_np, d_offset, d_ix, d_x, d_charge, stream or None))


def weibel_setup(sim, literal=False):
    """Weibel set-up of the reference test driver (openmp/em2d/main.cpp:179-259)."""
    sim.add_species(-1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, 0.6)), name='electrons')
    sim.add_species(-1.0 if literal else 1.0, (4, 4),
                    udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -0.6)), name='positrons')
    return sim
