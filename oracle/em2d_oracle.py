"""ctypes front end for the CPU checkers (test infrastructure only).

Two back ends share one Python interface:

* ``OracleSim``  -- the plain-C restatement ``oracle/em2d_oracle.c``
  (``real='f32'`` bit-exact restatement of the reference scalar build,
  ``real='f64'`` the FP64 build of the same path);
* ``RefSim``     -- the reference's own openmp/em2d sources compiled by
  ``oracle/Makefile`` into ``oracle/_ref/`` (``variant='scalar'`` is the
  parity pin, ``variant='avx2'`` the reference's fastest CPU path).

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline arms
may use this module; the product never imports it.

Specs shared with the product's Python binding:

* density: ``('none',)``, ``('uniform', n0)``, ``('step', n0, pos, dir)``,
  ``('slab', n0, begin, end, dir)``, ``('sphere', n0, cx, cy, r)``
  (``dir`` 0 = x, 1 = y) -- density.h:12-131
* udist: ``('none',)``, ``('cold', ufl)``, ``('thermal', uth, ufl)``,
  ``('thermalcorr', uth, ufl, npmin)`` -- udist.h:11-58
* bc: ``(xlo, xhi, ylo, yhi)`` with the reference's enum values
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_DENS = {'none': 0, 'uniform': 1, 'step': 2, 'slab': 3, 'sphere': 4}
_UDIST = {'none': 0, 'cold': 1, 'thermal': 2, 'thermalcorr': 3}


def density_params(spec):
    """(type code, [n0, a, b, c, dir]) for a density spec tuple."""
    kind = spec[0]
    p = [1.0, 0.0, 0.0, 0.0, 0.0]
    if kind == 'uniform':
        p[0] = spec[1]
    elif kind == 'step':
        p[0], p[1] = spec[1], spec[2]
        p[4] = spec[3] if len(spec) > 3 else 0
    elif kind == 'slab':
        p[0], p[1], p[2] = spec[1], spec[2], spec[3]
        p[4] = spec[4] if len(spec) > 4 else 0
    elif kind == 'sphere':
        p[0], p[1], p[2], p[3] = spec[1], spec[2], spec[3], spec[4]
    elif kind == 'none':
        p[0] = 0.0
    return _DENS[kind], p


def udist_params(spec):
    """(type code, uth[3], ufl[3], npmin) for a udist spec tuple."""
    kind = spec[0]
    uth, ufl, npmin = (0.0, 0.0, 0.0), (0.0, 0.0, 0.0), 2
    if kind == 'cold':
        ufl = spec[1]
    elif kind == 'thermal':
        uth, ufl = spec[1], spec[2]
    elif kind == 'thermalcorr':
        uth, ufl = spec[1], spec[2]
        if len(spec) > 3:
            npmin = spec[3]
    return _UDIST[kind], list(uth), list(ufl), npmin


def laser_params(**kw):
    """Parameter vector {start, fwhm, rise, flat, fall, a0, omega0, polarization,
    cos_pol, sin_pol, filter, W0, focus, axis} (laser.h:12-131 defaults)."""
    keys = ['start', 'fwhm', 'rise', 'flat', 'fall', 'a0', 'omega0', 'polarization',
            'cos_pol', 'sin_pol', 'filter', 'W0', 'focus', 'axis']
    d = dict.fromkeys(keys, 0.0)
    d['filter'] = 1.0
    d.update(kw)
    return [float(d[k]) for k in keys]


def _arr(x, ct):
    return (ct * len(x))(*x)


class _Sim:
    prefix = None

    def _fn(self, name, restype, argtypes):
        f = getattr(self.lib, self.prefix + name)
        f.restype = restype
        f.argtypes = argtypes
        return f

    def _setup(self, real):
        P, I, U, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint, ctypes.c_double
        F, FP, IP = ctypes.c_float, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int)
        self.real = real
        self._rt = np.float32 if real == 'f32' else np.float64
        RP = ctypes.POINTER(ctypes.c_float if real == 'f32' else ctypes.c_double)
        pre = 'osim_' if self.prefix == 'osim_' else 'ref_'
        self.f = {}
        if pre == 'osim_':
            self.f['set_clock'] = self._fn('set_clock', None, [P, U])
        tab = {
            'sim_create' if pre == 'ref_' else 'create': (P, [U, U, U, U, F, F, D]),
            'sim_destroy' if pre == 'ref_' else 'destroy': (None, [P]),
            'add_species': (I, [P] + ([ctypes.c_char_p] if pre == 'ref_' else []) +
                            [F, U, U, I, FP, I, FP, FP, I, I, IP]),
            'set_moving_window': (None, [P]),
            'emf_set_bc': (None, [P, IP]),
            'current_set_bc': (None, [P, IP]),
            'current_set_filter': (None, [P, I, I, U]),
            'add_laser': (I, [P, I, FP]),
            'advance': (None, [P, I]),
            'advance_mov_window': (None, [P, I]),
            'current_zero': (None, [P]),
            'current_advance': (None, [P]),
            'emf_advance': (None, [P, I]),
            'species_advance': (None, [P, I]),
            'species_advance_free': (None, [P, I]),
            'species_push': (None, [P, I]),
            'species_move': (None, [P, I]),
            'species_process_bc': (None, [P, I]),
            'species_tile_sort': (None, [P, I]),
            'iter': (U, [P]),
            'nmove': (ctypes.c_uint64, [P]),
            'species_energy': (D, [P, I]),
            'emf_energy': (None, [P, ctypes.POINTER(D)]),
            'species_tiles': (ctypes.c_uint64, [P, I, IP, IP]),
            'species_max_part': (ctypes.c_uint32, [P, I]),
            'species_get': (None, [P, I, IP, RP, RP]),
            'species_set': (I, [P, I, IP, IP, RP, RP]),
            'grid_size': (ctypes.c_uint64, [P, I]),
            'grid_get': (None, [P, I, RP]),
            'grid_set': (None, [P, I, RP]),
            'species_charge': (None, [P, I, RP]),
            'species_phasespace': (I, [P, I, I, FP, I, I, FP, I, RP]),
        }
        for k, (r, a) in tab.items():
            self.f[k.replace('sim_', '') if k.startswith('sim_') else k] = self._fn(k, r, a)
        self._RP = RP

    def _create(self, ntiles, nx, box, dt):
        self.ntiles = tuple(int(v) for v in ntiles)
        self.nx = tuple(int(v) for v in nx)
        self.box = tuple(float(v) for v in box)
        self.dt = float(dt)
        self.h = self.f['create'](self.ntiles[0], self.ntiles[1], self.nx[0], self.nx[1],
                                  self.box[0], self.box[1], self.dt)
        if not self.h:
            raise ValueError('invalid time step (Courant condition violation)')
        self.nsp = 0
        ext = (1 + self.nx[0] + 2, 1 + self.nx[1] + 2)
        self.ext = ext
        self.tile_vol = (ext[0] * ext[1] + 3) & ~3

    def close(self):
        if getattr(self, 'h', None):
            self.f['destroy'](self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- set-up ----
    def add_species(self, m_q, ppc, density=('uniform', 1.0), udist=('none',), push_type=0,
                    bc=None, name='species'):
        dt_, dp = density_params(density)
        ut, uth, ufl, npmin = udist_params(udist)
        F = ctypes.c_float
        args = [self.h]
        if self.prefix == 'ref_':
            args.append(name.encode())
        args += [float(m_q), int(ppc[0]), int(ppc[1]), dt_, _arr(dp, F), ut,
                 _arr(uth, F), _arr(ufl, F), int(npmin), int(push_type),
                 _arr(bc, ctypes.c_int) if bc is not None else None]
        r = self.f['add_species'](*args)
        if r < 0:
            raise ValueError('add_species failed')
        self.nsp += 1
        return r

    def set_moving_window(self):
        self.f['set_moving_window'](self.h)

    def emf_set_bc(self, bc):
        self.f['emf_set_bc'](self.h, _arr(bc, ctypes.c_int))

    def current_set_bc(self, bc):
        self.f['current_set_bc'](self.h, _arr(bc, ctypes.c_int))

    def current_set_filter(self, kind, direction=0, order=1):
        code = {'none': 0, 'binomial': 1, 'compensated': 2}[kind]
        self.f['current_set_filter'](self.h, code, int(direction), int(order))

    def add_laser(self, kind, **kw):
        return self.f['add_laser'](self.h, {'plane': 0, 'gaussian': 1}[kind],
                                   _arr(laser_params(**kw), ctypes.c_float))

    # ---- stepping ----
    def advance(self, n=1):
        self.f['advance'](self.h, int(n))

    def advance_mov_window(self, n=1):
        self.f['advance_mov_window'](self.h, int(n))

    def current_zero(self):
        self.f['current_zero'](self.h)

    def current_advance(self):
        self.f['current_advance'](self.h)

    def emf_advance(self, with_current=True):
        self.f['emf_advance'](self.h, int(bool(with_current)))

    def species_advance(self, sp):
        self.f['species_advance'](self.h, sp)

    def species_advance_free(self, sp):
        """Species::advance(): free streaming, no fields, no current (species.cpp:1998-2012)."""
        self.f['species_advance_free'](self.h, sp)

    def species_push(self, sp):
        self.f['species_push'](self.h, sp)

    def species_move(self, sp):
        self.f['species_move'](self.h, sp)

    def species_process_bc(self, sp):
        self.f['species_process_bc'](self.h, sp)

    def species_tile_sort(self, sp):
        self.f['species_tile_sort'](self.h, sp)

    def set_clock(self, k):
        """Oracle only: every clock (iterations, window moves) as k steps from
        t = 0 leave them; with set_particles / set_grid this continues a
        state taken at step k."""
        self.f['set_clock'](self.h, int(k))

    # ---- diagnostics ----
    def iter(self):
        return int(self.f['iter'](self.h))

    def nmove(self):
        return int(self.f['nmove'](self.h))

    def species_energy(self, sp):
        return float(self.f['species_energy'](self.h, sp))

    def emf_energy(self):
        out = (ctypes.c_double * 6)()
        self.f['emf_energy'](self.h, out)
        return np.array(out[:3]), np.array(out[3:])

    def tiles(self, sp):
        nt = self.ntiles[0] * self.ntiles[1]
        np_ = np.zeros(nt, np.int32)
        off = np.zeros(nt, np.int32)
        self.f['species_tiles'](self.h, sp, np_.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                off.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        return np_, off

    def max_part(self, sp):
        return int(self.f['species_max_part'](self.h, sp))

    def particles(self, sp):
        """Particles tile by tile: np[ntiles], ix[N,2] int32, x[N,2], u[N,3]."""
        npt, _ = self.tiles(sp)
        n = int(npt.sum())
        ix = np.zeros((n, 2), np.int32)
        x = np.zeros((n, 2), self._rt)
        u = np.zeros((n, 3), self._rt)
        self.f['species_get'](self.h, sp, ix.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                              x.ctypes.data_as(self._RP), u.ctypes.data_as(self._RP))
        return npt, ix, x, u

    def set_particles(self, sp, npt, ix, x, u):
        npt = np.ascontiguousarray(npt, np.int32)
        ix = np.ascontiguousarray(ix, np.int32)
        x = np.ascontiguousarray(x, self._rt)
        u = np.ascontiguousarray(u, self._rt)
        r = self.f['species_set'](self.h, sp, npt.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                  ix.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                  x.ctypes.data_as(self._RP), u.ctypes.data_as(self._RP))
        if r < 0:
            raise ValueError('too many particles')

    _WHICH = {'E': 0, 'B': 1, 'J': 2}

    def grid(self, which):
        """Tiled buffer incl. guard cells, shape [ntiles, tile_vol, 3]."""
        w = self._WHICH[which]
        n = int(self.f['grid_size'](self.h, w))
        out = np.zeros((n, 3), self._rt)
        self.f['grid_get'](self.h, w, out.ctypes.data_as(self._RP))
        return out.reshape(self.ntiles[0] * self.ntiles[1], self.tile_vol, 3)

    def set_grid(self, which, data):
        data = np.ascontiguousarray(data, self._rt)
        self.f['grid_set'](self.h, self._WHICH[which], data.ctypes.data_as(self._RP))

    def emf_save(self, field, fc):
        """EMF::save through the reference build (writes EMF/<name>-<iter>.zdf in the cwd)."""
        f = self.lib.ref_emf_save
        f.restype, f.argtypes = None, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        f(self.h, {'E': 0, 'B': 1}[field], int(fc))

    def species_save_charge(self, sp):
        f = self.lib.ref_species_save_charge
        f.restype, f.argtypes = None, [ctypes.c_void_p, ctypes.c_int]
        f(self.h, int(sp))

    def phasespace(self, sp, q0, range0, size0, q1=-1, range1=(0.0, 1.0), size1=1):
        """Species::dep_phasespace: out[size0] or out[size1, size0]; quantities
        0 x, 1 y, 2 ux, 3 uy, 4 uz."""
        FP = ctypes.POINTER(ctypes.c_float)
        r0 = (ctypes.c_float * 2)(*range0)
        r1 = (ctypes.c_float * 2)(*range1)
        shape = (size0,) if q1 < 0 else (size1, size0)
        out = np.zeros(shape, self._rt)
        rc = self.f['species_phasespace'](self.h, sp, int(q0), ctypes.cast(r0, FP), int(size0), int(q1),
                                          ctypes.cast(r1, FP), int(size1), out.ctypes.data_as(self._RP))
        if rc != 0:
            raise ValueError('invalid phasespace quantities')
        return out

    def charge(self, sp):
        dims = (self.ntiles[1] * self.nx[1], self.ntiles[0] * self.nx[0])
        out = np.zeros(dims, self._rt)
        self.f['species_charge'](self.h, sp, out.ctypes.data_as(self._RP))
        return out


class OracleSim(_Sim):
    """The plain-C restatement (oracle/em2d_oracle.c)."""
    prefix = 'osim_'
    _libs = {}

    def __init__(self, ntiles, nx, box, dt, real='f32'):
        path = os.path.join(HERE, '_build', 'libem2d_oracle_%s.so' % real)
        if path not in OracleSim._libs:
            if not os.path.exists(path):
                raise FileNotFoundError(path + ' (run make -C oracle)')
            OracleSim._libs[path] = ctypes.CDLL(path)
        self.lib = OracleSim._libs[path]
        self._setup(real)
        self._create(ntiles, nx, box, dt)


class RefSim(_Sim):
    """The reference's own openmp/em2d build (oracle/_ref/)."""
    prefix = 'ref_'
    _libs = {}

    def __init__(self, ntiles, nx, box, dt, variant='scalar', threads=None):
        name = 'libzpic_ref.so' if variant == 'scalar' else 'libzpic_ref_avx2.so'
        path = os.path.join(HERE, '_ref', name)
        if path not in RefSim._libs:
            if not os.path.exists(path):
                raise FileNotFoundError(path + ' (reference build unavailable)')
            RefSim._libs[path] = ctypes.CDLL(path)
        self.lib = RefSim._libs[path]
        self.lib.ref_num_threads.restype = ctypes.c_int
        self.lib.ref_num_threads.argtypes = [ctypes.c_int]
        self.threads = self.lib.ref_num_threads(int(threads) if threads else 0)
        self._setup('f32')
        self._create(ntiles, nx, box, dt)


def ref_available(variant='scalar'):
    name = 'libzpic_ref.so' if variant == 'scalar' else 'libzpic_ref_avx2.so'
    return os.path.exists(os.path.join(HERE, '_ref', name))


def weibel_setup(sim, literal=False):
    """Weibel instability set-up (openmp/em2d/main.cpp:179-259): two species,
    4x4 ppc, ThermalCorr uth 0.1, fluid uz +-0.6.  ``literal=True`` uses two
    electron species (m_q = -1 both) as the benchmark wording states."""
    sim.add_species(-1.0, (4, 4), udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, 0.6)),
                    name='electrons')
    sim.add_species(-1.0 if literal else 1.0, (4, 4),
                    udist=('thermalcorr', (0.1, 0.1, 0.1), (0, 0, -0.6)), name='positrons')
    return sim
