"""Python em2d interface with the class names, constructors, properties and
methods of the reference's Cython module (openmp/python/em2d/em2d.pyx), on
the B200 library.  A script written for the reference's module runs on the
GPU after changing its import, e.g. ``from zpic_b200 import em2d``:

    sim = em2d.Simulation([8, 8], [16, 16], [12.8, 12.8], 0.07,
                          species=[em2d.Species('electrons', -1, [4, 4],
                                   udist=em2d.udist.ThermalCorr([.1, .1, .1], [0, 0, .6]))])
    while sim.t < 35: sim.advance()
    Bz = sim.emf.B.gather('z')

Grids live on the GPU: ``gather`` copies a dense component to a numpy
array, and the Grid/Vec3Grid objects are read-only views (no tiled buffer
access).  The plotting helpers of the reference module (matplotlib) are not
provided.  ZDF output goes through zpic_b200.zdf with the reference's file
names and metadata.
"""
import numpy as np

from .. import Simulation as _Sim, ZpicError  # noqa: F401
from .. import zdf as _zdf
from . import density, filter, laser, udist  # noqa: F401

_FC = {'x': 0, 'y': 1, 'z': 2}
_TIME_UNITS = '1/\\omega_n'
_LEN_UNITS = 'c/\\omega_n'


class zpic:
    """zpic.courant(...) and zpic.sys_info() (em2d.pyx:12-72)."""

    @staticmethod
    def sys_info():
        from .. import lib
        print('B200 (sm_100a) em2d library, version %d' % lib().zpic_b200_version())

    @staticmethod
    def courant(dx=None, dims=None, ntiles=None, nx=None, box=None):
        """CFL time-step limit, in FP32 like the reference's zpic::courant."""
        f = np.float32
        if dx is None:
            if ntiles is not None:
                dims = [ntiles[0] * nx[0], ntiles[1] * nx[1]]
            dx = [f(box[0]) / f(dims[0]), f(box[1]) / f(dims[1])]
        dxx, dxy = f(dx[0]), f(dx[1])
        return float(np.sqrt(f(1) / (f(1) / (dxx * dxx) + f(1) / (dxy * dxy))))


class Grid:
    """Dense scalar grid (e.g. a species' charge density); ``gather()`` returns it."""

    def __init__(self, data):
        self._data = np.asarray(data, np.float32)

    def gather(self):
        return self._data.copy()


class Vec3Grid:
    """View of one of the simulation's vector grids (E, B or J)."""

    def __init__(self, sim, which):
        self._sim, self._which = sim, which

    def gather(self, fc):
        """Dense [ny, nx] float32 copy of field component fc ('x', 'y' or 'z')."""
        return self._sim._s.grid_gather(self._which, _FC[fc])


class EMF:
    """View of the simulation's electromagnetic fields (em2d.pyx:694-938)."""

    def __init__(self, sim):
        self._sim = sim

    @property
    def E(self):
        return Vec3Grid(self._sim, 'E')

    @property
    def B(self):
        return Vec3Grid(self._sim, 'B')

    @property
    def n(self):
        return self._sim.n

    @property
    def box(self):
        return self._sim.box

    def save(self, fld, fc):
        """EMF::save: EMF/<fld><fc>-<n>.zdf (emf.cpp:593-655)."""
        s = self._sim
        motion = s._emf_motion()
        data = s._s.grid_gather(fld, _FC[fc])
        return _zdf.save_grid(data, fld + fc, fld + '_' + fc, 'm_e c \\omega_n e^{-1}',
                              [('x', motion, s.box[0] + motion, 'x', _LEN_UNITS),
                               ('y', 0.0, s.box[1], 'y', _LEN_UNITS)],
                              s.n, s.n * s.dt, 'EMF', _TIME_UNITS)

    def get_energy(self):
        """EMF::get_energy: (sum E_x^2, ...), (sum B_x^2, ...)."""
        e, b = self._sim._s.emf_energy()
        return tuple(e), tuple(b)


class Current:
    """View of the simulation's current density (em2d.pyx:502-692)."""

    def __init__(self, sim):
        self._sim = sim

    @property
    def J(self):
        return Vec3Grid(self._sim, 'J')

    @property
    def n(self):
        return self._sim.n

    def set_filter(self, flt):
        """Current::set_filter with an em2d.filter object."""
        self._sim._s.current_set_filter(flt.kind, flt.direction, flt.level)

    def save(self, fc):
        """Current::save: CURRENT/J<fc>-<n>.zdf (current.cpp:262-313)."""
        s = self._sim
        motion = s._emf_motion()
        data = s._s.grid_gather('J', _FC[fc])
        return _zdf.save_grid(data, 'J' + fc, 'J_' + fc, 'e \\omega_n^2 / c',
                              [('x', motion, s.box[0], 'x', _LEN_UNITS),
                               ('y', motion, s.box[1], 'y', _LEN_UNITS)],
                              s.n, s.n * s.dt, 'CURRENT', _TIME_UNITS)


class _Window:
    """MovingWindow bookkeeping (moving_window.h): the window moves by one cell
    whenever t passes the next cell boundary."""

    def __init__(self):
        self.active, self.n_move, self.dx = False, 0, 0.0

    def init(self, dx):
        self.active, self.n_move, self.dx = True, 0, float(dx)

    def needs_move(self, t):
        return self.active and t > self.dx * (self.n_move + 1)

    def motion(self):
        return self.n_move * self.dx


_QUANTS = ('x', 'y', 'ux', 'uy', 'uz')


class Species:
    """Species( name, m_q, ppc, *, udist = None, density = None )
    (em2d.pyx:940-1417).  Becomes usable once a Simulation holds it."""

    def __init__(self, name=None, m_q=0.0, ppc=None, *, udist=None, density=None):
        self._name = name
        self.m_q = float(m_q)
        self.ppc = tuple(int(v) for v in ppc) if ppc is not None else None
        self._udist = udist
        self._density = density
        self._sim = None
        self._index = -1
        self._window = _Window()

    @property
    def name(self):
        return self._name

    def set_udist(self, u):
        self._udist = u

    def set_density(self, d):
        self._density = d

    # ---- helpers ----
    def _attached(self):
        if self._sim is None:
            raise ZpicError('species %s has not been added to a simulation' % self._name)
        return self._sim

    def _iter(self):
        return self._attached().n

    def _t32(self):
        # the species' time: iteration times its FP32 time step
        return float(np.float32(self._iter()) * np.float32(self._attached().dt))

    def _dx(self):
        s = self._attached()
        return (float(np.float32(s.box[0]) / np.float32(s.ntiles[0] * s.nx[0])),
                float(np.float32(s.box[1]) / np.float32(s.ntiles[1] * s.nx[1])))

    # ---- data ----
    def np_total(self):
        return self._attached()._s.np_total(self._index)

    def gather(self, q):
        """Species::gather: one quantity of every particle ('x', 'y' in simulation units)."""
        return self._attached()._s.gather(self._index, q)

    def get_charge(self):
        """Charge density (Species::deposit_charge + add_from_gc) as a Grid."""
        return Grid(self._attached()._s.charge(self._index))

    def get_phasespace(self, quant0, range0, size0, quant1=None, range1=None, size1=None):
        """Species::dep_phasespace: 1D [size0] or 2D [size1, size0] float32 density."""
        s = self._attached()._s
        if quant1 is None:
            return s.phasespace(self._index, quant0, range0, size0)
        if quant1 == quant0:
            raise Exception('Cannot generate a 2d phasespace with the same quantity on both axis')
        if _QUANTS.index(quant1) < _QUANTS.index(quant0):
            # the reference's deposit has no case for this order and leaves the grid zeroed
            return np.zeros((size1, size0), np.float32)
        return s.phasespace(self._index, quant0, range0, size0, quant1, range1, size1)

    # ---- diagnostics ----
    def save(self):
        """Species::save: PARTICLES/particles-<name>-<n>.zdf."""
        data = [self.gather(q) for q in _QUANTS]
        return _zdf.save_particles(data, self._name, self._name, list(_QUANTS),
                                   ['x', 'y', 'u_x', 'u_y', 'u_z'],
                                   [_LEN_UNITS, _LEN_UNITS, 'c', 'c', 'c'],
                                   self._iter(), self._t32(), 'PARTICLES', _TIME_UNITS)

    def save_charge(self):
        """Species::save_charge: CHARGE/<name>/<name>-charge-<n>.zdf."""
        s = self._attached()
        motion = self._window.motion()
        return _zdf.save_grid(s._s.charge(self._index), self._name + '-charge', self._name + ' \\rho', 'n_e',
                              [('x', motion, s.box[0] + motion, 'x', _LEN_UNITS),
                               ('y', 0.0, s.box[1], 'y', _LEN_UNITS)],
                              self._iter(), self._t32(), 'CHARGE/' + self._name, _TIME_UNITS, 'ITERATION')

    def save_phasespace(self, quant0, range0, size0, quant1=None, range1=None, size1=None):
        """Species::save_phasespace: PHASESPACE/<name>/<name>-<q0>[<q1>]-<n>.zdf."""
        labels = {'x': ('x', _LEN_UNITS), 'y': ('y', _LEN_UNITS), 'ux': ('u_x', 'c'),
                  'uy': ('u_y', 'c'), 'uz': ('u_z', 'c')}
        shift = self._window.motion() if quant0 == 'x' else 0.0
        l0, u0 = labels[quant0]
        axes = [(quant0, range0[0] + shift, range0[1] + shift, l0, u0)]
        if quant1 is None:
            name, label = self._name + '-' + quant0, self._name + '\\,(' + l0 + ')'
        else:
            if _QUANTS.index(quant0) >= _QUANTS.index(quant1):
                print('(*error*) for 2D phasespaces, the 2nd quantity must be indexed higher than the first one')
                return None
            l1, u1 = labels[quant1]
            axes.append((quant1, range1[0], range1[1], l1, u1))
            name = self._name + '-' + quant0 + quant1
            label = self._name + ' \\,(' + l0 + '\\rm{-}' + l1 + ')'
        data = self.get_phasespace(quant0, range0, size0, quant1, range1, size1)
        return _zdf.save_grid(data, name, label, 'n_e', axes, self._iter(), self._t32(),
                              'PHASESPACE/' + self._name, _TIME_UNITS, 'ITERATION')


class Simulation:
    """Simulation( ntiles, nx, box, dt, *, species = None, moving_window = False )
    (em2d.pyx:1419-1558)."""

    def __init__(self, ntiles, nx, box, dt, *, species=None, moving_window=False, device=None):
        self._s = _Sim(ntiles, nx, box, dt, device=device)
        self.ntiles = tuple(int(v) for v in ntiles)
        self.nx = tuple(int(v) for v in nx)
        self.box = tuple(float(v) for v in box)
        self.dt = float(dt)
        self._n = 0
        self._emf_window = _Window()
        self.species = []
        self._emf = EMF(self)
        self._current = Current(self)
        if isinstance(species, Species):
            species = [species]
        for sp in species or []:
            self._add_species(sp)
        self.mov_window = bool(moving_window)
        if self.mov_window:
            self._s.set_moving_window()
            self._emf_window.init(self.box[0] / (self.ntiles[0] * self.nx[0]))
            for sp in self.species:
                sp._window.init(sp._dx()[0])

    def _add_species(self, sp):
        if sp._sim is not None:
            raise ZpicError('species %s already belongs to a simulation' % sp.name)
        u = sp._udist.spec if sp._udist is not None else ('none',)
        d = sp._density.spec if sp._density is not None else ('uniform', 1.0)
        sp._index = self._s.add_species(sp.m_q, sp.ppc, density=d, udist=u, name=sp.name or 'species')
        sp._sim = self
        self.species.append(sp)

    def _add_laser(self, pulse):
        kw = {k: getattr(pulse, k) for k in pulse.KEYS}
        return self._s.add_laser(pulse.kind, **kw)

    def _emf_motion(self):
        return self._emf_window.motion()

    @property
    def t(self):
        return self._n * self.dt

    @property
    def n(self):
        return self._n

    @property
    def emf(self):
        return self._emf

    @property
    def current(self):
        return self._current

    def add(self, src):
        """add( src ): add a laser pulse (em2d.laser.PlaneWave or Gaussian)."""
        if isinstance(src, laser._Pulse):
            return src.add(self._emf)
        raise Exception('Invalid src object type')

    def advance(self):
        """One time step (Simulation::advance, or advance_mov_window with a moving window)."""
        if self.mov_window:
            self._s.advance_mov_window(1)
            for sp in self.species:
                if sp._window.needs_move(float(np.float32(self._n + 1) * np.float32(self.dt))):
                    sp._window.n_move += 1
            if self._emf_window.needs_move((self._n + 1) * self.dt):
                self._emf_window.n_move += 1
        else:
            self._s.advance(1)
        self._n += 1

    def energy_info(self):
        """Simulation::energy_info report."""
        print('(*info*) Energy at n = %d, t = %g' % (self._n, self.t))
        part = 0.0
        for sp in self.species:
            k = self._s.species_energy(sp._index)
            print('(*info*) %s = %g' % (sp.name, k))
            part += k
        if len(self.species) > 1:
            print('(*info*) Total particle energy = %g' % part)
        e, b = self._s.emf_energy()
        print('(*info*) Electric field = %g' % e.sum())
        print('(*info*) Magnetic field = %g' % b.sum())
        print('(*info*) total = %g' % (part + e.sum() + b.sum()))
