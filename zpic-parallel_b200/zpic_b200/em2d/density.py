"""Density profiles of the Python em2d interface (the reference's
em2d.density module, openmp/python/em2d/density/density.pyx): None,
Uniform, Step, Slab (and Sphere, which the C++ API also has).  ``None`` is
reached as ``getattr(density, 'None')`` (or ``density.Empty``)."""

_DIR = {'x': 0, 'y': 1}


class _Profile:
    spec = ('uniform', 1.0)


class Empty(_Profile):
    """None(): no particles are injected."""
    spec = ('none',)


class Uniform(_Profile):
    """Uniform( n0 )."""

    def __init__(self, n0):
        self.n0 = float(n0)
        self.spec = ('uniform', self.n0)


class Step(_Profile):
    """Step( dir, n0, pos ): density n0 beyond pos along dir ('x' or 'y')."""

    def __init__(self, dir, n0, pos):
        self.dir, self.n0, self.pos = dir, float(n0), float(pos)
        self.spec = ('step', self.n0, self.pos, _DIR[dir])


class Slab(_Profile):
    """Slab( dir, n0, begin, end ): density n0 between begin and end along dir."""

    def __init__(self, dir, n0, begin, end):
        self.dir, self.n0, self.begin, self.end = dir, float(n0), float(begin), float(end)
        self.spec = ('slab', self.n0, self.begin, self.end, _DIR[dir])


class Sphere(_Profile):
    """Sphere( n0, center, radius )."""

    def __init__(self, n0, center, radius):
        self.n0, self.center, self.radius = float(n0), tuple(float(v) for v in center), float(radius)
        self.spec = ('sphere', self.n0, self.center[0], self.center[1], self.radius)


globals()['None'] = Empty
