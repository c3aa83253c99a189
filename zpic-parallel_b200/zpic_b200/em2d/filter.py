"""Digital current filters of the Python em2d interface (the reference's
em2d.filter module, openmp/python/em2d/filter/filter.pyx): None, Binomial,
Compensated.  ``None`` is reached as ``getattr(filter, 'None')`` (or
``filter.Off``)."""

_DIR = {'x': 0, 'y': 1}


class Off:
    """None(): no filtering."""
    kind, direction, level = 'none', 0, 1


class Binomial:
    """Binomial( dir, level = 1 ): (1,2,1)/4 passes along dir."""

    def __init__(self, dir, level=1):
        self.kind, self.direction, self.level = 'binomial', _DIR[dir], int(level)


class Compensated:
    """Compensated( dir, level = 1 ): binomial passes plus the compensator."""

    def __init__(self, dir, level=1):
        self.kind, self.direction, self.level = 'compensated', _DIR[dir], int(level)


globals()['None'] = Off
