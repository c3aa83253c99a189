"""Momentum distributions of the Python em2d interface (the reference's
em2d.udist module, openmp/python/em2d/udist/udist.pyx): None, Cold, Thermal,
ThermalCorr.  ``None`` is a Python keyword, so that class is reached as
``getattr(udist, 'None')`` (or ``udist.Frozen``)."""


class _UDist:
    spec = ('none',)


class Frozen(_UDist):
    """None(): zero fluid momentum and zero temperature."""
    spec = ('none',)


class Cold(_UDist):
    """Cold( ufl ): zero temperature, fluid momentum ufl = [x, y, z]."""

    def __init__(self, ufl):
        self.ufl = tuple(float(v) for v in ufl)
        self.spec = ('cold', self.ufl)


class Thermal(_UDist):
    """Thermal( uth, ufl ): Gaussian thermal spread uth around fluid momentum ufl."""

    def __init__(self, uth, ufl):
        self.uth = tuple(float(v) for v in uth)
        self.ufl = tuple(float(v) for v in ufl)
        self.spec = ('thermal', self.uth, self.ufl)


class ThermalCorr(_UDist):
    """ThermalCorr( uth, ufl, npmin = 2 ): thermal, with the local fluid
    momentum corrected in cells holding more than npmin particles."""

    def __init__(self, uth, ufl, npmin=2):
        self.uth = tuple(float(v) for v in uth)
        self.ufl = tuple(float(v) for v in ufl)
        self.npmin = int(npmin)
        self.spec = ('thermalcorr', self.uth, self.ufl, self.npmin)


globals()['None'] = Frozen
