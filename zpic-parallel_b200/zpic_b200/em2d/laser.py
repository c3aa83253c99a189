"""Laser pulses of the Python em2d interface (the reference's em2d.laser
module, openmp/python/em2d/laser/laser.pyx): PlaneWave and Gaussian with the
reference's keyword parameters; ``add(emf)`` launches the pulse into the
fields of the simulation the EMF view belongs to."""


class _Pulse:
    kind = 'plane'
    KEYS = ('start', 'fwhm', 'rise', 'flat', 'fall', 'a0', 'omega0', 'polarization', 'cos_pol', 'sin_pol')

    def __init__(self, **kw):
        for k in self.KEYS:
            setattr(self, k, float(kw.pop(k, 0.0)))
        if kw:
            raise TypeError('unknown laser parameters: %s' % ', '.join(kw))

    def add(self, emf):
        """add( emf ): add the pulse to the EMF object; returns 0, or -1 for
        invalid parameters (Laser::Pulse::add)."""
        return emf._sim._add_laser(self)


class PlaneWave(_Pulse):
    """PlaneWave( *, start, fwhm, rise, flat, fall, a0, omega0, polarization, cos_pol, sin_pol )."""
    kind = 'plane'


class Gaussian(_Pulse):
    """Gaussian( *, ..., W0, focus, axis ): the PlaneWave parameters plus the
    waist W0, the focal plane position and the propagation axis."""
    kind = 'gaussian'
    KEYS = _Pulse.KEYS + ('W0', 'focus', 'axis')
