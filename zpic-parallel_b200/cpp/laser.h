// laser.h -- Laser::{PlaneWave, Gaussian} (laser.h:8-131 of the reference)
#ifndef ZPIC_B200_LASER_H_
#define ZPIC_B200_LASER_H_

#include "emf.h"

namespace Laser {

class Pulse {
public:
    float start, fwhm, rise, flat, fall;
    float a0, omega0;
    float polarization, cos_pol, sin_pol;
    unsigned int filter;
    Pulse() : start( 0 ), fwhm( 0 ), rise( 0 ), flat( 0 ), fall( 0 ), a0( 0 ), omega0( 0 ),
              polarization( 0 ), cos_pol( 0 ), sin_pol( 0 ), filter( 1 ) {}
    virtual ~Pulse() = default;
    virtual zpic_laser_desc desc() const = 0;
    // Laser::Pulse::add (laser.h:85-99): 0 on success, -1 on invalid parameters
    virtual int add( EMF & emf ) {
        zpic_laser_desc d = desc();
        return zpic_b200_laser_add( emf.handle(), &d ) == ZPIC_OK ? 0 : -1;
    }
protected:
    zpic_laser_desc base( int type ) const {
        zpic_laser_desc d{};
        d.type = type; d.start = start; d.fwhm = fwhm; d.rise = rise; d.flat = flat; d.fall = fall;
        d.a0 = a0; d.omega0 = omega0; d.polarization = polarization; d.cos_pol = cos_pol; d.sin_pol = sin_pol;
        d.filter = filter;
        return d;
    }
};

class PlaneWave : public Pulse {
public:
    zpic_laser_desc desc() const override { return base( ZPIC_LASER_PLANE ); }
};

class Gaussian : public Pulse {
public:
    float W0, focus, axis;
    Gaussian() : Pulse(), W0( 0 ), focus( 0 ), axis( 0 ) {}
    zpic_laser_desc desc() const override {
        zpic_laser_desc d = base( ZPIC_LASER_GAUSSIAN );
        d.W0 = W0; d.focus = focus; d.axis = axis;
        return d;
    }
};

}  // namespace Laser

#endif
