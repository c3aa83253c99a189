// density.h -- Density::{None, Uniform, Step, Slab, Sphere} (density.h:12-131 of the reference)
#ifndef ZPIC_B200_DENSITY_H_
#define ZPIC_B200_DENSITY_H_

#include "zpic.h"

namespace Density {

class Profile {
public:
    const float n0;
    Profile( float const n0 ) : n0( std::abs( n0 ) ) {}
    virtual Profile * clone() const = 0;
    virtual zpic_density desc() const = 0;
    virtual ~Profile() = default;
};

class None : public Profile {
public:
    None() : Profile( 0.f ) {}
    None * clone() const override { return new None(); }
    zpic_density desc() const override { return { ZPIC_DENSITY_NONE, 0.f, 0, 0, 0, 0 }; }
};

class Uniform : public Profile {
public:
    Uniform( float const n0 ) : Profile( n0 ) {}
    Uniform * clone() const override { return new Uniform( n0 ); }
    zpic_density desc() const override { return { ZPIC_DENSITY_UNIFORM, n0, 0, 0, 0, 0 }; }
};

class Step : public Profile {
public:
    const float pos; const coord::cart dir;
    Step( coord::cart dir, float const n0, float const pos ) : Profile( n0 ), pos( pos ), dir( dir ) {}
    Step * clone() const override { return new Step( dir, n0, pos ); }
    zpic_density desc() const override { return { ZPIC_DENSITY_STEP, n0, pos, 0, 0, (int32_t) dir }; }
};

class Slab : public Profile {
public:
    const float begin, end; const coord::cart dir;
    Slab( coord::cart dir, float const n0, float begin, float end ) : Profile( n0 ), begin( begin ), end( end ), dir( dir ) {}
    Slab * clone() const override { return new Slab( dir, n0, begin, end ); }
    zpic_density desc() const override { return { ZPIC_DENSITY_SLAB, n0, begin, end, 0, (int32_t) dir }; }
};

class Sphere : public Profile {
public:
    const float2 center; const float radius;
    Sphere( float const n0, float2 center, float radius ) : Profile( n0 ), center( center ), radius( radius ) {}
    Sphere * clone() const override { return new Sphere( n0, center, radius ); }
    zpic_density desc() const override { return { ZPIC_DENSITY_SPHERE, n0, center.x, center.y, radius, 0 }; }
};

}  // namespace Density

#endif
