// udist.h -- UDistribution::{None, Cold, Thermal, ThermalCorr} (udist.h:11-58 of the reference)
#ifndef ZPIC_B200_UDIST_H_
#define ZPIC_B200_UDIST_H_

#include "zpic.h"

namespace UDistribution {

class Type {
public:
    virtual Type * clone() const = 0;
    virtual zpic_udist desc() const = 0;
    virtual ~Type() = default;
};

class None : public Type {
public:
    None * clone() const override { return new None(); }
    zpic_udist desc() const override { return { ZPIC_UDIST_NONE, { 0, 0, 0 }, { 0, 0, 0 }, 2 }; }
};

class Cold : public Type {
public:
    const float3 ufl;
    Cold( float3 const ufl ) : ufl( ufl ) {}
    Cold * clone() const override { return new Cold( ufl ); }
    zpic_udist desc() const override { return { ZPIC_UDIST_COLD, { 0, 0, 0 }, { ufl.x, ufl.y, ufl.z }, 2 }; }
};

class Thermal : public Type {
public:
    const float3 uth, ufl;
    Thermal( float3 const uth, float3 const ufl ) : uth( uth ), ufl( ufl ) {}
    Thermal * clone() const override { return new Thermal( uth, ufl ); }
    zpic_udist desc() const override { return { ZPIC_UDIST_THERMAL, { uth.x, uth.y, uth.z }, { ufl.x, ufl.y, ufl.z }, 2 }; }
};

class ThermalCorr : public Type {
public:
    const float3 uth, ufl; const int npmin;
    ThermalCorr( float3 const uth, float3 const ufl, int const npmin = 2 ) : uth( uth ), ufl( ufl ), npmin( npmin ) {
        if ( npmin <= 1 ) { std::cout << "(*error*) invalid npmin parameter, must be > 1\n"; std::exit( 1 ); }
    }
    ThermalCorr * clone() const override { return new ThermalCorr( uth, ufl, npmin ); }
    zpic_udist desc() const override {
        return { ZPIC_UDIST_THERMALCORR, { uth.x, uth.y, uth.z }, { ufl.x, ufl.y, ufl.z }, npmin };
    }
};

}  // namespace UDistribution

#endif
