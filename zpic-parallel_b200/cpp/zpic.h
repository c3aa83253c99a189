// zpic.h -- common definitions of the drop-in C++ API over libzpic_b200.so
// (the reference's openmp/em2d/zpic.h, utils.h and timer.h roles).
#ifndef ZPIC_B200_ZPIC_H_
#define ZPIC_B200_ZPIC_H_

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <string>

#include "zpic_b200.h"
#include "vec_types.h"
#include "bnd.h"

namespace coord { enum cart { x = 0, y }; }
namespace fcomp { enum cart { x = 0, y, z }; }
namespace part { enum quant { x = 0, y, ux, uy, uz }; }

namespace zpic {

// Courant limit (zpic.h:59-73)
inline float courant( const float2 dx ) { return std::sqrt( 1.0f / ( 1.0f / ( dx.x * dx.x ) + 1.0f / ( dx.y * dx.y ) ) ); }
inline float courant( const uint2 gnx, const float2 box ) { return courant( make_float2( box.x / gnx.x, box.y / gnx.y ) ); }
inline float courant( const uint2 ntiles, const uint2 nx, const float2 box ) {
    return courant( make_float2( box.x / ( nx.x * ntiles.x ), box.y / ( nx.y * ntiles.y ) ) );
}

// Library errors follow the reference's convention: print "(*error*)" and exit.
inline void check( int rc ) {
    if ( rc != ZPIC_OK ) {
        std::cerr << "(*error*) " << zpic_b200_last_error() << '\n';
        std::exit( 1 );
    }
}

inline void sys_info() { std::cout << "B200 (sm_100a) em2d library, version " << zpic_b200_version() << '\n'; }

}  // namespace zpic

namespace ansi {
static const std::string bold( "\033[1m" );
static const std::string reset( "\033[0m" );
}

namespace timer { enum units { s, ms, us, ns }; }

// Wall-clock timer (timer.h:12-107)
class Timer {
    std::chrono::steady_clock::time_point t0, t1;
public:
    void start() { t0 = std::chrono::steady_clock::now(); }
    void stop() { t1 = std::chrono::steady_clock::now(); }
    double elapsed( timer::units u = timer::s ) const {
        const double s = std::chrono::duration<double>( t1 - t0 ).count();
        switch ( u ) { case timer::ms: return s * 1e3; case timer::us: return s * 1e6; case timer::ns: return s * 1e9; default: return s; }
    }
};

#endif
