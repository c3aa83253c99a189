// host_init.h -- host-side initial conditions of the em2d step: density
// injection, momentum distributions (with the reference's MWC generator and
// polar Box-Muller normals) and laser pulses.  They run once per species /
// laser on the host with the C library's double-precision math, exactly as
// the reference does (density.cpp, udist.cpp, random.h, laser.cpp), and the
// results are uploaded to the device.
#pragma once

#include <cstdint>
#include <vector>

#include "zpic_b200.h"

namespace zbhost {

struct TileGeom {
    int ntx, nty, nxx, nxy;
    int ntiles() const { return ntx * nty; }
};

// Injection rule for one density profile at window motion `motion`
// (Species::inject / np_inject, species.cpp:1806-1842).
struct Injector {
    zpic_density dens;
    uint32_t ppc[2];
    float dx[2];
    double motion;
    TileGeom g;
    int type() const { return dens.type; }
    // Step/Slab along y visit tiles tx < ntiles.y only (density.cpp:438, 470, 692)
    int tx_limit() const;
    // normalised step position / slab limits / shifted sphere centre
    void rule_params( float & a, float & b, float & cx, float & cy, float & r2 ) const;
    // Density::*::np_inject: particles per tile for the global cell range
    void count( const unsigned range[4], int * np ) const;
    // Density::*::inject: appends particles of the range to packed per-tile
    // storage (ix: 2 ints, x: 2 floats, u: 3 floats, at offset[t] + np[t])
    void inject( const unsigned range[4], const int * offset, int * np,
                 int32_t * ix, float * x, float * u ) const;
};

// UDistribution::*::set (udist.cpp:10-136) on packed per-tile storage.
void udist_set( const zpic_udist & ud, unsigned seed, const TileGeom & g,
                const int * offset, const int * np, const int32_t * ix, float * u );

// Laser::Pulse::launch (laser.cpp:225-443) into tiled E and B buffers with
// guard cells {1,2} (tile_vol floats3 per tile), periodic guard refresh,
// optional compensated filter and divergence correction, as Laser::Pulse::add
// builds its temporary grids (laser.h:85-99).  Returns 0 or -1 (invalid).
int laser_fields( zpic_laser_desc l, const TileGeom & g, const float box[2],
                  std::vector<float> & E, std::vector<float> & B );

// Run f(begin, end) over [0, n) on the host's cores.
void parallel_for( int n, void ( *f )( int, int, void * ), void * ctx );

}  // namespace zbhost
