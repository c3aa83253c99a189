// host_init.cpp -- host-side initial conditions (see host_init.h).
//
// Compiled with -ffp-contract=off: plain IEEE operations in source order, as
// the reference's g++ -std=c++17 build evaluates them.
#include "host_init.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <thread>

namespace zbhost {

void parallel_for( int n, void ( *f )( int, int, void * ), void * ctx ) {
    unsigned nt = std::thread::hardware_concurrency();
    if ( nt == 0 ) nt = 1;
    if ( n < 64 || nt == 1 ) { f( 0, n, ctx ); return; }
    nt = std::min<unsigned>( nt, 64 );
    std::vector<std::thread> th;
    const int per = ( n + nt - 1 ) / nt;
    for ( unsigned k = 0; k < nt; k++ ) {
        const int b = k * per, e = std::min( n, b + per );
        if ( b >= e ) break;
        th.emplace_back( f, b, e, ctx );
    }
    for ( auto & t : th ) t.join();
}

// ---------------------------------------------------------------------------
// Density profiles (density.cpp)
// ---------------------------------------------------------------------------
int Injector::tx_limit() const {
    if ( ( dens.type == ZPIC_DENSITY_STEP || dens.type == ZPIC_DENSITY_SLAB ) && dens.dir != 0 )
        return std::min( g.nty, g.ntx );
    return g.ntx;
}

void Injector::rule_params( float & a, float & b, float & cx, float & cy, float & r2 ) const {
    const float refx = (float) motion;          // make_float2( moving_window.motion(), 0 )
    a = b = cx = cy = r2 = 0;
    switch ( dens.type ) {
    case ZPIC_DENSITY_STEP: a = ( dens.a - refx ) / dx[0]; break;                       // density.cpp:418
    case ZPIC_DENSITY_SLAB: a = ( dens.a - refx ) / dx[0]; b = ( dens.b - refx ) / dx[0]; break;  // 677-678
    case ZPIC_DENSITY_SPHERE: cx = dens.a - refx; cy = dens.b - 0.0f; r2 = dens.c * dens.c; break; // 937-941, 875
    default: break;
    }
}

static bool tile_range( const TileGeom & g, int tx, int ty, const unsigned range[4],
                        int & ri0, int & ri1, int & rj0, int & rj1 ) {
    ri0 = range[0] - tx * g.nxx; ri1 = range[1] - tx * g.nxx;
    rj0 = range[2] - ty * g.nxy; rj1 = range[3] - ty * g.nxy;
    if ( ( ri0 < g.nxx ) && ( ri1 >= 0 ) && ( rj0 < g.nxy ) && ( rj1 >= 0 ) ) {
        if ( ri0 < 0 ) ri0 = 0;
        if ( rj0 < 0 ) rj0 = 0;
        if ( ri1 >= g.nxx ) ri1 = g.nxx - 1;
        if ( rj1 >= g.nxy ) rj1 = g.nxy - 1;
        return true;
    }
    return false;
}

static inline int inj_test( int type, int diry, float a, float b, float cx, float cy, float r2,
                            const float dx[2], int shiftx, int shifty, int cellx, int celly, float posx, float posy ) {
    float t;
    switch ( type ) {
    case ZPIC_DENSITY_UNIFORM: return 1;
    case ZPIC_DENSITY_STEP:
        t = diry ? ( shifty + celly ) + ( posy + 0.5 ) : ( shiftx + cellx ) + ( posx + 0.5 );
        return t > a;
    case ZPIC_DENSITY_SLAB:
        t = diry ? ( shifty + celly ) + ( posy + 0.5 ) : ( shiftx + cellx ) + ( posx + 0.5 );
        return ( t >= a ) && ( t < b );
    case ZPIC_DENSITY_SPHERE: {
        float gx = ( ( shiftx + cellx ) + ( posx + 0.5 ) ) * dx[0];
        float gy = ( ( shifty + celly ) + ( posy + 0.5 ) ) * dx[1];
        return ( gx - cx ) * ( gx - cx ) + ( gy - cy ) * ( gy - cy ) < r2;
    }
    }
    return 0;
}

void Injector::count( const unsigned range[4], int * np ) const {
    if ( dens.type == ZPIC_DENSITY_NONE ) return;   // density.h:39-42 leaves np untouched
    float a, b, cx, cy, r2;
    rule_params( a, b, cx, cy, r2 );
    const double dpcx = 1.0 / ppc[0], dpcy = 1.0 / ppc[1];
    const int txl = tx_limit();
    for ( int ty = 0; ty < g.nty; ty++ ) for ( int tx = 0; tx < txl; tx++ ) {
        const int tid = ty * g.ntx + tx;
        int ri0, ri1, rj0, rj1, n = 0;
        if ( tile_range( g, tx, ty, range, ri0, ri1, rj0, rj1 ) ) {
            const int row = ri1 - ri0 + 1, vol = ( rj1 - rj0 + 1 ) * row;
            if ( dens.type == ZPIC_DENSITY_UNIFORM ) n = vol * ppc[0] * ppc[1];
            else {
                const int shiftx = tx * g.nxx, shifty = ty * g.nxy;
                for ( int idx = 0; idx < vol; idx++ )
                    for ( unsigned i1 = 0; i1 < ppc[1]; i1++ )
                        for ( unsigned i0 = 0; i0 < ppc[0]; i0++ ) {
                            const float posx = dpcx * ( i0 + 0.5 ) - 0.5, posy = dpcy * ( i1 + 0.5 ) - 0.5;
                            n += inj_test( dens.type, dens.dir, a, b, cx, cy, r2, dx, shiftx, shifty,
                                           idx % row + ri0, idx / row + rj0, posx, posy );
                        }
            }
        }
        np[tid] = n;
    }
}

namespace {
struct InjCtx {
    const Injector * self; const unsigned * range; const int * offset; int * np;
    int32_t * ix; float * x; float * u;
    float a, b, cx, cy, r2;
};
void inject_tiles( int t0, int t1, void * pv ) {
    InjCtx & c = *static_cast<InjCtx *>( pv );
    const Injector & I = *c.self;
    const TileGeom & g = I.g;
    const double dpcx = 1.0 / I.ppc[0], dpcy = 1.0 / I.ppc[1];
    const int txl = I.tx_limit();
    for ( int tid = t0; tid < t1; tid++ ) {
        const int tx = tid % g.ntx, ty = tid / g.ntx;
        if ( tx >= txl ) continue;
        int ri0, ri1, rj0, rj1;
        if ( !tile_range( g, tx, ty, c.range, ri0, ri1, rj0, rj1 ) ) continue;
        const int row = ri1 - ri0 + 1, vol = ( rj1 - rj0 + 1 ) * row;
        int np = c.np[tid];
        const size_t base = c.offset[tid];
        const int shiftx = tx * g.nxx, shifty = ty * g.nxy;
        for ( unsigned i1 = 0; i1 < I.ppc[1]; i1++ )
            for ( unsigned i0 = 0; i0 < I.ppc[0]; i0++ ) {
                const float posx = dpcx * ( i0 + 0.5 ) - 0.5, posy = dpcy * ( i1 + 0.5 ) - 0.5;
                const int ppc_idx = i1 * I.ppc[0] + i0;
                for ( int idx = 0; idx < vol; idx++ ) {
                    const int cellx = idx % row + ri0, celly = idx / row + rj0;
                    int k;
                    if ( I.dens.type == ZPIC_DENSITY_UNIFORM ) k = np + vol * ppc_idx + idx;   // mk2 order
                    else {
                        if ( !inj_test( I.dens.type, I.dens.dir, c.a, c.b, c.cx, c.cy, c.r2, I.dx,
                                        shiftx, shifty, cellx, celly, posx, posy ) ) continue;
                        k = np++;
                    }
                    const size_t p = base + k;
                    c.ix[2*p] = cellx; c.ix[2*p+1] = celly;
                    c.x[2*p] = posx;   c.x[2*p+1] = posy;
                    c.u[3*p] = 0; c.u[3*p+1] = 0; c.u[3*p+2] = 0;
                }
            }
        c.np[tid] = ( I.dens.type == ZPIC_DENSITY_UNIFORM ) ? np + vol * (int) ( I.ppc[0] * I.ppc[1] ) : np;
    }
}
}  // namespace

void Injector::inject( const unsigned range[4], const int * offset, int * np,
                       int32_t * ix, float * x, float * u ) const {
    if ( dens.type == ZPIC_DENSITY_NONE ) return;
    InjCtx c{ this, range, offset, np, ix, x, u, 0, 0, 0, 0, 0 };
    rule_params( c.a, c.b, c.cx, c.cy, c.r2 );
    parallel_for( g.ntiles(), inject_tiles, &c );
}

// ---------------------------------------------------------------------------
// Random numbers (random.h:23-155) and momentum distributions (udist.cpp)
// ---------------------------------------------------------------------------
namespace {
struct Rng {
    unsigned x, y; double norm;
    Rng( int global_id, unsigned sx, unsigned sy ) {
        norm = DBL_MAX;
        x = sx + global_id;
        y = sy + ( ( global_id ) ^ ( 0xFFFFFFFF ) );
    }
    unsigned next() {
        x = 36969 * ( x & 65535 ) + ( x >> 16 );
        y = 18000 * ( y & 65535 ) + ( y >> 16 );
        return ( x << 16 ) + y;
    }
    double real3() { return ( next() + 1.0 ) * 0x1.fffffffep-33; }
    double normal() {
        double res;
        if ( norm == DBL_MAX ) {
            double v1, v2, rsq, fac;
            do {
                v1 = real3() * 2.0 - 1.0;
                v2 = real3() * 2.0 - 1.0;
                rsq = v1 * v1 + v2 * v2;
            } while ( rsq == 0.0 || rsq >= 1.0 );
            fac = std::sqrt( -2.0 * std::log( rsq ) / rsq );
            norm = v1 * fac;
            res = v2 * fac;
        } else {
            res = norm;
            norm = DBL_MAX;
        }
        return res;
    }
};

struct UdCtx {
    zpic_udist ud; unsigned seed; TileGeom g;
    const int * offset; const int * np; const int32_t * ix; float * u;
};

// The reference builds each momentum as make_float3( f(), f(), f() ); g++
// evaluates those arguments right to left, so the first normal of a
// particle goes to u.z (udist.cpp:58-62, 101-105).
void udist_tiles( int t0, int t1, void * pv ) {
    UdCtx & c = *static_cast<UdCtx *>( pv );
    const zpic_udist & ud = c.ud;
    const unsigned sx = 12345 + c.seed, sy = 67890;
    std::vector<float> fluid;
    std::vector<int> npcell;
    for ( int tid = t0; tid < t1; tid++ ) {
        const size_t off = c.offset[tid];
        const int np = c.np[tid];
        float * u = c.u + 3 * off;
        const int32_t * ix = c.ix + 2 * off;
        if ( ud.type == ZPIC_UDIST_NONE || ud.type == ZPIC_UDIST_COLD ) {
            for ( int i = 0; i < np; i++ ) {
                u[3*i]   = ud.type == ZPIC_UDIST_COLD ? ud.ufl[0] : 0.f;
                u[3*i+1] = ud.type == ZPIC_UDIST_COLD ? ud.ufl[1] : 0.f;
                u[3*i+2] = ud.type == ZPIC_UDIST_COLD ? ud.ufl[2] : 0.f;
            }
        } else if ( ud.type == ZPIC_UDIST_THERMAL ) {
            Rng r( tid, sx, sy );
            for ( int i = 0; i < np; i++ ) {
                const float z = ud.ufl[2] + ud.uth[2] * r.normal();
                const float y = ud.ufl[1] + ud.uth[1] * r.normal();
                const float x = ud.ufl[0] + ud.uth[0] * r.normal();
                u[3*i] = x; u[3*i+1] = y; u[3*i+2] = z;
            }
        } else {
            const int bsize = c.g.nxx * c.g.nxy, ystride = c.g.nxx;
            fluid.assign( 3 * bsize, 0.f );
            npcell.assign( bsize, 0 );
            Rng r( tid, sx, sy );
            for ( int i = 0; i < np; i++ ) {
                const float z = ud.uth[2] * r.normal();
                const float y = ud.uth[1] * r.normal();
                const float x = ud.uth[0] * r.normal();
                u[3*i] = x; u[3*i+1] = y; u[3*i+2] = z;
                const int idx = ix[2*i] + ystride * ix[2*i+1];
                npcell[idx] += 1;
                fluid[3*idx] += x; fluid[3*idx+1] += y; fluid[3*idx+2] += z;
            }
            for ( int idx = 0; idx < bsize; idx++ ) {
                if ( npcell[idx] > ud.npmin ) {
                    fluid[3*idx] /= npcell[idx]; fluid[3*idx+1] /= npcell[idx]; fluid[3*idx+2] /= npcell[idx];
                } else {
                    fluid[3*idx] = fluid[3*idx+1] = fluid[3*idx+2] = 0.f;
                }
            }
            for ( int i = 0; i < np; i++ ) {
                const int idx = ix[2*i] + ystride * ix[2*i+1];
                u[3*i]   += ud.ufl[0] - fluid[3*idx];
                u[3*i+1] += ud.ufl[1] - fluid[3*idx+1];
                u[3*i+2] += ud.ufl[2] - fluid[3*idx+2];
            }
        }
    }
}
}  // namespace

void udist_set( const zpic_udist & ud, unsigned seed, const TileGeom & g,
                const int * offset, const int * np, const int32_t * ix, float * u ) {
    UdCtx c{ ud, seed, g, offset, np, ix, u };
    parallel_for( g.ntiles(), udist_tiles, &c );
}

// ---------------------------------------------------------------------------
// Lasers (laser.h:46-64, laser.cpp)
// ---------------------------------------------------------------------------
namespace {
constexpr int GL = 1, GU = 2;

struct HGrid {
    TileGeom g; int extx, exty, off, tv;
    std::vector<float> * buf;
    float * cell( int tid, int c ) { return buf->data() + ( (size_t) tid * tv + c ) * 3; }
};

float lon_env( const zpic_laser_desc & l, float z ) {
    if ( z > l.start ) return 0.0f;
    else if ( z > l.start - l.rise ) {
        float csi = z - l.start;
        float e = std::sin( M_PI_2 * csi / l.rise );
        return e * e;
    } else if ( z > l.start - ( l.rise + l.flat ) ) return 1.0f;
    else if ( z > l.start - ( l.rise + l.flat + l.fall ) ) {
        float csi = z - ( l.start - l.rise - l.flat - l.fall );
        float e = std::sin( M_PI_2 * csi / l.fall );
        return e * e;
    }
    return 0.0f;
}

// laser.cpp:318-330; atan2 on floats resolves to the double overload
float gauss_phase( float omega0, float W0, float z, float r ) {
    const float z0 = omega0 * ( W0 * W0 ) / 2;
    const float rho2 = r * r;
    const float curv = rho2 * z / ( z0 * z0 + z * z );
    const float rWl2 = ( z0 * z0 ) / ( z0 * z0 + z * z );
    const float gouy_shift = ::atan2( (double) z, (double) z0 );
    return std::sqrt( std::sqrt( rWl2 ) ) * std::exp( -rho2 * rWl2 / ( W0 * W0 ) ) *
           std::cos( omega0 * ( z + curv ) - gouy_shift );
}

// grid.h:253-340, periodic
void copy_to_gc( HGrid & h, int axes ) {
    const TileGeom & g = h.g;
    if ( axes & 1 )
        for ( int tid = 0; tid < g.ntiles(); tid++ ) {
            const int tx = tid % g.ntx, ty = tid / g.ntx;
            const int lo = ty * g.ntx + ( tx - 1 + g.ntx ) % g.ntx, hi = ty * g.ntx + ( tx + 1 ) % g.ntx;
            for ( int j = 0; j < h.exty; j++ ) {
                for ( int i = 0; i < GL; i++ ) std::memcpy( h.cell( tid, i + j * h.extx ), h.cell( lo, g.nxx + i + j * h.extx ), 12 );
                for ( int i = 0; i < GU; i++ ) std::memcpy( h.cell( tid, GL + g.nxx + i + j * h.extx ), h.cell( hi, GL + i + j * h.extx ), 12 );
            }
        }
    if ( axes & 2 )
        for ( int tid = 0; tid < g.ntiles(); tid++ ) {
            const int tx = tid % g.ntx, ty = tid / g.ntx;
            const int lo = ( ( ty - 1 + g.nty ) % g.nty ) * g.ntx + tx, hi = ( ( ty + 1 ) % g.nty ) * g.ntx + tx;
            for ( int j = 0; j < GL; j++ )
                for ( int i = 0; i < h.extx; i++ ) std::memcpy( h.cell( tid, i + j * h.extx ), h.cell( lo, i + ( g.nxy + j ) * h.extx ), 12 );
            for ( int j = 0; j < GU; j++ )
                for ( int i = 0; i < h.extx; i++ )
                    std::memcpy( h.cell( tid, i + ( GL + g.nxy + j ) * h.extx ), h.cell( hi, i + ( GL + j ) * h.extx ), 12 );
        }
}

// grid.h:495-541 kernel3_x followed by copy_to_gc_x
void kernel3_x( HGrid & h, float a, float b, float c ) {
    std::vector<float> A( (size_t) h.tv * 3 );
    for ( int tid = 0; tid < h.g.ntiles(); tid++ ) {
        float * buf = h.cell( tid, 0 );
        std::memcpy( A.data(), buf, A.size() * sizeof( float ) );
        for ( int iy = 0; iy < h.exty; iy++ )
            for ( int ix = GL; ix < GL + h.g.nxx; ix++ )
                for ( int k = 0; k < 3; k++ )
                    buf[3 * ( iy * h.extx + ix ) + k] = A[3 * ( iy * h.extx + ix - 1 ) + k] * a +
                                                       A[3 * ( iy * h.extx + ix ) + k] * b +
                                                       A[3 * ( iy * h.extx + ix + 1 ) + k] * c;
    }
    copy_to_gc( h, 1 );
}

// laser.cpp:20-70; tile rows are independent (the sums run along x), so
// they are spread over host threads when there are enough of them
struct DivCorrCtx { HGrid * E; HGrid * B; double dx_dy; };

void div_corr_rows( int ty0, int ty1, void * vctx ) {
    DivCorrCtx & c = *static_cast<DivCorrCtx *>( vctx );
    HGrid & E = *c.E;
    HGrid & B = *c.B;
    const TileGeom & g = E.g;
    const int ys = E.extx;
    const double dx_dy = c.dx_dy;
    std::vector<double> divEx( g.nxy ), divBx( g.nxy );
    for ( int ty = ty0; ty < ty1; ty++ ) {
        std::fill( divEx.begin(), divEx.end(), 0.0 );
        std::fill( divBx.begin(), divBx.end(), 0.0 );
        for ( int tx = g.ntx - 1; tx >= 0; tx-- ) {
            const int tid = ty * g.ntx + tx;
            float * tE = E.cell( tid, E.off );
            float * tB = B.cell( tid, B.off );
            for ( int iy = 0; iy < g.nxy; iy++ ) {
                double a = divEx[iy], b = divBx[iy];
                for ( int ix = g.nxx - 1; ix >= 0; ix-- ) {
                    a += dx_dy * ( tE[3 * ( ix + 1 + iy * ys ) + 1] - tE[3 * ( ix + 1 + ( iy - 1 ) * ys ) + 1] );
                    tE[3 * ( ix + iy * ys )] = a;
                    b += dx_dy * ( tB[3 * ( ix + ( iy + 1 ) * ys ) + 1] - tB[3 * ( ix + iy * ys ) + 1] );
                    tB[3 * ( ix + iy * ys )] = b;
                }
                divEx[iy] = a; divBx[iy] = b;
            }
        }
    }
}

void div_corr_x( HGrid & E, HGrid & B, const float dx[2] ) {
    DivCorrCtx c{ &E, &B, ( (double) dx[0] ) / ( (double) dx[1] ) };
    parallel_for( E.g.nty, div_corr_rows, &c );
}

// The pulse's fields, cell by cell (laser.cpp:233-292 plane wave,
// 361-443 Gaussian), for tiles [t0, t1): every value depends on its own cell
// only, so tiles are spread over host threads.
struct PulseCtx { const zpic_laser_desc * l; HGrid * E; HGrid * B; float dx[2]; };

void pulse_tiles( int t0, int t1, void * vctx ) {
    PulseCtx & c = *static_cast<PulseCtx *>( vctx );
    const zpic_laser_desc & l = *c.l;
    HGrid & E = *c.E;
    HGrid & B = *c.B;
    const TileGeom & g = E.g;
    const float * dx = c.dx;
    const int ys = E.extx;
    const float amp = l.omega0 * l.a0;
    for ( int tid = t0; tid < t1; tid++ ) {
        const int tx = tid % g.ntx, ty = tid / g.ntx;
        float * pE = E.cell( tid, E.off );
        float * pB = B.cell( tid, B.off );
        const int ix0 = tx * g.nxx, iy0 = ty * g.nxy;
        for ( unsigned iy = 0; iy < (unsigned) g.nxy; iy++ )
            for ( unsigned ix = 0; ix < (unsigned) g.nxx; ix++ ) {
                const float z = ( ix0 + ix ) * dx[0];
                const float z_2 = ( ix0 + ix + 0.5 ) * dx[0];
                const float lenv = amp * lon_env( l, z ), lenv_2 = amp * lon_env( l, z_2 );
                float * e = pE + 3 * ( ix + iy * ys );
                float * b = pB + 3 * ( ix + iy * ys );
                if ( l.type == ZPIC_LASER_PLANE ) {
                    const float k = l.omega0;
                    e[0] = 0; e[1] = +lenv * std::cos( k * z ) * l.cos_pol; e[2] = +lenv * std::cos( k * z ) * l.sin_pol;
                    b[0] = 0; b[1] = -lenv_2 * std::cos( k * z_2 ) * l.sin_pol; b[2] = +lenv_2 * std::cos( k * z_2 ) * l.cos_pol;
                } else {
                    const float r = ( iy0 + iy ) * dx[1] - l.axis;
                    const float r_2 = ( iy0 + iy + 0.5 ) * dx[1] - l.axis;
                    e[0] = 0;
                    e[1] = +lenv * gauss_phase( l.omega0, l.W0, z - l.focus, r_2 ) * l.cos_pol;
                    e[2] = +lenv * gauss_phase( l.omega0, l.W0, z - l.focus, r ) * l.sin_pol;
                    b[0] = 0;
                    b[1] = -lenv_2 * gauss_phase( l.omega0, l.W0, z_2 - l.focus, r ) * l.sin_pol;
                    b[2] = +lenv_2 * gauss_phase( l.omega0, l.W0, z_2 - l.focus, r_2 ) * l.cos_pol;
                }
            }
    }
}
}  // namespace

int laser_fields( zpic_laser_desc l, const TileGeom & g, const float box[2],
                  std::vector<float> & Ev, std::vector<float> & Bv ) {
    // Laser::Pulse::validate (laser.cpp:174-207), Gaussian::validate (299-310)
    if ( l.a0 <= 0 || l.omega0 <= 0 ) return -1;
    if ( l.fwhm > 0 ) { l.rise = l.fwhm; l.fall = l.fwhm; l.flat = 0.f; }
    else if ( l.rise <= 0 || l.flat < 0 || l.fall <= 0 ) return -1;
    if ( l.type == ZPIC_LASER_GAUSSIAN && l.W0 <= 0 ) return -1;
    if ( l.cos_pol == 0 && l.sin_pol == 0 ) {
        l.cos_pol = std::cos( l.polarization );
        l.sin_pol = std::sin( l.polarization );
    }
    HGrid E{ g, GL + g.nxx + GU, GL + g.nxy + GU, 0, 0, &Ev };
    E.off = GL * E.extx + GL;
    E.tv = ( E.extx * E.exty + 3 ) & ~3;
    HGrid B = E; B.buf = &Bv;
    Ev.assign( (size_t) E.tv * g.ntiles() * 3, 0.f );
    Bv.assign( (size_t) E.tv * g.ntiles() * 3, 0.f );
    const float dx[2] = { box[0] / ( g.nxx * g.ntx ), box[1] / ( g.nxy * g.nty ) };
    PulseCtx pc{ &l, &E, &B, { dx[0], dx[1] } };
    parallel_for( g.ntiles(), pulse_tiles, &pc );
    copy_to_gc( E, 3 );
    copy_to_gc( B, 3 );
    if ( l.filter > 0 ) {
        // Filter::Compensated( coord::x, filter ) (filter.h:54-80)
        const unsigned order = l.filter;
        const float a = -1.0f;
        const float bb = ( 4.0 + 2.0 * order ) / order;
        const float norm = 2 * a + bb;
        for ( HGrid * h : { &E, &B } ) {
            for ( unsigned i = 0; i < order; i++ ) kernel3_x( *h, 0.25f, 0.5f, 0.25f );
            kernel3_x( *h, a / norm, bb / norm, a / norm );
        }
    }
    if ( l.type == ZPIC_LASER_GAUSSIAN ) div_corr_x( E, B, dx );
    return 0;
}

}  // namespace zbhost
