/*
 * em2d_oracle.c -- plain-C restatement of the zpic-parallel openmp/em2d step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Not part of the product: only the
 * tests, __graft_entry__.smoke() and bench.py's CPU-baseline arms load it.
 *
 * Every function cites the reference file:line it restates (paths relative
 * to the zpic-parallel project, openmp/em2d/).  The restatement is serial and
 * follows the reference's loop orders, so with ORACLE_REAL=float it is
 * bit-exact with the reference's scalar build run on one OpenMP thread
 * (pinned in tests/test_oracle_pin.py against oracle/_ref).
 *
 * Floating-point rules mirrored from the reference build (g++ -std=c++17,
 * i.e. no implicit FMA contraction): explicit fused multiply-adds are
 * ops::fma -> std::fma (utils.h:105-136), everything else is plain IEEE
 * single operations in source order; double literals promote as in C++.
 */
#include "em2d_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#include <stdio.h>

#define r_fma(a, b, c) _Generic( (real) 0, float: fmaf, double: fma )( (a), (b), (c) )
#define r_sqrt(a)      _Generic( (real) 0, float: sqrtf, double: sqrt )( a )
#define r_sin(a)       _Generic( (real) 0, float: sinf, double: sin )( a )
#define r_cos(a)       _Generic( (real) 0, float: cosf, double: cos )( a )
#define r_exp(a)       _Generic( (real) 0, float: expf, double: exp )( a )

#ifndef M_PI_2
#define M_PI_2 1.57079632679489661923
#endif

typedef struct { real x, y; } real2;
typedef struct { real x, y, z; } real3;

static unsigned roundup4( unsigned n ) { return ( n + 3u ) & ~3u; }

int oracle_real_size( void ) { return (int) sizeof( real ); }

/* ======================================================================== */
/* Moving window (moving_window.h:1-57)                                     */
/* ======================================================================== */
typedef struct { int active; unsigned n_move; double dx; } omw;

static void mw_init( omw * m, real dx ) { m->active = 1; m->n_move = 0; m->dx = dx; }
static void mw_advance( omw * m ) { if ( m->active ) m->n_move++; }
static double mw_motion( const omw * m ) { return m->n_move * m->dx; }
static int mw_needs_move( const omw * m, double t ) {
    return m->active && ( t > m->dx * ( m->n_move + 1 ) );
}

/* ======================================================================== */
/* Tiled grid (grid.h:14-638, vec3grid.h)                                   */
/* ======================================================================== */
typedef struct {
    unsigned ntx, nty, nxx, nxy;
    unsigned gxl, gxu, gyl, gyu;
    unsigned extx, exty, offset, tile_vol;
    int perx, pery;
    int nc;                  /* 3 for vec3grid<float3>, 1 for grid<float> */
    real * buf;
} ogrid;

/* grid.h:77-92 */
static void grid_init( ogrid * g, unsigned ntx, unsigned nty, unsigned nxx, unsigned nxy,
                       unsigned gxl, unsigned gxu, unsigned gyl, unsigned gyu, int nc ) {
    g->ntx = ntx; g->nty = nty; g->nxx = nxx; g->nxy = nxy;
    g->gxl = gxl; g->gxu = gxu; g->gyl = gyl; g->gyu = gyu;
    g->extx = gxl + nxx + gxu; g->exty = gyl + nxy + gyu;
    g->offset = gyl * g->extx + gxl;
    g->tile_vol = roundup4( g->extx * g->exty );
    g->perx = g->pery = 1;
    g->nc = nc;
    g->buf = (real *) calloc( (size_t) g->tile_vol * ntx * nty * nc, sizeof( real ) );
}
static void grid_free( ogrid * g ) { free( g->buf ); g->buf = NULL; }
static size_t grid_cells( const ogrid * g ) { return (size_t) g->tile_vol * g->ntx * g->nty; }
static real * gcell( const ogrid * g, unsigned tid, int c ) {
    return g->buf + ( (size_t) tid * g->tile_vol + c ) * g->nc;
}
static void grid_zero( ogrid * g ) { memset( g->buf, 0, grid_cells( g ) * g->nc * sizeof( real ) ); }

static void cell_copy( const ogrid * g, real * dst, const real * src ) {
    for ( int k = 0; k < g->nc; k++ ) dst[k] = src[k];
}
static void cell_add( const ogrid * g, real * dst, const real * src ) {
    for ( int k = 0; k < g->nc; k++ ) dst[k] += src[k];
}

/* grid.h:253-296 */
static void grid_copy_to_gc_x( ogrid * g ) {
    const int ntx = g->ntx;
    for ( unsigned tid = 0; tid < g->ntx * g->nty; tid++ ) {
        int tx = tid % g->ntx, ty = tid / g->ntx;
        {
            int n = tx - 1;
            if ( g->perx && n < 0 ) n += ntx;
            if ( n >= 0 ) {
                unsigned nid = ty * g->ntx + n;
                for ( unsigned j = 0; j < g->exty; j++ )
                    for ( unsigned i = 0; i < g->gxl; i++ )
                        cell_copy( g, gcell( g, tid, i + j * g->extx ), gcell( g, nid, g->nxx + i + j * g->extx ) );
            }
        }
        {
            int n = tx + 1;
            if ( g->perx && n >= ntx ) n -= ntx;
            if ( n < ntx ) {
                unsigned nid = ty * g->ntx + n;
                for ( unsigned j = 0; j < g->exty; j++ )
                    for ( unsigned i = 0; i < g->gxu; i++ )
                        cell_copy( g, gcell( g, tid, g->gxl + g->nxx + i + j * g->extx ),
                                   gcell( g, nid, g->gxl + i + j * g->extx ) );
            }
        }
    }
}

/* grid.h:302-340 */
static void grid_copy_to_gc_y( ogrid * g ) {
    const int nty = g->nty;
    for ( unsigned tid = 0; tid < g->ntx * g->nty; tid++ ) {
        int tx = tid % g->ntx, ty = tid / g->ntx;
        {
            int n = ty - 1;
            if ( g->pery && n < 0 ) n += nty;
            if ( n >= 0 ) {
                unsigned nid = n * g->ntx + tx;
                for ( unsigned j = 0; j < g->gyl; j++ )
                    for ( unsigned i = 0; i < g->extx; i++ )
                        cell_copy( g, gcell( g, tid, i + j * g->extx ), gcell( g, nid, i + ( g->nxy + j ) * g->extx ) );
            }
        }
        {
            int n = ty + 1;
            if ( g->pery && n >= nty ) n -= nty;
            if ( n < nty ) {
                unsigned nid = n * g->ntx + tx;
                for ( unsigned j = 0; j < g->gyu; j++ )
                    for ( unsigned i = 0; i < g->extx; i++ )
                        cell_copy( g, gcell( g, tid, i + ( g->gyl + g->nxy + j ) * g->extx ),
                                   gcell( g, nid, i + ( g->gyl + j ) * g->extx ) );
            }
        }
    }
}

/* grid.h:346-354 */
static void grid_copy_to_gc( ogrid * g ) { grid_copy_to_gc_x( g ); grid_copy_to_gc_y( g ); }

/* grid.h:360-445 (x pass over all tiles, then y pass) */
static void grid_add_from_gc( ogrid * g ) {
    const int ntx = g->ntx, nty = g->nty;
    for ( unsigned tid = 0; tid < g->ntx * g->nty; tid++ ) {
        int tx = tid % g->ntx, ty = tid / g->ntx;
        {
            int n = tx - 1;
            if ( g->perx && n < 0 ) n += ntx;
            if ( n >= 0 ) {
                unsigned nid = ty * g->ntx + n;
                for ( unsigned j = 0; j < g->exty; j++ )
                    for ( unsigned i = 0; i < g->gxu; i++ )
                        cell_add( g, gcell( g, tid, g->gxl + i + j * g->extx ),
                                  gcell( g, nid, g->gxl + g->nxx + i + j * g->extx ) );
            }
        }
        {
            int n = tx + 1;
            if ( g->perx && n >= ntx ) n -= ntx;
            if ( n < ntx ) {
                unsigned nid = ty * g->ntx + n;
                for ( unsigned j = 0; j < g->exty; j++ )
                    for ( unsigned i = 0; i < g->gxl; i++ )
                        cell_add( g, gcell( g, tid, g->nxx + i + j * g->extx ), gcell( g, nid, i + j * g->extx ) );
            }
        }
    }
    for ( unsigned tid = 0; tid < g->ntx * g->nty; tid++ ) {
        int tx = tid % g->ntx, ty = tid / g->ntx;
        {
            int n = ty - 1;
            if ( g->pery && n < 0 ) n += nty;
            if ( n >= 0 ) {
                unsigned nid = n * g->ntx + tx;
                for ( unsigned j = 0; j < g->gyu; j++ )
                    for ( unsigned i = 0; i < g->extx; i++ )
                        cell_add( g, gcell( g, tid, i + ( g->gyl + j ) * g->extx ),
                                  gcell( g, nid, i + ( g->gyl + g->nxy + j ) * g->extx ) );
            }
        }
        {
            int n = ty + 1;
            if ( g->pery && n >= nty ) n -= nty;
            if ( n < nty ) {
                unsigned nid = n * g->ntx + tx;
                for ( unsigned j = 0; j < g->gyl; j++ )
                    for ( unsigned i = 0; i < g->extx; i++ )
                        cell_add( g, gcell( g, tid, i + ( g->nxy + j ) * g->extx ), gcell( g, nid, i + j * g->extx ) );
            }
        }
    }
}

/* grid.h:455-485 */
static void grid_x_shift_left( ogrid * g, unsigned shift ) {
    if ( !( shift > 0 && shift < g->gxu ) ) {
        fprintf( stderr, "x_shift_left(), invalid shift value\n" );
        exit( 1 );
    }
    const int ystride = g->extx;
    for ( unsigned tid = 0; tid < g->ntx * g->nty; tid++ ) {
        for ( int iy = 0; iy < (int) g->exty; iy++ ) {
            for ( int ix = 0; ix < (int) ( g->extx - shift ); ix++ )
                cell_copy( g, gcell( g, tid, ix + iy * ystride ), gcell( g, tid, ix + shift + iy * ystride ) );
            for ( int ix = g->extx - shift; ix < (int) g->extx; ix++ ) {
                real * d = gcell( g, tid, ix + iy * ystride );
                for ( int k = 0; k < g->nc; k++ ) d[k] = 0;
            }
        }
    }
    grid_copy_to_gc_x( g );
}

/* grid.h:495-541 (kernel3_x) and 549-593 (kernel3_y); a, b, c are FP32 in the reference */
static void grid_kernel3( ogrid * g, int diry, real a, real b, real c ) {
    const int ystride = g->extx;
    const unsigned tv = g->tile_vol;
    real * A = (real *) malloc( (size_t) tv * g->nc * sizeof( real ) );
    real * B = (real *) malloc( (size_t) tv * g->nc * sizeof( real ) );
    for ( unsigned tid = 0; tid < g->ntx * g->nty; tid++ ) {
        real * buffer = gcell( g, tid, 0 );
        memcpy( A, buffer, (size_t) tv * g->nc * sizeof( real ) );
        memcpy( B, buffer, (size_t) tv * g->nc * sizeof( real ) );
        if ( !diry ) {
            for ( int iy = 0; iy < (int) g->exty; iy++ )
                for ( int ix = g->gxl; ix < (int) ( g->gxl + g->nxx ); ix++ )
                    for ( int k = 0; k < g->nc; k++ )
                        B[ ( iy * ystride + ix ) * g->nc + k ] =
                            A[ ( iy * ystride + ix - 1 ) * g->nc + k ] * a +
                            A[ ( iy * ystride + ix ) * g->nc + k ] * b +
                            A[ ( iy * ystride + ix + 1 ) * g->nc + k ] * c;
        } else {
            for ( int iy = g->gyl; iy < (int) ( g->nxy + g->gyl ); iy++ )
                for ( int ix = 0; ix < (int) g->extx; ix++ )
                    for ( int k = 0; k < g->nc; k++ )
                        B[ ( iy * ystride + ix ) * g->nc + k ] =
                            A[ ( ( iy - 1 ) * ystride + ix ) * g->nc + k ] * a +
                            A[ ( iy * ystride + ix ) * g->nc + k ] * b +
                            A[ ( ( iy + 1 ) * ystride + ix ) * g->nc + k ] * c;
        }
        memcpy( buffer, B, (size_t) tv * g->nc * sizeof( real ) );
    }
    free( A ); free( B );
    if ( !diry ) grid_copy_to_gc_x( g ); else grid_copy_to_gc_y( g );
}

/* ======================================================================== */
/* Digital filters (filter.h:9-86)                                          */
/* ======================================================================== */
static void filter_apply( ogrid * g, int type, int diry, unsigned order ) {
    if ( type == 0 ) return;
    if ( order == 0 ) order = 1;                 /* filter.h:35 */
    for ( unsigned i = 0; i < order; i++ )
        grid_kernel3( g, diry, (real) 0.25f, (real) 0.5f, (real) 0.25f );
    if ( type == 2 ) {                           /* filter.h:62-80 */
        float a = -1.0f;
        float b = ( 4.0 + 2.0 * order ) / order;
        float norm = 2 * a + b;
        grid_kernel3( g, diry, (real) ( a / norm ), (real) ( b / norm ), (real) ( a / norm ) );
    }
}

/* ======================================================================== */
/* Particles (particles.h:82-351, particles.cpp)                            */
/* ======================================================================== */
typedef struct {
    unsigned ntx, nty, nxx, nxy;
    int * np; int * offset;
    int * ix; real * x; real * u;
    uint32_t max_part;
    int perx, pery;
} oparts;

typedef struct { int * idx; int * nidx; int * npt; int * new_np; int ntiles; } osort;

static oparts * parts_new( unsigned ntx, unsigned nty, unsigned nxx, unsigned nxy, uint32_t max_part ) {
    oparts * p = (oparts *) calloc( 1, sizeof( oparts ) );
    p->ntx = ntx; p->nty = nty; p->nxx = nxx; p->nxy = nxy;
    p->np = (int *) calloc( ntx * nty, sizeof( int ) );
    p->offset = (int *) calloc( ntx * nty, sizeof( int ) );
    p->max_part = max_part;
    p->ix = (int *) malloc( (size_t) max_part * 2 * sizeof( int ) );
    p->x = (real *) malloc( (size_t) max_part * 2 * sizeof( real ) );
    p->u = (real *) malloc( (size_t) max_part * 3 * sizeof( real ) );
    p->perx = p->pery = 1;
    return p;
}
static void parts_free( oparts * p ) {
    if ( !p ) return;
    free( p->np ); free( p->offset ); free( p->ix ); free( p->x ); free( p->u ); free( p );
}
static void sort_init( osort * s, unsigned ntiles, uint32_t max_part ) {
    s->ntiles = ntiles;
    s->idx = (int *) malloc( (size_t) max_part * sizeof( int ) );
    s->nidx = (int *) calloc( ntiles, sizeof( int ) );
    s->npt = (int *) calloc( 9 * ntiles, sizeof( int ) );
    s->new_np = (int *) calloc( ntiles, sizeof( int ) );
}
static void sort_free( osort * s ) { free( s->idx ); free( s->nidx ); free( s->npt ); free( s->new_np ); }

static void pcopy( oparts * d, size_t l, const oparts * s, size_t k ) {
    d->ix[2*l] = s->ix[2*k]; d->ix[2*l+1] = s->ix[2*k+1];
    d->x[2*l] = s->x[2*k];   d->x[2*l+1] = s->x[2*k+1];
    d->u[3*l] = s->u[3*k];   d->u[3*l+1] = s->u[3*k+1]; d->u[3*l+2] = s->u[3*k+2];
}

/* particles.h:174-190: grow without copying, in 64k blocks */
static void parts_grow( oparts * p, uint32_t new_max ) {
    if ( new_max > p->max_part ) {
        free( p->ix ); free( p->x ); free( p->u );
        p->max_part = ( new_max + 65535u ) & ~65535u;
        p->ix = (int *) malloc( (size_t) p->max_part * 2 * sizeof( int ) );
        p->x = (real *) malloc( (size_t) p->max_part * 2 * sizeof( real ) );
        p->u = (real *) malloc( (size_t) p->max_part * 3 * sizeof( real ) );
    }
}
/* particles.h:192-206 */
static void parts_swap( oparts * a, oparts * b ) {
    int * ti; real * tr; uint32_t tm;
    ti = a->ix; a->ix = b->ix; b->ix = ti;
    tr = a->x; a->x = b->x; b->x = tr;
    tr = a->u; a->u = b->u; b->u = tr;
    tm = a->max_part; a->max_part = b->max_part; b->max_part = tm;
    ti = a->np; a->np = b->np; b->np = ti;
    ti = a->offset; a->offset = b->offset; b->offset = ti;
}
static uint32_t parts_np_total( const oparts * p ) {
    uint32_t t = 0;
    for ( unsigned i = 0; i < p->ntx * p->nty; i++ ) t += p->np[i];
    return t;
}

/* particles.cpp:212-303 */
static void bnd_check( oparts * part, osort * sort ) {
    const int ntx = part->ntx, nty = part->nty;
    const int limx = part->nxx, limy = part->nxy;
    for ( int tid = 0; tid < ntx * nty; tid++ ) {
        int tx = tid % ntx, ty = tid / ntx;
        const int np = part->np[tid], offset = part->offset[tid];
        const int * ix = part->ix + 2 * (size_t) offset;
        int * idx = sort->idx + offset;
        int npt[9] = { 0 };
        int nout = 0;
        for ( int i = 0; i < np; i++ ) {
            int xcross = ( ix[2*i] >= limx ) - ( ix[2*i] < 0 );
            int ycross = ( ix[2*i+1] >= limy ) - ( ix[2*i+1] < 0 );
            if ( xcross || ycross ) {
                npt[ ( ycross + 1 ) * 3 + ( xcross + 1 ) ] += 1;
                idx[nout++] = i;
            }
        }
        npt[4] = np - nout;
        for ( int i = 0; i < 9; i++ ) {
            int ttx = tx + ( i % 3 - 1 ), tty = ty + ( i / 3 - 1 );
            if ( part->perx ) { if ( ttx < 0 ) ttx += ntx; if ( ttx >= ntx ) ttx -= ntx; }
            if ( part->pery ) { if ( tty < 0 ) tty += nty; if ( tty >= nty ) tty -= nty; }
            if ( ttx >= 0 && ttx < ntx && tty >= 0 && tty < nty ) sort->new_np[ tty * ntx + ttx ] += npt[i];
        }
        for ( int i = 0; i < 9; i++ ) sort->npt[ 9 * tid + i ] = npt[i];
        sort->nidx[tid] = nout;
    }
}

/* particles.cpp:314-357 */
static uint32_t update_tile_info( oparts * tmp, const int * new_np, const int * extra ) {
    uint32_t total = 0;
    for ( unsigned i = 0; i < tmp->ntx * tmp->nty; i++ ) {
        tmp->offset[i] = total;
        tmp->np[i] = 0;
        total += new_np[i] + ( extra ? extra[i] : 0 );
    }
    return total;
}

static int target_offset( oparts * part, oparts * tmp, int tx, int ty, int i, int count, int atomic_add ) {
    const int ntx = part->ntx, nty = part->nty;
    int ttx = tx + i % 3 - 1, tty = ty + i / 3 - 1;
    int valid = 1;
    if ( part->perx ) { if ( ttx < 0 ) ttx += ntx; if ( ttx >= ntx ) ttx -= ntx; }
    else valid &= ( ttx >= 0 ) && ( ttx < ntx );
    if ( part->pery ) { if ( tty < 0 ) tty += nty; if ( tty >= nty ) tty -= nty; }
    else valid &= ( tty >= 0 ) && ( tty < nty );
    if ( !valid ) return -1;
    int t = tty * ntx + ttx;
    int off = tmp->offset[t] + tmp->np[t];
    (void) atomic_add;
    tmp->np[t] += count;
    return off;
}

/* particles.cpp:379-550 */
static void copy_out( oparts * part, oparts * tmp, osort * sort ) {
    const int ntx = part->ntx, nty = part->nty;
    const int limx = part->nxx, limy = part->nxy;
    for ( int tid = 0; tid < ntx * nty; tid++ ) {
        int tx = tid % ntx, ty = tid / ntx;
        const int old_offset = part->offset[tid];
        const int * npt = sort->npt + 9 * tid;
        int * idx = sort->idx + old_offset;
        const int nidx = sort->nidx[tid];
        const int new_offset = tmp->offset[tid];
        const int new_np = sort->new_np[tid];
        int dir_offset[9];
        const int n0 = npt[4];
        int nshift;
        if ( new_offset >= old_offset ) nshift = new_offset - old_offset;
        else { nshift = ( old_offset + n0 ) - ( new_offset + new_np ); if ( nshift < 0 ) nshift = 0; }
        if ( nshift > n0 ) nshift = n0;

        dir_offset[4] = new_offset + tmp->np[tid];
        tmp->np[tid] += nshift;
        for ( int i = 0; i < 9; i++ )
            if ( i != 4 ) dir_offset[i] = target_offset( part, tmp, tx, ty, i, npt[i], 1 );

        int c_ = n0;
        for ( int i = 0; i < nidx; i++ ) {
            int k = idx[i];
            size_t gk = (size_t) old_offset + k;
            int nixx = part->ix[2*gk], nixy = part->ix[2*gk+1];
            int xcross = ( nixx >= limx ) - ( nixx < 0 );
            int ycross = ( nixy >= limy ) - ( nixy < 0 );
            const int dir = ( ycross + 1 ) * 3 + ( xcross + 1 );
            if ( dir_offset[dir] >= 0 ) {
                int l = dir_offset[dir]; dir_offset[dir] += 1;
                pcopy( tmp, l, part, gk );
                tmp->ix[2*(size_t)l]   = nixx - xcross * limx;
                tmp->ix[2*(size_t)l+1] = nixy - ycross * limy;
            }
            if ( k < n0 ) {
                int c, invalid;
                do {
                    c = c_; c_ += 1;
                    size_t gc = (size_t) old_offset + c;
                    invalid = ( part->ix[2*gc] < 0 ) || ( part->ix[2*gc] >= limx ) ||
                              ( part->ix[2*gc+1] < 0 ) || ( part->ix[2*gc+1] >= limy );
                } while ( invalid );
                pcopy( part, gk, part, (size_t) old_offset + c );
            }
        }
        const int new_idx = dir_offset[4];
        if ( new_offset >= old_offset ) {
            for ( int i = 0; i < nshift; i++ ) pcopy( tmp, new_idx + i, part, (size_t) old_offset + i );
        } else {
            const int old_idx = n0 - nshift;
            for ( int i = 0; i < nshift; i++ ) pcopy( tmp, new_idx + i, part, (size_t) old_offset + old_idx + i );
        }
        part->np[tid] = n0 - nshift;
    }
}

/* particles.cpp:559-614 */
static void copy_in( oparts * part, oparts * tmp ) {
    for ( unsigned tid = 0; tid < part->ntx * part->nty; tid++ ) {
        const int old_offset = part->offset[tid], old_np = part->np[tid];
        const int new_offset = tmp->offset[tid], tmp_np = tmp->np[tid];
        if ( new_offset >= old_offset ) {
            for ( int i = 0; i < tmp_np; i++ )
                pcopy( part, (size_t) new_offset + old_np + i, tmp, (size_t) new_offset + i );
        } else {
            int np0 = old_offset - new_offset;
            if ( np0 > tmp_np ) np0 = tmp_np;
            for ( int i = 0; i < np0; i++ ) pcopy( part, (size_t) new_offset + i, tmp, (size_t) new_offset + i );
            for ( int i = np0; i < tmp_np; i++ )
                pcopy( part, (size_t) new_offset + old_np + i, tmp, (size_t) new_offset + i );
        }
        part->np[tid] = old_np + tmp_np;
        part->offset[tid] = new_offset;
    }
}

/* particles.cpp:628-763 (buffer-grow path) */
static void copy_sorted( oparts * part, oparts * tmp, osort * sort ) {
    const int ntx = part->ntx, nty = part->nty;
    const int limx = part->nxx, limy = part->nxy;
    for ( int ty = 0; ty < nty; ty++ ) for ( int tx = 0; tx < ntx; tx++ ) {
        int tid = ty * ntx + tx;
        const int old_offset = part->offset[tid];
        const int * npt = sort->npt + 9 * tid;
        int * idx = sort->idx + old_offset;
        const int nidx = sort->nidx[tid];
        int dir_offset[9];
        for ( int i = 0; i < 9; i++ ) dir_offset[i] = target_offset( part, tmp, tx, ty, i, npt[i], 0 );
        const int n0 = npt[4];
        int c_ = n0;
        for ( int i = 0; i < nidx; i++ ) {
            int k = idx[i];
            size_t gk = (size_t) old_offset + k;
            int nixx = part->ix[2*gk], nixy = part->ix[2*gk+1];
            int xcross = ( nixx >= limx ) - ( nixx < 0 );
            int ycross = ( nixy >= limy ) - ( nixy < 0 );
            const int dir = ( ycross + 1 ) * 3 + ( xcross + 1 );
            if ( dir_offset[dir] >= 0 ) {
                int l = dir_offset[dir]; dir_offset[dir] += 1;
                pcopy( tmp, l, part, gk );
                tmp->ix[2*(size_t)l]   = nixx - xcross * limx;
                tmp->ix[2*(size_t)l+1] = nixy - ycross * limy;
            }
            if ( k < n0 ) {
                int c, invalid;
                do {
                    c = c_; c_ += 1;
                    size_t gc = (size_t) old_offset + c;
                    invalid = ( part->ix[2*gc] < 0 ) || ( part->ix[2*gc] >= limx ) ||
                              ( part->ix[2*gc+1] < 0 ) || ( part->ix[2*gc+1] >= limy );
                } while ( invalid );
                pcopy( part, gk, part, (size_t) old_offset + c );
            }
        }
        const int start = dir_offset[4];
        for ( int i = 0; i < n0; i++ ) pcopy( tmp, (size_t) start + i, part, (size_t) old_offset + i );
    }
}

/* particles.cpp:855-904 */
static void tile_sort( oparts * part, oparts * tmp, osort * sort, const int * extra ) {
    memset( sort->new_np, 0, sort->ntiles * sizeof( int ) );
    bnd_check( part, sort );
    if ( extra ) {
        uint32_t total_np = update_tile_info( tmp, sort->new_np, extra );
        if ( total_np > part->max_part ) {
            parts_grow( tmp, total_np );
            copy_sorted( part, tmp, sort );
            parts_swap( part, tmp );
            parts_grow( tmp, part->max_part );
        } else {
            copy_out( part, tmp, sort );
            copy_in( part, tmp );
        }
    } else {
        update_tile_info( tmp, sort->new_np, NULL );
        copy_out( part, tmp, sort );
        copy_in( part, tmp );
    }
}

/* ======================================================================== */
/* Random numbers (random.h:23-155)                                         */
/* ======================================================================== */
typedef struct { unsigned x, y; } ustate;

static void rand_init( int global_id, unsigned sx, unsigned sy, ustate * st, double * norm ) {
    *norm = DBL_MAX;
    st->x = sx + global_id;
    st->y = sy + ( ( global_id ) ^ ( 0xFFFFFFFF ) );
}
static unsigned rand_uint32( ustate * st ) {
    st->x = 36969 * ( st->x & 65535 ) + ( st->x >> 16 );
    st->y = 18000 * ( st->y & 65535 ) + ( st->y >> 16 );
    return ( st->x << 16 ) + st->y;
}
static double rand_real3( ustate * st ) { return ( rand_uint32( st ) + 1.0 ) * 0x1.fffffffep-33; }
static double rand_norm( ustate * st, double * norm ) {
    double res;
    if ( *norm == DBL_MAX ) {
        double v1, v2, rsq, fac;
        do {
            v1 = rand_real3( st ) * 2.0 - 1.0;
            v2 = rand_real3( st ) * 2.0 - 1.0;
            rsq = v1 * v1 + v2 * v2;
        } while ( rsq == 0.0 || rsq >= 1.0 );
        fac = sqrt( -2.0 * log( rsq ) / rsq );
        *norm = v1 * fac;
        res = v2 * fac;
    } else {
        res = *norm;
        *norm = DBL_MAX;
    }
    return res;
}

/* ======================================================================== */
/* Species                                                                  */
/* ======================================================================== */
typedef struct {
    int id;
    unsigned ppcx, ppcy;
    real q;
    real2 dx, box;
    real dt;
    int iter;
    oparts * part; oparts * tmp; osort sort;
    int dens_type; float dens_p[5];
    int * np_inj;
    int bc[4];
    omw mw;
    int udist_type; float uth[3], ufl[3]; int npmin;
    double d_energy; uint64_t d_nmove;
    float m_q; int push_type;
} ospecies;

/* ------------------------------------------------------------------------ */
/* Injection (density.cpp)                                                  */
/* ------------------------------------------------------------------------ */

/* tile range clip shared by all profiles (density.cpp:134-160) */
static int tile_range( const oparts * p, unsigned tx, unsigned ty, const unsigned * range,
                       int * ri0, int * ri1, int * rj0, int * rj1 ) {
    const int nxx = p->nxx, nxy = p->nxy;
    *ri0 = range[0] - tx * p->nxx; *ri1 = range[1] - tx * p->nxx;
    *rj0 = range[2] - ty * p->nxy; *rj1 = range[3] - ty * p->nxy;
    if ( ( *ri0 < nxx ) && ( *ri1 >= 0 ) && ( *rj0 < nxy ) && ( *rj1 >= 0 ) ) {
        if ( *ri0 < 0 ) *ri0 = 0;
        if ( *rj0 < 0 ) *rj0 = 0;
        if ( *ri1 >= nxx ) *ri1 = nxx - 1;
        if ( *rj1 >= nxy ) *rj1 = nxy - 1;
        return 1;
    }
    return 0;
}

/*
 * Does in-cell position (pos) of cell (cell) in tile (tx,ty) receive a
 * particle?  Uniform: density.cpp:103-186; Step: 330-412; Slab: 574-672;
 * Sphere: 855-933.  step/begin/end are already normalised to cells.
 */
typedef struct { int type; float a, b; float cx, cy, r2; float dxx, dxy; int diry; } inj_rule;

static int inj_test( const inj_rule * r, int shiftx, int shifty, int cx, int cy, float posx, float posy ) {
    float t;
    switch ( r->type ) {
    case 1: return 1;
    case 2:
        t = r->diry ? (float) ( ( shifty + cy ) + ( posy + 0.5 ) ) : (float) ( ( shiftx + cx ) + ( posx + 0.5 ) );
        return t > r->a;
    case 3:
        t = r->diry ? (float) ( ( shifty + cy ) + ( posy + 0.5 ) ) : (float) ( ( shiftx + cx ) + ( posx + 0.5 ) );
        return ( t >= r->a ) && ( t < r->b );
    case 4: {
        float gx = (float) ( ( ( shiftx + cx ) + ( posx + 0.5 ) ) * r->dxx );
        float gy = (float) ( ( ( shifty + cy ) + ( posy + 0.5 ) ) * r->dxy );
        return ( gx - r->cx ) * ( gx - r->cx ) + ( gy - r->cy ) * ( gy - r->cy ) < r->r2;
    }
    }
    return 0;
}

static void make_rule( const ospecies * sp, double motion, inj_rule * r ) {
    float refx = (float) motion;     /* float2 ref = make_float2( moving_window.motion(), 0 ) */
    const float * p = sp->dens_p;
    r->type = sp->dens_type;
    r->diry = p[4] != 0;
    r->dxx = (float) sp->dx.x; r->dxy = (float) sp->dx.y;
    switch ( sp->dens_type ) {
    case 2: r->a = ( p[1] - refx ) / (float) sp->dx.x; break;                         /* density.cpp:418 */
    case 3: r->a = ( p[1] - refx ) / (float) sp->dx.x;                               /* density.cpp:677-678 */
            r->b = ( p[2] - refx ) / (float) sp->dx.x; break;
    case 4: r->cx = p[1] - refx; r->cy = p[2] - 0.0f; r->r2 = p[3] * p[3]; break;     /* density.cpp:937-941 */
    default: break;
    }
}

/* Step/Slab with dir = y loop tx < ntiles.y in the reference (density.cpp:438, 470, 692) */
static unsigned inj_tx_limit( const ospecies * sp ) {
    const oparts * p = sp->part;
    if ( ( sp->dens_type == 2 || sp->dens_type == 3 ) && sp->dens_p[4] != 0 )
        return p->nty < p->ntx ? p->nty : p->ntx;
    return p->ntx;
}

/* np_inject (density.cpp:217-299 and the per-profile counting kernels) */
static void species_np_inject( ospecies * sp, const unsigned * range, int * np ) {
    oparts * p = sp->part;
    if ( sp->dens_type == 0 ) {                 /* density.h:39-42: zero_np() */
        memset( p->np, 0, p->ntx * p->nty * sizeof( int ) );
        return;
    }
    inj_rule r; make_rule( sp, mw_motion( &sp->mw ), &r );
    double dpcx = 1.0 / sp->ppcx, dpcy = 1.0 / sp->ppcy;
    unsigned txl = inj_tx_limit( sp );
    for ( unsigned ty = 0; ty < p->nty; ty++ ) for ( unsigned tx = 0; tx < txl; tx++ ) {
        int tid = ty * p->ntx + tx;
        int ri0, ri1, rj0, rj1, n = 0;
        if ( tile_range( p, tx, ty, range, &ri0, &ri1, &rj0, &rj1 ) ) {
            int row = ri1 - ri0 + 1, vol = ( rj1 - rj0 + 1 ) * row;
            if ( sp->dens_type == 1 ) n = vol * sp->ppcx * sp->ppcy;
            else {
                int shiftx = tx * p->nxx, shifty = ty * p->nxy;
                for ( int idx = 0; idx < vol; idx++ )
                    for ( unsigned i1 = 0; i1 < sp->ppcy; i1++ )
                        for ( unsigned i0 = 0; i0 < sp->ppcx; i0++ ) {
                            float posx = dpcx * ( i0 + 0.5 ) - 0.5, posy = dpcy * ( i1 + 0.5 ) - 0.5;
                            n += inj_test( &r, shiftx, shifty, idx % row + ri0, idx / row + rj0, posx, posy );
                        }
            }
        }
        np[tid] = n;
    }
}

/* inject (density.cpp:188-216 mk2 ordering for Uniform; 330-412 Step etc.) */
static void species_inject( ospecies * sp, const unsigned * range ) {
    oparts * p = sp->part;
    if ( sp->dens_type == 0 ) return;
    inj_rule r; make_rule( sp, mw_motion( &sp->mw ), &r );
    double dpcx = 1.0 / sp->ppcx, dpcy = 1.0 / sp->ppcy;
    unsigned txl = inj_tx_limit( sp );
    for ( unsigned ty = 0; ty < p->nty; ty++ ) for ( unsigned tx = 0; tx < txl; tx++ ) {
        int tid = ty * p->ntx + tx;
        int ri0, ri1, rj0, rj1;
        if ( !tile_range( p, tx, ty, range, &ri0, &ri1, &rj0, &rj1 ) ) continue;
        int row = ri1 - ri0 + 1, vol = ( rj1 - rj0 + 1 ) * row;
        int np = p->np[tid];
        size_t base = p->offset[tid];
        int shiftx = tx * p->nxx, shifty = ty * p->nxy;
        for ( unsigned i1 = 0; i1 < sp->ppcy; i1++ )
            for ( unsigned i0 = 0; i0 < sp->ppcx; i0++ ) {
                float posx = dpcx * ( i0 + 0.5 ) - 0.5, posy = dpcy * ( i1 + 0.5 ) - 0.5;
                int ppc_idx = i1 * sp->ppcx + i0;
                for ( int idx = 0; idx < vol; idx++ ) {
                    int cx = idx % row + ri0, cy = idx / row + rj0;
                    int k;
                    if ( sp->dens_type == 1 ) k = np + vol * ppc_idx + idx;
                    else {
                        if ( !inj_test( &r, shiftx, shifty, cx, cy, posx, posy ) ) continue;
                        k = np++;
                    }
                    size_t g = base + k;
                    p->ix[2*g] = cx; p->ix[2*g+1] = cy;
                    p->x[2*g] = posx; p->x[2*g+1] = posy;
                    p->u[3*g] = 0; p->u[3*g+1] = 0; p->u[3*g+2] = 0;
                }
            }
        if ( sp->dens_type == 1 ) p->np[tid] = np + vol * sp->ppcx * sp->ppcy;
        else p->np[tid] = np;
    }
}

/* udist.cpp:10-136 */
static void species_udist( ospecies * sp ) {
    oparts * p = sp->part;
    const unsigned nt = p->ntx * p->nty;
    const unsigned sx = 12345 + sp->id, sy = 67890;
    for ( unsigned tid = 0; tid < nt; tid++ ) {
        size_t off = p->offset[tid];
        int np = p->np[tid];
        real * u = p->u + 3 * off;
        const int * ix = p->ix + 2 * off;
        if ( sp->udist_type == 0 || sp->udist_type == 1 ) {
            for ( int i = 0; i < np; i++ ) {
                u[3*i]   = sp->udist_type ? sp->ufl[0] : 0;
                u[3*i+1] = sp->udist_type ? sp->ufl[1] : 0;
                u[3*i+2] = sp->udist_type ? sp->ufl[2] : 0;
            }
        } else if ( sp->udist_type == 2 ) {
            ustate st; double norm;
            rand_init( tid, sx, sy, &st, &norm );
            for ( int i = 0; i < np; i++ ) {
                /* make_float3( f(), f(), f() ): g++ evaluates the arguments right to left */
                double c = sp->ufl[2] + sp->uth[2] * rand_norm( &st, &norm );
                double b = sp->ufl[1] + sp->uth[1] * rand_norm( &st, &norm );
                double a = sp->ufl[0] + sp->uth[0] * rand_norm( &st, &norm );
                u[3*i] = (real) (float) a; u[3*i+1] = (real) (float) b; u[3*i+2] = (real) (float) c;
            }
        } else {
            const unsigned bsize = p->nxx * p->nxy;
            const int ystride = p->nxx;
            real * fluid = (real *) calloc( 3 * bsize, sizeof( real ) );
            int * npcell = (int *) calloc( bsize, sizeof( int ) );
            ustate st; double norm;
            rand_init( tid, sx, sy, &st, &norm );
            for ( int i = 0; i < np; i++ ) {
                /* make_float3( f(), f(), f() ): g++ evaluates the arguments right to left */
                float uz = sp->uth[2] * rand_norm( &st, &norm );
                float uy = sp->uth[1] * rand_norm( &st, &norm );
                float ux = sp->uth[0] * rand_norm( &st, &norm );
                u[3*i] = ux; u[3*i+1] = uy; u[3*i+2] = uz;
                int idx = ix[2*i] + ystride * ix[2*i+1];
                npcell[idx] += 1;
                fluid[3*idx] += (real) ux; fluid[3*idx+1] += (real) uy; fluid[3*idx+2] += (real) uz;
            }
            for ( unsigned idx = 0; idx < bsize; idx++ ) {
                if ( npcell[idx] > sp->npmin ) {
                    fluid[3*idx] /= npcell[idx]; fluid[3*idx+1] /= npcell[idx]; fluid[3*idx+2] /= npcell[idx];
                } else {
                    fluid[3*idx] = fluid[3*idx+1] = fluid[3*idx+2] = 0;
                }
            }
            for ( int i = 0; i < np; i++ ) {
                int idx = ix[2*i] + ystride * ix[2*i+1];
                /* u[i] += ufl - fluid[idx]  (float3 ops: (ufl - fluid) then += ) */
                u[3*i]   += (real) sp->ufl[0] - fluid[3*idx];
                u[3*i+1] += (real) sp->ufl[1] - fluid[3*idx+1];
                u[3*i+2] += (real) sp->ufl[2] - fluid[3*idx+2];
            }
            free( fluid ); free( npcell );
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Push (species.cpp:22-254, 1626-1682, 2302-2335)                          */
/* ------------------------------------------------------------------------ */
static real rgamma( real ux, real uy, real uz ) {
    return (real) 1 / r_sqrt( r_fma( uz, uz, r_fma( uy, uy, r_fma( ux, ux, (real) 1 ) ) ) );
}

/* species.cpp:43-92 */
static void interpolate_fld( const real3 * E, const real3 * B, int ystride,
                             int i, int j, real xx, real xy, real3 * e, real3 * b ) {
    const real s0x = (real) 0.5 - xx, s1x = (real) 0.5 + xx;
    const real s0y = (real) 0.5 - xy, s1y = (real) 0.5 + xy;
    const int hx = xx < 0, hy = xy < 0;
    const int ih = i - hx, jh = j - hy;
    const real s0xh = ( 1 - hx ) - xx, s1xh = ( hx ) + xx;
    const real s0yh = ( 1 - hy ) - xy, s1yh = ( hy ) + xy;

    e->x = ( E[ih +     j*ystride].x * s0xh + E[ih+1 +     j*ystride].x * s1xh ) * s0y +
           ( E[ih + (j+1)*ystride].x * s0xh + E[ih+1 + (j+1)*ystride].x * s1xh ) * s1y;
    e->y = ( E[i  +    jh*ystride].y * s0x  + E[i+1  +    jh*ystride].y * s1x  ) * s0yh +
           ( E[i  + (jh+1)*ystride].y * s0x + E[i+1  + (jh+1)*ystride].y * s1x  ) * s1yh;
    e->z = ( E[i  +     j*ystride].z * s0x  + E[i+1  +     j*ystride].z * s1x  ) * s0y +
           ( E[i  + (j+1)*ystride].z * s0x  + E[i+1  + (j+1)*ystride].z * s1x  ) * s1y;

    b->x = ( B[i  +    jh*ystride].x * s0x  + B[i+1  +    jh*ystride].x * s1x  ) * s0yh +
           ( B[i  + (jh+1)*ystride].x * s0x + B[i+1  + (jh+1)*ystride].x * s1x  ) * s1yh;
    b->y = ( B[ih +     j*ystride].y * s0xh + B[ih+1 +     j*ystride].y * s1xh ) * s0y +
           ( B[ih + (j+1)*ystride].y * s0xh + B[ih+1 + (j+1)*ystride].y * s1xh ) * s1y;
    b->z = ( B[ih +    jh*ystride].z * s0xh + B[ih+1 +    jh*ystride].z * s1xh ) * s0yh +
           ( B[ih + (jh+1)*ystride].z * s0xh + B[ih+1 + (jh+1)*ystride].z * s1xh ) * s1yh;
}

/* species.cpp:117-178 */
static real3 dudt_boris( real alpha, real3 e, real3 b, real3 u, double * energy ) {
    e.x *= alpha; e.y *= alpha; e.z *= alpha;
    real3 ut = { u.x + e.x, u.y + e.y, u.z + e.z };
    {
        const real utsq = r_fma( ut.z, ut.z, r_fma( ut.y, ut.y, ut.x * ut.x ) );
        const real gamma = r_sqrt( (real) 1 + utsq );
        *energy += utsq / ( gamma + (real) 1 );
        const real alpha_gamma = alpha / gamma;
        b.x *= alpha_gamma; b.y *= alpha_gamma; b.z *= alpha_gamma;
    }
    u.x = r_fma( b.z, ut.y, ut.x );
    u.y = r_fma( b.x, ut.z, ut.y );
    u.z = r_fma( b.y, ut.x, ut.z );
    u.x = r_fma( -b.y, ut.z, u.x );
    u.y = r_fma( -b.z, ut.x, u.y );
    u.z = r_fma( -b.x, ut.y, u.z );
    {
        const real otsq = (real) 2 / r_fma( b.z, b.z, r_fma( b.y, b.y, r_fma( b.x, b.x, (real) 1 ) ) );
        b.x *= otsq; b.y *= otsq; b.z *= otsq;
    }
    ut.x = r_fma( b.z, u.y, ut.x );
    ut.y = r_fma( b.x, u.z, ut.y );
    ut.z = r_fma( b.y, u.x, ut.z );
    ut.x = r_fma( -b.y, u.z, ut.x );
    ut.y = r_fma( -b.z, u.x, ut.y );
    ut.z = r_fma( -b.x, u.y, ut.z );
    ut.x += e.x; ut.y += e.y; ut.z += e.z;
    return ut;
}

/* species.cpp:193-254 (exact Euler-Rodrigues rotation) */
static real3 dudt_boris_euler( real alpha, real3 e, real3 b, real3 u, double * energy ) {
    e.x *= alpha; e.y *= alpha; e.z *= alpha;
    real3 ut = { u.x + e.x, u.y + e.y, u.z + e.z };
    {
        const real utsq = r_fma( ut.z, ut.z, r_fma( ut.y, ut.y, ut.x * ut.x ) );
        const real gamma = r_sqrt( (real) 1 + utsq );
        *energy += utsq / ( gamma + (real) 1 );
        const real alpha2_gamma = ( alpha * 2 ) / gamma;
        b.x *= alpha2_gamma; b.y *= alpha2_gamma; b.z *= alpha2_gamma;
    }
    {
        const real bnorm = r_sqrt( r_fma( b.x, b.x, r_fma( b.y, b.y, b.z * b.z ) ) );
        const real s = -( ( bnorm > 0 ) ? r_sin( bnorm / 2 ) / bnorm : 1 );
        const real ra = r_cos( bnorm / 2 );
        const real rb = b.x * s, rc = b.y * s, rd = b.z * s;
        const real r11 =     r_fma( ra, ra, rb * rb ) - r_fma( rc, rc, rd * rd );
        const real r12 = 2 * r_fma( rb, rc, ra * rd );
        const real r13 = 2 * r_fma( rb, rd, -ra * rc );
        const real r21 = 2 * r_fma( rb, rc, -ra * rd );
        const real r22 =     r_fma( ra, ra, rc * rc ) - r_fma( rb, rb, rd * rd );
        const real r23 = 2 * r_fma( rc, rd, ra * rb );
        const real r31 = 2 * r_fma( rb, rd, ra * rc );
        const real r32 = 2 * r_fma( rc, rd, -ra * rb );
        const real r33 =     r_fma( ra, ra, rd * rd ) - r_fma( rb, rb, -rc * rc );
        u.x = r_fma( r11, ut.x, r_fma( r21, ut.y, r31 * ut.z ) );
        u.y = r_fma( r12, ut.x, r_fma( r22, ut.y, r32 * ut.z ) );
        u.z = r_fma( r13, ut.x, r_fma( r23, ut.y, r33 * ut.z ) );
    }
    u.x += e.x; u.y += e.y; u.z += e.z;
    return u;
}

/* species.cpp:1626-1682 (tiles in order, energy summed per tile) and 2302-2335 */
static void species_push( ospecies * sp, const ogrid * E, const ogrid * B ) {
    oparts * p = sp->part;
    const real alpha = (real) ( 0.5 * sp->dt / sp->m_q );
    const int ystride = E->extx;
    double total = 0;
    for ( unsigned tid = 0; tid < p->ntx * p->nty; tid++ ) {
        const real3 * Et = (const real3 *) gcell( E, tid, E->offset );
        const real3 * Bt = (const real3 *) gcell( B, tid, B->offset );
        size_t off = p->offset[tid];
        const int np = p->np[tid];
        double energy = 0;
        for ( int i = 0; i < np; i++ ) {
            size_t g = off + i;
            real3 e, b;
            interpolate_fld( Et, Bt, ystride, p->ix[2*g], p->ix[2*g+1], p->x[2*g], p->x[2*g+1], &e, &b );
            real3 pu = { p->u[3*g], p->u[3*g+1], p->u[3*g+2] };
            real3 nu = sp->push_type ? dudt_boris_euler( alpha, e, b, pu, &energy )
                                     : dudt_boris( alpha, e, b, pu, &energy );
            p->u[3*g] = nu.x; p->u[3*g+1] = nu.y; p->u[3*g+2] = nu.z;
        }
        total += energy;
    }
    sp->d_energy = 0 + total;
}

/* ------------------------------------------------------------------------ */
/* Move + deposit (species.cpp:267-430, 1400-1597, 2138-2198)               */
/* ------------------------------------------------------------------------ */

/* species.cpp:267-310 */
static void dep_current_seg( int ixx, int ixy, real x0x, real x0y, real x1x, real x1y,
                             real qnxx, real qnxy, real qvz, real * J, int stride ) {
    const real S0x0 = (real) 0.5 - x0x, S0x1 = (real) 0.5 + x0x;
    const real S1x0 = (real) 0.5 - x1x, S1x1 = (real) 0.5 + x1x;
    const real S0y0 = (real) 0.5 - x0y, S0y1 = (real) 0.5 + x0y;
    const real S1y0 = (real) 0.5 - x1y, S1y1 = (real) 0.5 + x1y;
    const real wl1 = qnxx * ( x1x - x0x );
    const real wl2 = qnxy * ( x1y - x0y );
    const real wp10 = (real) 0.5 * ( S0y0 + S1y0 ), wp11 = (real) 0.5 * ( S0y1 + S1y1 );
    const real wp20 = (real) 0.5 * ( S0x0 + S1x0 ), wp21 = (real) 0.5 * ( S0x1 + S1x1 );
    real * Js = J + 3 * ( ixx + stride * ixy );
    const int stride3 = 3 * stride;
    Js[0 + 0 + 0] += wl1 * wp10;
    Js[0 + 0 + 1] += wl2 * wp20;
    Js[0 + 0 + 2] += qvz * ( S0x0 * S0y0 + S1x0 * S1y0 + ( S0x0 * S1y0 - S1x0 * S0y0 ) / (real) 2 );
    Js[0 + 3 + 1] += wl2 * wp21;
    Js[0 + 3 + 2] += qvz * ( S0x1 * S0y0 + S1x1 * S1y0 + ( S0x1 * S1y0 - S1x1 * S0y0 ) / (real) 2 );
    Js[stride3 + 0 + 0] += wl1 * wp11;
    Js[stride3 + 0 + 2] += qvz * ( S0x0 * S0y1 + S1x0 * S1y1 + ( S0x0 * S1y1 - S1x0 * S0y1 ) / (real) 2 );
    Js[stride3 + 3 + 2] += qvz * ( S0x1 * S0y1 + S1x1 * S1y1 + ( S0x1 * S1y1 - S1x1 * S0y1 ) / (real) 2 );
}

typedef struct { int ix, iy; real x0x, x0y, x1x, x1y, qvz; } vseg;

/* species.cpp:336-430 */
static void split2d( int ix, int iy, real x0x, real x0y, real x1x, real x1y,
                     real dx, real dy, real qvz, int * dix, int * diy, vseg * v, int * crossx, int * crossy ) {
    *dix = ( ( x1x >= (real) 0.5 ) - ( x1x < (real) -0.5 ) );
    *diy = ( ( x1y >= (real) 0.5 ) - ( x1y < (real) -0.5 ) );
    *crossx = *dix != 0; *crossy = *diy != 0;
    v[0].ix = ix; v[0].iy = iy; v[0].x0x = x0x; v[0].x0y = x0y;
    v[0].x1x = x1x; v[0].x1y = x1y; v[0].qvz = qvz;
    memset( &v[1], 0, 2 * sizeof( vseg ) );

    if ( *crossy && !*crossx ) {
        real yint = (real) 0.5 * *diy;
        real eps = ( yint - x0y ) / dy;
        real xint = x0x + dx * eps;
        v[0].x1x = xint; v[0].x1y = yint; v[0].qvz = qvz * eps;
        v[1].ix = ix; v[1].iy = iy + *diy;
        v[1].x0x = xint; v[1].x0y = -yint;
        v[1].x1x = x1x; v[1].x1y = x1y - *diy;
        v[1].qvz = qvz * ( 1 - eps );
    }
    if ( *crossx ) {
        real xint = (real) 0.5 * *dix;
        real eps = ( xint - x0x ) / dx;
        real yint = x0y + dy * eps;
        v[0].x1x = xint; v[0].x1y = yint; v[0].qvz = qvz * eps;
        v[1].ix = ix + *dix; v[1].iy = iy;
        v[1].x0x = -xint; v[1].x0y = yint;
        v[1].x1x = x1x - *dix; v[1].x1y = x1y;
        v[1].qvz = qvz * ( 1 - eps );
        if ( *crossy ) {
            real yint2 = (real) 0.5 * *diy;
            if ( yint >= (real) -0.5 && yint < (real) 0.5 ) {
                eps = ( yint2 - yint ) / ( x1y - yint );
                real xint2 = -xint + ( x1x - xint ) * eps;
                v[2].ix = v[1].ix; v[2].iy = v[1].iy + *diy;
                v[2].x0x = xint2; v[2].x0y = -yint2;
                v[2].x1x = v[1].x1x; v[2].x1y = v[1].x1y - *diy;
                v[2].qvz = v[1].qvz * ( 1 - eps );
                v[1].x1x = xint2; v[1].x1y = yint2;
                v[1].qvz *= eps;
            } else {
                eps = ( yint2 - x0y ) / ( yint - x0y );
                real xint2 = x0x + ( xint - x0x ) * eps;
                v[2].ix = v[0].ix; v[2].iy = v[0].iy + *diy;
                v[2].x0x = xint2; v[2].x0y = -yint2;
                v[2].x1x = v[0].x1x; v[2].x1y = v[0].x1y - *diy;
                v[2].qvz = v[0].qvz * ( 1 - eps );
                v[0].x1x = xint2; v[0].x1y = yint2;
                v[0].qvz *= eps;
                v[1].iy += *diy;
                v[1].x0y -= *diy;
                v[1].x1y -= *diy;
            }
        }
    }
}

/*
 * move_deposit_kernel / move_deposit_shift_kernel / move_kernel
 * (species.cpp:1400-1493, 1508-1597, 2209-2264)
 * deposit = 0 -> free streaming, no current
 */
static void species_move( ospecies * sp, ogrid * J, int shiftx, int shifty, int deposit ) {
    oparts * p = sp->part;
    const real dt_dxx = sp->dt / sp->dx.x, dt_dxy = sp->dt / sp->dx.y;
    const real qnxx = sp->q * sp->dx.x / sp->dt, qnxy = sp->q * sp->dx.y / sp->dt;
    const int ystride = J->extx;
    const unsigned tv = J->tile_vol;
    real * local = (real *) malloc( (size_t) tv * 3 * sizeof( real ) );
    for ( unsigned tid = 0; tid < p->ntx * p->nty; tid++ ) {
        memset( local, 0, (size_t) tv * 3 * sizeof( real ) );
        real * Jt = local + 3 * J->offset;
        size_t off = p->offset[tid];
        const int np = p->np[tid];
        for ( int i = 0; i < np; i++ ) {
            size_t g = off + i;
            real ux = p->u[3*g], uy = p->u[3*g+1], uz = p->u[3*g+2];
            real x0x = p->x[2*g], x0y = p->x[2*g+1];
            int ix0 = p->ix[2*g], iy0 = p->ix[2*g+1];
            const real rg = rgamma( ux, uy, uz );
            const real dx = dt_dxx * rg * ux, dy = dt_dxy * rg * uy;
            real x1x = x0x + dx, x1y = x0y + dy;
            int dix, diy;
            if ( deposit ) {
                const real qvz = sp->q * uz * rg * (real) 0.5;
                vseg v[3]; int cx, cy;
                split2d( ix0, iy0, x0x, x0y, x1x, x1y, dx, dy, qvz, &dix, &diy, v, &cx, &cy );
                dep_current_seg( v[0].ix, v[0].iy, v[0].x0x, v[0].x0y, v[0].x1x, v[0].x1y, qnxx, qnxy, v[0].qvz, Jt, ystride );
                if ( cx || cy )
                    dep_current_seg( v[1].ix, v[1].iy, v[1].x0x, v[1].x0y, v[1].x1x, v[1].x1y, qnxx, qnxy, v[1].qvz, Jt, ystride );
                if ( cx && cy )
                    dep_current_seg( v[2].ix, v[2].iy, v[2].x0x, v[2].x0y, v[2].x1x, v[2].x1y, qnxx, qnxy, v[2].qvz, Jt, ystride );
            } else {
                dix = ( ( x1x >= (real) 0.5 ) - ( x1x < (real) -0.5 ) );
                diy = ( ( x1y >= (real) 0.5 ) - ( x1y < (real) -0.5 ) );
            }
            x1x -= dix; x1y -= diy;
            p->x[2*g] = x1x; p->x[2*g+1] = x1y;
            p->ix[2*g] = ix0 + dix + shiftx; p->ix[2*g+1] = iy0 + diy + shifty;
        }
        if ( deposit ) {
            real * gJ = gcell( J, tid, 0 );
            for ( unsigned i = 0; i < J->extx * J->exty * 3; i++ ) gJ[i] += local[i];
        }
    }
    free( local );
    for ( unsigned tid = 0; tid < p->ntx * p->nty; tid++ ) sp->d_nmove += p->np[tid];
}

/* species.cpp:1854-1989 (reflecting walls; open/periodic are handled by the sort) */
static void species_process_bc( ospecies * sp ) {
    oparts * p = sp->part;
    const int bcr = 2;
    if ( sp->bc[0] > 1 || sp->bc[1] > 1 ) {
        for ( unsigned ty = 0; ty < p->nty; ty++ ) {
            unsigned txs[2] = { 0u, p->ntx - 1 };
            for ( int q = 0; q < 2; q++ ) {
                unsigned tx = txs[q], tid = ty * p->ntx + tx;
                size_t off = p->offset[tid]; int np = p->np[tid];
                int lower = ( tx == 0 );
                int type = lower ? sp->bc[0] : sp->bc[1];
                if ( type != bcr ) continue;
                for ( int i = 0; i < np; i++ ) {
                    size_t g = off + i;
                    if ( lower ? ( p->ix[2*g] < 0 ) : ( p->ix[2*g] >= (int) p->nxx ) ) {
                        p->ix[2*g] += lower ? 1 : -1;
                        p->x[2*g] = -p->x[2*g];
                        p->u[3*g] = -p->u[3*g];
                    }
                }
            }
        }
    }
    if ( sp->bc[2] > 1 || sp->bc[3] > 1 ) {
        unsigned tys[2] = { 0u, p->nty - 1 };
        for ( int q = 0; q < 2; q++ ) {
            unsigned ty = tys[q];
            for ( unsigned tx = 0; tx < p->ntx; tx++ ) {
                unsigned tid = ty * p->ntx + tx;
                size_t off = p->offset[tid]; int np = p->np[tid];
                int lower = ( ty == 0 );
                int type = lower ? sp->bc[2] : sp->bc[3];
                if ( type != bcr ) continue;
                for ( int i = 0; i < np; i++ ) {
                    size_t g = off + i;
                    if ( lower ? ( p->ix[2*g+1] < 0 ) : ( p->ix[2*g+1] >= (int) p->nxy ) ) {
                        p->ix[2*g+1] += lower ? 1 : -1;
                        p->x[2*g+1] = -p->x[2*g+1];
                        p->u[3*g+1] = -p->u[3*g+1];
                    }
                }
            }
        }
    }
}

/* species.cpp:2348-2410 (dep_charge_kernel, tiles in order) */
static void species_deposit_charge( ospecies * sp, ogrid * charge ) {
    oparts * p = sp->part;
    const int ystride = charge->extx;
    const unsigned tv = charge->tile_vol;
    real * local = (real *) malloc( tv * sizeof( real ) );
    for ( unsigned tid = 0; tid < p->ntx * p->nty; tid++ ) {
        for ( unsigned i = 0; i < charge->extx * charge->exty; i++ ) local[i] = 0;
        real * c = local + charge->offset;
        size_t off = p->offset[tid]; int np = p->np[tid];
        for ( int i = 0; i < np; i++ ) {
            size_t g = off + i;
            const int idx = p->ix[2*g+1] * ystride + p->ix[2*g];
            const real s0x = (real) 0.5 - p->x[2*g], s1x = (real) 0.5 + p->x[2*g];
            const real s0y = (real) 0.5 - p->x[2*g+1], s1y = (real) 0.5 + p->x[2*g+1];
            c[idx]               += s0y * s0x * sp->q;
            c[idx + 1]           += s0y * s1x * sp->q;
            c[idx + ystride]     += s1y * s0x * sp->q;
            c[idx + 1 + ystride] += s1y * s1x * sp->q;
        }
        real * gc = gcell( charge, tid, 0 );
        for ( unsigned i = 0; i < charge->extx * charge->exty; i++ ) gc[i] += local[i];
    }
    free( local );
}

/* ======================================================================== */
/* EMF (emf.cpp) and Current (current.cpp)                                  */
/* ======================================================================== */
typedef struct { ogrid E, B; int bc[4]; real2 dx; double dt; int iter; omw mw; real2 box; } oemf;
typedef struct { ogrid J; real2 dx; double dt; omw mw; int bc[4]; int iter;
                 int ftype, fdir; unsigned forder; real2 box; } ocur;

#define MAX_SPECIES 16
struct osim {
    unsigned ntx, nty, nxx, nxy;
    real2 box; double dt; unsigned iter;
    oemf emf; ocur cur;
    int nsp; ospecies * sp[MAX_SPECIES];
};

/* emf.cpp:67-81 */
static void yee_b( const real3 * E, real3 * B, unsigned nxx, unsigned nxy, int ystride, real dtx, real dty ) {
    for ( int iy = -1; iy < (int) nxy + 1; iy++ )
        for ( int ix = -1; ix < (int) nxx + 1; ix++ ) {
            B[ix + iy*ystride].x += ( -dty * ( E[ix + (iy+1)*ystride].z - E[ix + iy*ystride].z ) );
            B[ix + iy*ystride].y += (  dtx * ( E[(ix+1) + iy*ystride].z - E[ix + iy*ystride].z ) );
            B[ix + iy*ystride].z += ( -dtx * ( E[(ix+1) + iy*ystride].y - E[ix + iy*ystride].y ) +
                                       dty * ( E[ix + (iy+1)*ystride].x - E[ix + iy*ystride].x ) );
        }
}

/* emf.cpp:93-110 */
static void yee_e( real3 * E, const real3 * B, unsigned nxx, unsigned nxy, int ystride, real dtx, real dty ) {
    for ( int iy = 0; iy < (int) nxy + 2; iy++ )
        for ( int ix = 0; ix < (int) nxx + 2; ix++ ) {
            E[ix + iy*ystride].x += ( +dty * ( B[ix + iy*ystride].z - B[ix + (iy-1)*ystride].z ) );
            E[ix + iy*ystride].y += ( -dtx * ( B[ix + iy*ystride].z - B[(ix-1) + iy*ystride].z ) );
            E[ix + iy*ystride].z += ( +dtx * ( B[ix + iy*ystride].y - B[(ix-1) + iy*ystride].y ) -
                                       dty * ( B[ix + iy*ystride].x - B[ix + (iy-1)*ystride].x ) );
        }
}

/* emf.cpp:486-506 */
static void yeeJ_e( real3 * E, const real3 * B, unsigned nxx, unsigned nxy, int ystride,
                    const real3 * J, int jstride, real dtx, real dty, real dt ) {
    for ( int iy = 0; iy < (int) nxy + 2; iy++ )
        for ( int ix = 0; ix < (int) nxx + 2; ix++ ) {
            E[ix + iy*ystride].x += ( +dty * ( B[ix + iy*ystride].z - B[ix + (iy-1)*ystride].z ) )
                                    - dt * J[ix + iy*jstride].x;
            E[ix + iy*ystride].y += ( -dtx * ( B[ix + iy*ystride].z - B[(ix-1) + iy*ystride].z ) )
                                    - dt * J[ix + iy*jstride].y;
            E[ix + iy*ystride].z += ( +dtx * ( B[ix + iy*ystride].y - B[(ix-1) + iy*ystride].y ) -
                                       dty * ( B[ix + iy*ystride].x - B[ix + (iy-1)*ystride].x ) )
                                    - dt * J[ix + iy*jstride].z;
        }
}

/* emf.cpp:207-303 */
static void emf_bcx( unsigned tx, real3 * E, real3 * B, unsigned nxx, unsigned extx, unsigned exty, const int * bc ) {
    const int ystride = extx;
    const int pec = 2, pmc = 3;
    const int nx = nxx;
    if ( tx == 0 ) {
        if ( bc[0] == pmc ) {
            for ( int idx = 0; idx < (int) exty; idx++ ) {
                const int iy = idx * ystride;
                E[-1 + iy].x = -E[0 + iy].x; E[-1 + iy].y = E[1 + iy].y; E[-1 + iy].z = E[1 + iy].z;
                B[-1 + iy].x = B[1 + iy].x; B[-1 + iy].y = -B[0 + iy].y; B[-1 + iy].z = -B[0 + iy].z;
            }
        } else if ( bc[0] == pec ) {
            for ( int idx = 0; idx < (int) exty; idx++ ) {
                const int iy = idx * ystride;
                E[-1 + iy].x = E[0 + iy].x; E[-1 + iy].y = -E[1 + iy].y; E[-1 + iy].z = -E[1 + iy].z;
                E[0 + iy].y = 0; E[0 + iy].z = 0;
                B[-1 + iy].x = -B[1 + iy].x; B[-1 + iy].y = B[0 + iy].y; B[-1 + iy].z = B[0 + iy].z;
                B[0 + iy].x = 0;
            }
        }
    } else {
        if ( bc[1] == pmc ) {
            for ( int idx = 0; idx < (int) exty; idx++ ) {
                const int iy = idx * ystride;
                E[nx + iy].x = -E[nx-1 + iy].x;
                E[nx+1 + iy].x = -E[nx-2 + iy].x; E[nx+1 + iy].y = E[nx-1 + iy].y; E[nx+1 + iy].z = E[nx-1 + iy].z;
                B[nx + iy].y = -B[nx-1 + iy].y; B[nx + iy].z = -B[nx-1 + iy].z;
                B[nx+1 + iy].x = B[nx-1 + iy].x; B[nx+1 + iy].y = -B[nx-2 + iy].y; B[nx+1 + iy].z = -B[nx-2 + iy].z;
            }
        } else if ( bc[1] == pec ) {
            for ( int idx = 0; idx < (int) exty; idx++ ) {
                const int iy = idx * ystride;
                E[nx + iy].x = E[nx-1 + iy].x; E[nx + iy].y = 0; E[nx + iy].z = 0;
                E[nx+1 + iy].x = E[nx-2 + iy].x; E[nx+1 + iy].y = -E[nx-1 + iy].y; E[nx+1 + iy].z = -E[nx-1 + iy].z;
                B[nx + iy].x = 0; B[nx + iy].y = B[nx-1 + iy].y; B[nx + iy].z = B[nx-1 + iy].z;
                B[nx+1 + iy].x = -B[nx-1 + iy].x; B[nx+1 + iy].y = B[nx-2 + iy].y; B[nx+1 + iy].z = B[nx-2 + iy].z;
            }
        }
    }
}

/* emf.cpp:315-410 (note the reference's nx.x in a few upper-y row indices, kept as is) */
static void emf_bcy( unsigned ty, real3 * E, real3 * B, unsigned nxx, unsigned nxy, unsigned extx, const int * bc ) {
    const int ystride = extx;
    const int pec = 2, pmc = 3;
    const int ny = nxy, nx = nxx;
    if ( ty == 0 ) {
        if ( bc[2] == pmc ) {
            for ( int ix = 0; ix < (int) extx; ix++ ) {
                E[ix - ystride].x = E[ix + ystride].x; E[ix - ystride].y = -E[ix].y; E[ix - ystride].z = E[ix + ystride].z;
                B[ix - ystride].x = -B[ix].x; B[ix - ystride].y = B[ix + ystride].y; B[ix - ystride].z = -B[ix].z;
            }
        } else if ( bc[2] == pec ) {
            for ( int ix = 0; ix < (int) extx; ix++ ) {
                E[ix - ystride].x = -E[ix + ystride].x; E[ix - ystride].y = E[ix].y; E[ix - ystride].z = -E[ix + ystride].z;
                E[ix].x = 0; E[ix].z = 0;
                B[ix - ystride].x = B[ix].x; B[ix - ystride].y = -B[ix + ystride].y; B[ix - ystride].z = B[ix].z;
                B[ix].y = 0;
            }
        }
    } else {
        if ( bc[3] == pmc ) {
            for ( int ix = 0; ix < (int) extx; ix++ ) {
                E[ix + ny*ystride].y = -E[ix + (ny-1)*ystride].y;
                E[ix + (ny+1)*ystride].x = E[ix + (ny-1)*ystride].x;
                E[ix + (ny+1)*ystride].y = -E[ix + (ny-2)*ystride].y;
                E[ix + (ny+1)*ystride].z = E[ix + (ny-1)*ystride].z;
                B[ix + ny*ystride].x = -B[ix + (ny-1)*ystride].x;
                B[ix + ny*ystride].z = -B[ix + (ny-1)*ystride].z;
                B[ix + (ny+1)*ystride].x = -B[ix + (nx-2)*ystride].x;
                B[ix + (ny+1)*ystride].y = B[ix + (nx-1)*ystride].y;
                B[ix + (ny+1)*ystride].z = -B[ix + (nx-2)*ystride].z;
            }
        } else if ( bc[3] == pec ) {
            for ( int ix = 0; ix < (int) extx; ix++ ) {
                E[ix + ny*ystride].x = 0;
                E[ix + ny*ystride].y = E[ix + (ny-1)*ystride].y;
                E[ix + ny*ystride].z = 0;
                E[ix + (ny+1)*ystride].x = -E[ix + (nx-1)*ystride].x;
                E[ix + (ny+1)*ystride].y = E[ix + (nx-2)*ystride].y;
                E[ix + (ny+1)*ystride].z = -E[ix + (nx-1)*ystride].z;
                B[ix + ny*ystride].x = B[ix + (ny-1)*ystride].x;
                B[ix + ny*ystride].y = 0;
                B[ix + ny*ystride].z = B[ix + (ny-1)*ystride].z;
                B[ix + (ny+1)*ystride].x = B[ix + (ny-2)*ystride].x;
                B[ix + (ny+1)*ystride].y = -B[ix + (ny-1)*ystride].y;
                B[ix + (ny+1)*ystride].z = B[ix + (ny-2)*ystride].z;
            }
        }
    }
}

/* emf.cpp:417-471 */
static void emf_process_bc( oemf * f ) {
    ogrid * E = &f->E; ogrid * B = &f->B;
    if ( f->bc[0] > 1 || f->bc[1] > 1 ) {
        for ( unsigned ty = 0; ty < E->nty; ty++ ) {
            unsigned txs[2] = { 0u, E->ntx - 1 };
            for ( int q = 0; q < 2; q++ ) {
                unsigned tid = ty * E->ntx + txs[q];
                emf_bcx( txs[q], (real3 *) gcell( E, tid, E->gxl ), (real3 *) gcell( B, tid, B->gxl ),
                         E->nxx, E->extx, E->exty, f->bc );
            }
        }
    }
    if ( f->bc[2] > 1 || f->bc[3] > 1 ) {
        unsigned tys[2] = { 0u, E->nty - 1 };
        for ( int q = 0; q < 2; q++ )
            for ( unsigned tx = 0; tx < E->ntx; tx++ ) {
                unsigned tid = tys[q] * E->ntx + tx;
                emf_bcy( tys[q], (real3 *) gcell( E, tid, E->gyl * E->extx ), (real3 *) gcell( B, tid, B->gyl * B->extx ),
                         E->nxx, E->nxy, E->extx, f->bc );
            }
    }
}

/* emf.cpp:120-129 */
static void emf_move_window( oemf * f ) {
    if ( mw_needs_move( &f->mw, f->iter * f->dt ) ) {
        grid_x_shift_left( &f->E, 1 );
        grid_x_shift_left( &f->B, 1 );
        mw_advance( &f->mw );
    }
}

/* emf.cpp:135-194 (no current) and 513-580 (with current) */
static void emf_advance( oemf * f, ocur * c ) {
    ogrid * E = &f->E; ogrid * B = &f->B;
    const unsigned tv = E->tile_vol;
    const int ystride = E->extx;
    const real dtx = (real) ( f->dt / f->dx.x ), dty = (real) ( f->dt / f->dx.y );
    const real dtx2 = dtx / 2, dty2 = dty / 2;
    real * El = (real *) malloc( (size_t) tv * 3 * sizeof( real ) );
    real * Bl = (real *) malloc( (size_t) tv * 3 * sizeof( real ) );
    for ( unsigned tid = 0; tid < E->ntx * E->nty; tid++ ) {
        memcpy( El, gcell( E, tid, 0 ), (size_t) tv * 3 * sizeof( real ) );
        memcpy( Bl, gcell( B, tid, 0 ), (size_t) tv * 3 * sizeof( real ) );
        real3 * tE = (real3 *) El + E->offset;
        real3 * tB = (real3 *) Bl + B->offset;
        yee_b( tE, tB, E->nxx, E->nxy, ystride, dtx2, dty2 );
        if ( c ) {
            const real3 * tJ = (const real3 *) gcell( &c->J, tid, c->J.offset );
            yeeJ_e( tE, tB, E->nxx, E->nxy, ystride, tJ, c->J.extx, dtx, dty, (real) f->dt );
        } else {
            yee_e( tE, tB, E->nxx, E->nxy, ystride, dtx, dty );
        }
        yee_b( tE, tB, E->nxx, E->nxy, ystride, dtx2, dty2 );
        memcpy( gcell( E, tid, 0 ), El, (size_t) tv * 3 * sizeof( real ) );
        memcpy( gcell( B, tid, 0 ), Bl, (size_t) tv * 3 * sizeof( real ) );
    }
    free( El ); free( Bl );
    grid_copy_to_gc( E );
    grid_copy_to_gc( B );
    emf_process_bc( f );
    f->iter += 1;
    if ( f->mw.active ) emf_move_window( f );
}

/* emf.cpp:662-713 (inner loop bound nx.y as in the reference) */
static void emf_energy( oemf * f, double * out ) {
    ogrid * E = &f->E; ogrid * B = &f->B;
    for ( int k = 0; k < 6; k++ ) out[k] = 0;
    for ( unsigned tid = 0; tid < E->ntx * E->nty; tid++ ) {
        double te[3] = { 0, 0, 0 }, tb[3] = { 0, 0, 0 };
        const real3 * Et = (const real3 *) gcell( E, tid, E->offset );
        const real3 * Bt = (const real3 *) gcell( B, tid, B->offset );
        for ( unsigned iy = 0; iy < E->nxy; iy++ )
            for ( unsigned ix = 0; ix < E->nxy; ix++ ) {
                real3 e = Et[iy * E->extx + ix], b = Bt[iy * E->extx + ix];
                te[0] += e.x * e.x; te[1] += e.y * e.y; te[2] += e.z * e.z;
                tb[0] += b.x * b.x; tb[1] += b.y * b.y; tb[2] += b.z * b.z;
            }
        for ( int k = 0; k < 3; k++ ) { out[k] += te[k]; out[3 + k] += tb[k]; }
    }
}

/* current.cpp:53-160 */
static void current_bcx( unsigned tx, real3 * J, unsigned nxx, unsigned extx, unsigned exty, const int * bc ) {
    const int ystride = extx, nx = nxx, refl = 2;
    if ( tx == 0 ) {
        if ( bc[0] == refl )
            for ( unsigned idx = 0; idx < exty; idx++ ) {
                const int iy = idx * ystride;
                real jx0 = -J[-1 + iy].x + J[0 + iy].x;
                real jy1 = J[-1 + iy].y + J[1 + iy].y;
                real jz1 = J[-1 + iy].z + J[1 + iy].z;
                J[-1 + iy].x = J[0 + iy].x = jx0;
                J[-1 + iy].y = J[1 + iy].y = jy1;
                J[-1 + iy].z = J[1 + iy].z = jz1;
            }
    } else {
        if ( bc[1] == refl )
            for ( unsigned idx = 0; idx < exty; idx++ ) {
                const int iy = idx * ystride;
                real jx0 = J[nx-1 + iy].x - J[nx + 0 + iy].x;
                real jy1 = J[nx-1 + iy].y + J[nx + 1 + iy].y;
                real jz1 = J[nx-1 + iy].z + J[nx + 1 + iy].z;
                J[nx-1 + iy].x = J[nx + 0 + iy].x = jx0;
                J[nx-1 + iy].y = J[nx + 1 + iy].y = jy1;
                J[nx-1 + iy].z = J[nx + 1 + iy].z = jz1;
            }
    }
}
static void current_bcy( unsigned ty, real3 * J, unsigned nxy, unsigned extx, const int * bc ) {
    const int ystride = extx, ny = nxy, refl = 2;
    if ( ty == 0 ) {
        if ( bc[2] == refl )
            for ( int ix = 0; ix < (int) extx; ix++ ) {
                real jx1 = J[ix - ystride].x + J[ix + ystride].x;
                real jy0 = -J[ix - ystride].y + J[ix].y;
                real jz1 = J[ix - ystride].z + J[ix + ystride].z;
                J[ix - ystride].x = J[ix + ystride].x = jx1;
                J[ix - ystride].y = J[ix].y = jy0;
                J[ix - ystride].z = J[ix + ystride].z = jz1;
            }
    } else {
        if ( bc[3] == refl )
            for ( int ix = 0; ix < (int) extx; ix++ ) {
                real jx1 = J[ix + (ny-1)*ystride].x + J[ix + (ny+1)*ystride].x;
                real jy0 = J[ix + (ny-1)*ystride].y - J[ix + ny*ystride].y;
                real jz1 = J[ix + (ny-1)*ystride].z + J[ix + (ny+1)*ystride].z;
                J[ix + (ny-1)*ystride].x = J[ix + (ny+1)*ystride].x = jx1;
                J[ix + (ny-1)*ystride].y = J[ix + ny*ystride].y = jy0;
                J[ix + (ny-1)*ystride].z = J[ix + (ny+1)*ystride].z = jz1;
            }
    }
}

/* current.cpp:166-221 */
static void current_process_bc( ocur * c ) {
    ogrid * J = &c->J;
    if ( c->bc[0] > 1 || c->bc[1] > 1 )
        for ( unsigned ty = 0; ty < J->nty; ty++ ) {
            unsigned txs[2] = { 0u, J->ntx - 1 };
            for ( int q = 0; q < 2; q++ )
                current_bcx( txs[q], (real3 *) gcell( J, ty * J->ntx + txs[q], J->gxl ), J->nxx, J->extx, J->exty, c->bc );
        }
    if ( c->bc[2] > 1 || c->bc[3] > 1 ) {
        unsigned tys[2] = { 0u, J->nty - 1 };
        for ( int q = 0; q < 2; q++ )
            for ( unsigned tx = 0; tx < J->ntx; tx++ )
                current_bcy( tys[q], (real3 *) gcell( J, tys[q] * J->ntx + tx, J->gyl * J->extx ), J->nxy, J->extx, c->bc );
    }
}

/* current.cpp:227-246 */
static void current_advance( ocur * c ) {
    grid_add_from_gc( &c->J );
    grid_copy_to_gc( &c->J );
    current_process_bc( c );
    filter_apply( &c->J, c->ftype, c->fdir, c->forder );
    c->iter++;
    if ( mw_needs_move( &c->mw, c->iter * c->dt ) ) mw_advance( &c->mw );
}

/* ======================================================================== */
/* Species lifecycle (species.cpp:1693-1842, 2051-2128)                     */
/* ======================================================================== */
static void species_initialize( ospecies * sp, real2 box, unsigned ntx, unsigned nty,
                                unsigned nxx, unsigned nxy, double dt, int id ) {
    sp->box = box;
    sp->dt = (real) dt;
    sp->id = id;
    /* q = copysign( n0, m_q ) / ( ppc.x * ppc.y ) */
    float n0 = fabsf( sp->dens_p[0] );
    if ( sp->dens_type == 0 ) n0 = 0.f;
    sp->q = (real) ( copysignf( n0, sp->m_q ) / (float) ( sp->ppcx * sp->ppcy ) );
    real dimsx = (real) (float) ( nxx * ntx ), dimsy = (real) (float) ( nxy * nty );
    sp->dx.x = box.x / dimsx; sp->dx.y = box.y / dimsy;
    uint32_t max_part = (uint32_t) ( 1.2 * (float) ( nxx * ntx ) * (float) ( nxy * nty ) * sp->ppcx * sp->ppcy );
    sp->part = parts_new( ntx, nty, nxx, nxy, max_part );
    sp->part->perx = ( sp->bc[0] == 1 ); sp->part->pery = ( sp->bc[2] == 1 );
    sp->tmp = parts_new( ntx, nty, nxx, nxy, max_part );
    sort_init( &sp->sort, ntx * nty, max_part );
    sp->np_inj = (int *) calloc( ntx * nty, sizeof( int ) );
    sp->d_energy = 0; sp->d_nmove = 0; sp->iter = 0;
    unsigned range[4] = { 0, nxx * ntx - 1, 0, nxy * nty - 1 };
    species_np_inject( sp, range, sp->np_inj );
    uint32_t off = 0;
    for ( unsigned i = 0; i < ntx * nty; i++ ) { sp->part->offset[i] = off; off += sp->np_inj[i]; }
    species_inject( sp, range );
    species_udist( sp );
}

static void species_free( ospecies * sp ) {
    parts_free( sp->part ); parts_free( sp->tmp ); sort_free( &sp->sort ); free( sp->np_inj ); free( sp );
}

/* species.cpp:2051-2068 */
static void species_advance( osim * s, ospecies * sp ) {
    species_push( sp, &s->emf.E, &s->emf.B );
    species_move( sp, &s->cur.J, 0, 0, 1 );
    species_process_bc( sp );
    sp->iter++;
    tile_sort( sp->part, sp->tmp, &sp->sort, NULL );
}

/* species.cpp:2083-2128 */
static void species_advance_mov_window( osim * s, ospecies * sp ) {
    species_push( sp, &s->emf.E, &s->emf.B );
    if ( mw_needs_move( &sp->mw, (double) ( ( sp->iter + 1 ) * sp->dt ) ) ) {
        species_move( sp, &s->cur.J, -1, 0, 1 );
        species_process_bc( sp );
        unsigned gx = sp->part->nxx * sp->part->ntx, gy = sp->part->nxy * sp->part->nty;
        unsigned range[4] = { gx - 1, gx - 1, 0, gy - 1 };
        species_np_inject( sp, range, sp->np_inj );
        tile_sort( sp->part, sp->tmp, &sp->sort, sp->np_inj );
        species_inject( sp, range );
        mw_advance( &sp->mw );
    } else {
        species_move( sp, &s->cur.J, 0, 0, 1 );
        species_process_bc( sp );
        tile_sort( sp->part, sp->tmp, &sp->sort, NULL );
    }
    sp->iter++;
}

/* ======================================================================== */
/* Lasers (laser.h:46-64, laser.cpp)                                        */
/* ======================================================================== */
typedef struct { float start, fwhm, rise, flat, fall, a0, omega0, polarization, cos_pol, sin_pol;
                 unsigned filter; float W0, focus, axis; } olaser;

/* laser.h:46-64 */
static float lon_env( const olaser * l, float z ) {
    if ( z > l->start ) return 0.0f;
    else if ( z > l->start - l->rise ) {
        float csi = z - l->start;
        float e = (float) sin( M_PI_2 * csi / l->rise );
        return e * e;
    } else if ( z > l->start - ( l->rise + l->flat ) ) return 1.0f;
    else if ( z > l->start - ( l->rise + l->flat + l->fall ) ) {
        float csi = z - ( l->start - l->rise - l->flat - l->fall );
        float e = (float) sin( M_PI_2 * csi / l->fall );
        return e * e;
    }
    return 0.0f;
}

/* laser.cpp:174-207 */
static int laser_validate( olaser * l, int gaussian ) {
    if ( l->a0 <= 0 ) return -1;
    if ( l->omega0 <= 0 ) return -1;
    if ( l->fwhm > 0 ) { l->rise = l->fwhm; l->fall = l->fwhm; l->flat = 0.f; }
    else {
        if ( l->rise <= 0 ) return -1;
        if ( l->flat < 0 ) return -1;
        if ( l->fall <= 0 ) return -1;
    }
    if ( gaussian && l->W0 <= 0 ) return -1;
    return 0;
}

/* laser.cpp:318-330 (atan2 on floats resolves to the double overload) */
static float gauss_phase( float omega0, float W0, float z, float r ) {
    const float z0 = omega0 * ( W0 * W0 ) / 2;
    const float rho2 = r * r;
    const float curv = rho2 * z / ( z0 * z0 + z * z );
    const float rWl2 = ( z0 * z0 ) / ( z0 * z0 + z * z );
    const float gouy_shift = (float) atan2( (double) z, (double) z0 );
    return sqrtf( sqrtf( rWl2 ) ) * expf( -rho2 * rWl2 / ( W0 * W0 ) ) * cosf( omega0 * ( z + curv ) - gouy_shift );
}

/* laser.cpp:20-70 */
static void div_corr_x( ogrid * E, ogrid * B, float dxx, float dxy ) {
    const int ntx = E->ntx, nty = E->nty, nxx = E->nxx, nxy = E->nxy;
    const int ystride = E->extx;
    const double dx_dy = ( (double) dxx ) / ( (double) dxy );
    double * divEx = (double *) malloc( nxy * sizeof( double ) );
    double * divBx = (double *) malloc( nxy * sizeof( double ) );
    for ( int ty = 0; ty < nty; ty++ ) {
        for ( int iy = 0; iy < nxy; iy++ ) divEx[iy] = divBx[iy] = 0;
        for ( int tx = ntx - 1; tx >= 0; tx-- ) {
            unsigned tid = ty * ntx + tx;
            real3 * tE = (real3 *) gcell( E, tid, E->offset );
            real3 * tB = (real3 *) gcell( B, tid, B->offset );
            for ( int iy = 0; iy < nxy; iy++ ) {
                double a = divEx[iy], b = divBx[iy];
                for ( int ix = nxx - 1; ix >= 0; ix-- ) {
                    a += dx_dy * ( tE[ix+1 + iy*ystride].y - tE[ix+1 + (iy-1)*ystride].y );
                    tE[ix + iy*ystride].x = (real) a;
                    b += dx_dy * ( tB[ix + (iy+1)*ystride].y - tB[ix + iy*ystride].y );
                    tB[ix + iy*ystride].x = (real) b;
                }
                divEx[iy] = a; divBx[iy] = b;
            }
        }
    }
    free( divEx ); free( divBx );
}

/* laser.cpp:225-296 (plane wave), 341-443 (gaussian), laser.h:85-99 (add) */
static int laser_add( osim * s, int type, olaser * l ) {
    if ( laser_validate( l, type == 1 ) < 0 ) return -1;
    if ( l->cos_pol == 0 && l->sin_pol == 0 ) {
        l->cos_pol = cosf( l->polarization );
        l->sin_pol = sinf( l->polarization );
    }
    ogrid tE, tB;
    ogrid * E = &s->emf.E;
    grid_init( &tE, E->ntx, E->nty, E->nxx, E->nxy, E->gxl, E->gxu, E->gyl, E->gyu, 3 );
    grid_init( &tB, E->ntx, E->nty, E->nxx, E->nxy, E->gxl, E->gxu, E->gyl, E->gyu, 3 );
    float dxx = s->box.x / ( E->nxx * E->ntx ), dxy = s->box.y / ( E->nxy * E->nty );
    const int ystride = E->extx;
    const float amp = l->omega0 * l->a0;
    for ( unsigned ty = 0; ty < E->nty; ty++ ) for ( unsigned tx = 0; tx < E->ntx; tx++ ) {
        unsigned tid = ty * E->ntx + tx;
        real3 * pE = (real3 *) gcell( &tE, tid, E->offset );
        real3 * pB = (real3 *) gcell( &tB, tid, E->offset );
        const int ix0 = tx * E->nxx, iy0 = ty * E->nxy;
        for ( unsigned iy = 0; iy < E->nxy; iy++ )
            for ( unsigned ix = 0; ix < E->nxx; ix++ ) {
                const float z = ( ix0 + ix ) * dxx;
                const float z_2 = ( ix0 + ix + 0.5 ) * dxx;
                const float lenv = amp * lon_env( l, z ), lenv_2 = amp * lon_env( l, z_2 );
                real3 e, b;
                if ( type == 0 ) {
                    const float k = l->omega0;
                    e.x = 0; e.y = +lenv * cosf( k * z ) * l->cos_pol; e.z = +lenv * cosf( k * z ) * l->sin_pol;
                    b.x = 0; b.y = -lenv_2 * cosf( k * z_2 ) * l->sin_pol; b.z = +lenv_2 * cosf( k * z_2 ) * l->cos_pol;
                } else {
                    const float r = ( iy0 + iy ) * dxy - l->axis;
                    const float r_2 = ( iy0 + iy + 0.5 ) * dxy - l->axis;
                    e.x = 0;
                    e.y = +lenv * gauss_phase( l->omega0, l->W0, z - l->focus, r_2 ) * l->cos_pol;
                    e.z = +lenv * gauss_phase( l->omega0, l->W0, z - l->focus, r ) * l->sin_pol;
                    b.x = 0;
                    b.y = -lenv_2 * gauss_phase( l->omega0, l->W0, z_2 - l->focus, r ) * l->sin_pol;
                    b.z = +lenv_2 * gauss_phase( l->omega0, l->W0, z_2 - l->focus, r_2 ) * l->cos_pol;
                }
                pE[ix + iy * ystride] = e;
                pB[ix + iy * ystride] = b;
            }
    }
    /* the temporary laser grids are new grid objects, hence periodic (grid.h:79) */
    grid_copy_to_gc( &tE );
    grid_copy_to_gc( &tB );
    if ( l->filter > 0 ) {
        filter_apply( &tE, 2, 0, l->filter );
        filter_apply( &tB, 2, 0, l->filter );
    }
    if ( type == 1 ) div_corr_x( &tE, &tB, dxx, dxy );
    size_t n = grid_cells( E ) * 3;
    for ( size_t i = 0; i < n; i++ ) { s->emf.E.buf[i] += tE.buf[i]; s->emf.B.buf[i] += tB.buf[i]; }
    grid_free( &tE ); grid_free( &tB );
    return 0;
}

/* ======================================================================== */
/* Public entry points                                                      */
/* ======================================================================== */

/* simulation.h:39-46, emf.cpp:16-54, current.cpp:14-42 */
osim * osim_create( unsigned ntx, unsigned nty, unsigned nxx, unsigned nxy, float boxx, float boxy, double dt ) {
    float dxx = boxx / ( nxx * ntx ), dxy = boxy / ( nxy * nty );
    float cour = sqrtf( 1.0f / ( 1.0f / ( dxx * dxx ) + 1.0f / ( dxy * dxy ) ) );
    if ( dt >= cour ) return NULL;
    osim * s = (osim *) calloc( 1, sizeof( osim ) );
    s->ntx = ntx; s->nty = nty; s->nxx = nxx; s->nxy = nxy;
    s->box.x = boxx; s->box.y = boxy; s->dt = dt;
    grid_init( &s->emf.E, ntx, nty, nxx, nxy, 1, 2, 1, 2, 3 );
    grid_init( &s->emf.B, ntx, nty, nxx, nxy, 1, 2, 1, 2, 3 );
    s->emf.dx.x = dxx; s->emf.dx.y = dxy; s->emf.dt = dt; s->emf.box = s->box;
    for ( int k = 0; k < 4; k++ ) s->emf.bc[k] = 1;
    grid_init( &s->cur.J, ntx, nty, nxx, nxy, 1, 2, 1, 2, 3 );
    s->cur.dx = s->emf.dx; s->cur.dt = dt; s->cur.box = s->box;
    for ( int k = 0; k < 4; k++ ) s->cur.bc[k] = 1;
    return s;
}

void osim_destroy( osim * s ) {
    if ( !s ) return;
    grid_free( &s->emf.E ); grid_free( &s->emf.B ); grid_free( &s->cur.J );
    for ( int i = 0; i < s->nsp; i++ ) species_free( s->sp[i] );
    free( s );
}

/* species.cpp:1693-1718 + simulation.h:68-71 */
int osim_add_species( osim * s, float m_q, unsigned ppcx, unsigned ppcy, int dens_type, const float * dens_p,
                      int udist_type, const float * uth, const float * ufl, int npmin, int push_type, const int * bc ) {
    if ( s->nsp >= MAX_SPECIES || m_q == 0 || ppcx < 1 || ppcy < 1 ) return -1;
    ospecies * sp = (ospecies *) calloc( 1, sizeof( ospecies ) );
    sp->m_q = m_q; sp->ppcx = ppcx; sp->ppcy = ppcy;
    sp->dens_type = dens_type;
    for ( int k = 0; k < 5; k++ ) sp->dens_p[k] = dens_p ? dens_p[k] : ( k == 0 ? 1.0f : 0.0f );
    sp->udist_type = udist_type;
    for ( int k = 0; k < 3; k++ ) { sp->uth[k] = uth ? uth[k] : 0; sp->ufl[k] = ufl ? ufl[k] : 0; }
    sp->npmin = npmin;
    sp->push_type = push_type;
    for ( int k = 0; k < 4; k++ ) sp->bc[k] = bc ? bc[k] : 1;
    s->sp[s->nsp++] = sp;
    species_initialize( sp, s->box, s->ntx, s->nty, s->nxx, s->nxy, s->dt, s->nsp );
    return s->nsp - 1;
}

/* simulation.h:56-62, emf.h:137-148, current.h:122-133, species.h:254-265 */
void osim_set_moving_window( osim * s ) {
    if ( s->emf.iter == 0 ) {
        mw_init( &s->emf.mw, s->emf.dx.x );
        s->emf.bc[0] = s->emf.bc[1] = 0;
        s->emf.E.perx = s->emf.B.perx = 0;
    }
    if ( s->cur.iter == 0 ) {
        mw_init( &s->cur.mw, s->cur.dx.x );
        s->cur.bc[0] = s->cur.bc[1] = 0;
        s->cur.J.perx = 0;
    }
    for ( int i = 0; i < s->nsp; i++ ) {
        ospecies * sp = s->sp[i];
        if ( sp->iter == 0 ) {
            mw_init( &sp->mw, sp->dx.x );
            sp->bc[0] = sp->bc[1] = 0;
            sp->part->perx = 0;
        }
    }
}

void osim_emf_set_bc( osim * s, const int * bc ) {
    for ( int k = 0; k < 4; k++ ) s->emf.bc[k] = bc[k];
    s->emf.E.perx = s->emf.B.perx = ( bc[0] == 1 );
    s->emf.E.pery = s->emf.B.pery = ( bc[2] == 1 );
}
void osim_current_set_bc( osim * s, const int * bc ) {
    for ( int k = 0; k < 4; k++ ) s->cur.bc[k] = bc[k];
    s->cur.J.perx = ( bc[0] == 1 );
    s->cur.J.pery = ( bc[2] == 1 );
}
void osim_current_set_filter( osim * s, int type, int dir, unsigned order ) {
    s->cur.ftype = type; s->cur.fdir = dir; s->cur.forder = order;
}
int osim_add_laser( osim * s, int type, const float * p ) {
    olaser l;
    l.start = p[0]; l.fwhm = p[1]; l.rise = p[2]; l.flat = p[3]; l.fall = p[4];
    l.a0 = p[5]; l.omega0 = p[6]; l.polarization = p[7]; l.cos_pol = p[8]; l.sin_pol = p[9];
    l.filter = (unsigned) p[10]; l.W0 = p[11]; l.focus = p[12]; l.axis = p[13];
    return laser_add( s, type, &l );
}

/* simulation.h:90-107 */
void osim_advance( osim * s, int n ) {
    for ( int k = 0; k < n; k++ ) {
        grid_zero( &s->cur.J );
        for ( int i = 0; i < s->nsp; i++ ) species_advance( s, s->sp[i] );
        current_advance( &s->cur );
        emf_advance( &s->emf, &s->cur );
        s->iter++;
    }
}

/* simulation.h:113-130 */
void osim_advance_mov_window( osim * s, int n ) {
    for ( int k = 0; k < n; k++ ) {
        grid_zero( &s->cur.J );
        for ( int i = 0; i < s->nsp; i++ ) species_advance_mov_window( s, s->sp[i] );
        current_advance( &s->cur );
        emf_advance( &s->emf, &s->cur );
        s->iter++;
    }
}

void osim_current_zero( osim * s ) { grid_zero( &s->cur.J ); }
void osim_current_advance( osim * s ) { current_advance( &s->cur ); }
void osim_emf_advance( osim * s, int with_current ) { emf_advance( &s->emf, with_current ? &s->cur : NULL ); }
void osim_species_advance( osim * s, int sp ) { species_advance( s, s->sp[sp] ); }
/* Species::advance() free streaming (species.cpp:1998-2012): move, walls, sort */
void osim_species_advance_free( osim * s, int sp ) {
    ospecies * p = s->sp[sp];
    species_move( p, &s->cur.J, 0, 0, 0 );
    species_process_bc( p );
    tile_sort( p->part, p->tmp, &p->sort, NULL );
    p->iter++;
}
void osim_species_push( osim * s, int sp ) { species_push( s->sp[sp], &s->emf.E, &s->emf.B ); }
void osim_species_move( osim * s, int sp ) { species_move( s->sp[sp], &s->cur.J, 0, 0, 1 ); }
void osim_species_process_bc( osim * s, int sp ) { species_process_bc( s->sp[sp] ); }
void osim_species_tile_sort( osim * s, int sp ) {
    ospecies * p = s->sp[sp];
    tile_sort( p->part, p->tmp, &p->sort, NULL );
}

/* Test support, no reference counterpart: puts every clock of the
 * simulation -- its own iteration count and those of the fields, the current
 * and each species, and their moving windows' move counts -- where k steps of
 * osim_advance / osim_advance_mov_window from t = 0 leave them, doing none of
 * the steps' work.  The rules are the ones the steps apply:
 * species_advance_mov_window (species.cpp:2083-2128), current_advance
 * (current.cpp:227-246), emf_advance + emf_move_window (emf.cpp:120-129,
 * 575-579).  Used to continue from a state taken at step k. */
void osim_set_clock( osim * s, unsigned k ) {
    oemf * f = &s->emf; ocur * c = &s->cur;
    f->iter = 0; f->mw.n_move = 0;
    c->iter = 0; c->mw.n_move = 0;
    for ( int i = 0; i < s->nsp; i++ ) { s->sp[i]->iter = 0; s->sp[i]->mw.n_move = 0; }
    for ( unsigned n = 0; n < k; n++ ) {
        for ( int i = 0; i < s->nsp; i++ ) {
            ospecies * sp = s->sp[i];
            if ( mw_needs_move( &sp->mw, (double) ( ( sp->iter + 1 ) * sp->dt ) ) ) mw_advance( &sp->mw );
            sp->iter++;
        }
        c->iter++;
        if ( mw_needs_move( &c->mw, c->iter * c->dt ) ) mw_advance( &c->mw );
        f->iter += 1;
        if ( f->mw.active && mw_needs_move( &f->mw, f->iter * f->dt ) ) mw_advance( &f->mw );
    }
    s->iter = k;
}

unsigned osim_iter( osim * s ) { return s->iter; }
uint64_t osim_nmove( osim * s ) {
    uint64_t n = 0;
    for ( int i = 0; i < s->nsp; i++ ) n += s->sp[i]->d_nmove;
    return n;
}

/* species.h:365-368 */
double osim_species_energy( osim * s, int sp ) {
    ospecies * p = s->sp[sp];
    return p->d_energy * p->q * p->m_q * p->dx.x * p->dx.y;
}
void osim_emf_energy( osim * s, double * out6 ) { emf_energy( &s->emf, out6 ); }

uint64_t osim_species_tiles( osim * s, int sp, int * np, int * offset ) {
    oparts * p = s->sp[sp]->part;
    unsigned nt = p->ntx * p->nty;
    if ( np ) memcpy( np, p->np, nt * sizeof( int ) );
    if ( offset ) memcpy( offset, p->offset, nt * sizeof( int ) );
    return parts_np_total( p );
}
uint32_t osim_species_max_part( osim * s, int sp ) { return s->sp[sp]->part->max_part; }

void osim_species_get( osim * s, int sp, int * ix, real * x, real * u ) {
    oparts * p = s->sp[sp]->part;
    size_t k = 0;
    for ( unsigned t = 0; t < p->ntx * p->nty; t++ )
        for ( int i = 0; i < p->np[t]; i++, k++ ) {
            size_t g = (size_t) p->offset[t] + i;
            ix[2*k] = p->ix[2*g]; ix[2*k+1] = p->ix[2*g+1];
            x[2*k] = p->x[2*g]; x[2*k+1] = p->x[2*g+1];
            u[3*k] = p->u[3*g]; u[3*k+1] = p->u[3*g+1]; u[3*k+2] = p->u[3*g+2];
        }
}

int osim_species_set( osim * s, int sp, const int * np, const int * ix, const real * x, const real * u ) {
    oparts * p = s->sp[sp]->part;
    size_t total = 0;
    for ( unsigned t = 0; t < p->ntx * p->nty; t++ ) total += np[t];
    if ( total > p->max_part ) return -1;
    size_t off = 0;
    for ( unsigned t = 0; t < p->ntx * p->nty; t++ ) { p->offset[t] = off; p->np[t] = np[t]; off += np[t]; }
    memcpy( p->ix, ix, total * 2 * sizeof( int ) );
    memcpy( p->x, x, total * 2 * sizeof( real ) );
    memcpy( p->u, u, total * 3 * sizeof( real ) );
    return 0;
}

static ogrid * pick( osim * s, int which ) {
    return which == 0 ? &s->emf.E : which == 1 ? &s->emf.B : &s->cur.J;
}
uint64_t osim_grid_size( osim * s, int which ) { return grid_cells( pick( s, which ) ); }
void osim_grid_get( osim * s, int which, real * out ) {
    ogrid * g = pick( s, which );
    memcpy( out, g->buf, grid_cells( g ) * 3 * sizeof( real ) );
}
void osim_grid_set( osim * s, int which, const real * in ) {
    ogrid * g = pick( s, which );
    memcpy( g->buf, in, grid_cells( g ) * 3 * sizeof( real ) );
}

/* species.cpp:2486-2511 (deposit + add_from_gc + gather), dense output */
/*
 * Species::dep_phasespace, 1D (species.cpp:2631-2709) and 2D (2863-3022),
 * with dep_pha1_kernel (2579-2620) / dep_pha2_kernel (2786-2852): tiles in
 * order, particles in order, serial sums.  The normalisation calls fabs() on
 * the float charge without std::; in the reference build that is C's double
 * fabs, so the normalisation is evaluated in double and rounded once.
 * Returns -1 for an invalid 2D pair (quant1 <= quant0).
 */
static real pha_value( int q, int shiftx, int shifty, const int * ix, const real * x, const real * u ) {
    switch ( q ) {
    case 0:  return ( shiftx + ix[0] ) + ( x[0] + (real) 0.5 );
    case 1:  return ( shifty + ix[1] ) + ( x[1] + (real) 0.5 );
    case 2:  return u[0];
    case 3:  return u[1];
    default: return u[2];
    }
}

int osim_species_phasespace( osim * s, int sp, int q0, const float * range0, int size0,
                             int q1, const float * range1, int size1, real * out ) {
    ospecies * p = s->sp[sp];
    oparts * part = p->part;
    const int two = q1 >= 0;
    if ( two && q0 >= q1 ) return -1;
    real r0x = range0[0], r0y = range0[1], r1x = 0, r1y = 0;
    if ( two ) { r1x = range1[0]; r1y = range1[1]; }
    real norm;
    if ( !two ) norm = fabs( (double) p->q ) * ( p->dx.x * p->dx.y ) * (unsigned) size0 / ( r0y - r0x );
    else norm = fabs( (double) p->q ) * ( p->dx.x * p->dx.y ) * ( (unsigned) size0 / ( r0y - r0x ) ) *
                ( (unsigned) size1 / ( r1y - r1x ) );
    if ( q0 == 0 ) { r0y /= p->dx.x; r0x /= p->dx.x; }
    if ( q0 == 1 ) { r0y /= p->dx.y; r0x /= p->dx.y; }
    if ( two && q1 == 1 ) { r1y /= p->dx.y; r1x /= p->dx.y; }
    const size_t nbins = (size_t) size0 * ( two ? size1 : 1 );
    for ( size_t i = 0; i < nbins; i++ ) out[i] = 0;
    const real rdx0 = size0 / ( r0y - r0x ), rdx1 = two ? size1 / ( r1y - r1x ) : 0;
    for ( unsigned ty = 0; ty < part->nty; ty++ )
        for ( unsigned tx = 0; tx < part->ntx; tx++ ) {
            const int tid = ty * part->ntx + tx;
            const int shiftx = tx * part->nxx, shifty = ty * part->nxy;
            for ( int i = 0; i < part->np[tid]; i++ ) {
                const size_t g = (size_t) part->offset[tid] + i;
                const int * ix = part->ix + 2 * g; const real * x = part->x + 2 * g; const real * u = part->u + 3 * g;
                const real n0 = ( pha_value( q0, shiftx, shifty, ix, x, u ) - r0x ) * rdx0 - (real) 0.5;
                const int k0 = (int) ( n0 + 1 ) - 1;
                const real w0 = n0 - k0;
                if ( !two ) {
                    if ( ( k0 >= 0 ) && ( k0 < size0 - 1 ) ) out[k0] += ( 1 - w0 ) * norm;
                    if ( ( k0 + 1 >= 0 ) && ( k0 + 1 < size0 - 1 ) ) out[k0 + 1] += w0 * norm;
                } else {
                    const real n1 = ( pha_value( q1, shiftx, shifty, ix, x, u ) - r1x ) * rdx1 - (real) 0.5;
                    const int k1 = (int) ( n1 + 1 ) - 1;
                    const real w1 = n1 - k1;
                    const int a0 = ( k0 >= 0 ) && ( k0 < size0 - 1 ), b0 = ( k0 + 1 >= 0 ) && ( k0 + 1 < size0 - 1 );
                    const int a1 = ( k1 >= 0 ) && ( k1 < size1 - 1 ), b1 = ( k1 + 1 >= 0 ) && ( k1 + 1 < size1 - 1 );
                    if ( a0 && a1 ) out[k1 * size0 + k0]           += ( 1 - w0 ) * ( 1 - w1 ) * norm;
                    if ( b0 && a1 ) out[k1 * size0 + k0 + 1]       += w0 * ( 1 - w1 ) * norm;
                    if ( a0 && b1 ) out[( k1 + 1 ) * size0 + k0]   += ( 1 - w0 ) * w1 * norm;
                    if ( b0 && b1 ) out[( k1 + 1 ) * size0 + k0 + 1] += w0 * w1 * norm;
                }
            }
        }
    return 0;
}

void osim_species_charge( osim * s, int sp, real * out ) {
    ospecies * p = s->sp[sp];
    ogrid ch;
    grid_init( &ch, s->ntx, s->nty, s->nxx, s->nxy, 0, 1, 0, 1, 1 );
    species_deposit_charge( p, &ch );
    grid_add_from_gc( &ch );
    const unsigned dimx = s->ntx * s->nxx;
    for ( unsigned tid = 0; tid < s->ntx * s->nty; tid++ ) {
        unsigned tx = tid % s->ntx, ty = tid / s->ntx;
        const real * d = gcell( &ch, tid, ch.offset );
        for ( unsigned iy = 0; iy < s->nxy; iy++ )
            for ( unsigned ix = 0; ix < s->nxx; ix++ )
                out[( ty * s->nxy + iy ) * dimx + tx * s->nxx + ix] = d[iy * ch.extx + ix];
    }
    grid_free( &ch );
}
